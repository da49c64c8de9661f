// Heterogeneous batch: several worlds (articulated chains and trees, free-
// body piles of any body count) advanced by ONE persistent launch per
// horizon of control steps.  Every resident warp repeatedly claims the next
// work item from a device queue (an atomic counter over a claim-ordered
// item list) and advances that environment of that world through the
// horizon with the world's own device code path, until the queue is empty.
// Environments are independent, so no environment waits for another between
// control steps.  The claim order is the host's choice (longest items first
// by default), so the long-running environments start first and short
// ones fill the tail.
#pragma once

#include <cstddef>
#include <cstdint>

#include <cuda_runtime.h>

#include "device_model.h"
#include "layout.h"
#include "scene.h"

namespace numi {

enum MixKind : std::int32_t { kMixFreeMotion = 0, kMixContact = 1, kMixScene = 2 };

// One world of a batch at one control step: the launch parameters its own
// kernel would get (this step's actions, reset masks and outputs).
struct MixWorld {
    std::int32_t kind;  // MixKind
    std::int32_t envs;
    StepParams step;    // articulated worlds
    WarpLayout layout;  // articulated worlds: the per-warp shared-memory layout
    SceneParams scene;  // free-body worlds
};

// Work item: world index in bits 24-31, environment slot in bits 0-23.
constexpr int kMixWorldShift = 24;
constexpr std::uint32_t kMixEnvMask = (1u << kMixWorldShift) - 1u;
constexpr int kMixMaxWorlds = 256;

// Shared memory one warp needs for an articulated layout (floats): the
// layout copy plus its sections.
int mix_articulated_warp_floats(const WarpLayout& layout);
// ... and for a free-body world.
int mix_scene_warp_floats();

// Kernel families: the fused kernel runs every item; the per-family
// kernels run one family's items at that family's own register budget.
// kMixFamilySceneConvex is the free-body kernel with the support-mapped
// (GJK / EPA) narrowphase, for batches with such pairs.
enum MixFamily : int { kMixFamilyFused = 0, kMixFamilyArticulated = 1, kMixFamilyScene = 2, kMixFamilySceneConvex = 3 };

cudaError_t configure_mix_kernel(int family, size_t max_dynamic_smem);
cudaError_t mix_occupancy(int family, int warps_per_block, size_t smem_per_block, int* blocks_per_sm);
// `steps` control steps of every item: `worlds` (device) holds the
// descriptors [steps][world_count], `items` (device) the claim order,
// `next_item` (device) a counter that must be zero at launch.  A claimed
// environment runs all its steps before the warp claims the next one.
// The scene family runs one warp per CTA.
cudaError_t launch_mix_horizon(int family, const MixWorld* worlds, int world_count, int steps, const std::uint32_t* items,
                               int item_count, unsigned* next_item, int warps_per_block, int smem_floats_per_warp, int grid,
                               cudaStream_t stream);

// The free-body family kernels (scene_step.cu); `convex`: the instance with
// the support-mapped narrowphase.
cudaError_t configure_mix_scene_kernel(bool convex, size_t max_dynamic_smem);
cudaError_t mix_scene_occupancy(bool convex, int warps_per_block, size_t smem_per_block, int* blocks_per_sm);
cudaError_t launch_mix_scene(bool convex, const MixWorld* worlds, int world_count, int steps, const std::uint32_t* items,
                             int item_count, unsigned* next_item, int warps_per_block, int smem_floats_per_warp, int grid,
                             cudaStream_t stream);

}  // namespace numi
