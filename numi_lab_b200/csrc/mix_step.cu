// The heterogeneous batch kernel (mix.h): one persistent launch per control
// step over the environments of several worlds.  Each warp claims items
// from a device queue and runs the claimed world's own device code path
// (world_step.cuh for articulated worlds, scene_step.cuh for piles) on its
// own slice of shared memory, so articulated trees, chains and piles of any
// body count share the launch; warps of one CTA never synchronise with each
// other.
#include "mix.h"
#include "scene_step.cuh"
#include "world_step.cuh"

namespace numi {
namespace {

constexpr int kLayoutFloats = (static_cast<int>(sizeof(WarpLayout)) / 4 + 3) & ~3;

// Same register budget as the articulated kernel: 3 CTAs of 4 warps, i.e.
// at most 170 registers; the FP32 contact path sets it (about 141).
__global__ void __launch_bounds__(128, 3) mix_step_kernel(const MixWorld* __restrict__ worlds, const std::uint32_t* __restrict__ items,
                                                          int item_count, unsigned* next_item, int smem_floats_per_warp) {
    extern __shared__ float4 smem4[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    float* base = reinterpret_cast<float*>(smem4) + static_cast<size_t>(warp) * smem_floats_per_warp;
    for (;;) {
        unsigned claimed = 0u;
        if (lane == 0) claimed = atomicAdd(next_item, 1u);
        claimed = __shfl_sync(0xffffffffu, claimed, 0);
        if (claimed >= static_cast<unsigned>(item_count)) break;
        const std::uint32_t code = items[claimed];
        const MixWorld& W = worlds[code >> kMixWorldShift];
        const int env = static_cast<int>(code & kMixEnvMask);
        const int kind = W.kind;
        if (kind == kMixScene) {
            scene_step_item<false, false>(W.scene, base, env, env);
        } else {
            // The layout is read in every inner loop: keep a copy beside the
            // warp's sections instead of reading the descriptor in HBM.
            WarpLayout* L = reinterpret_cast<WarpLayout*>(base);
            if (lane < static_cast<int>(sizeof(WarpLayout) / 4))
                reinterpret_cast<int*>(L)[lane] = reinterpret_cast<const int*>(&W.layout)[lane];
            __syncwarp();
            if (kind == kMixContact)
                control_step_item<true, float, false>(W.step, *L, &W.step.model->tables, base + kLayoutFloats, env, env);
            else
                control_step_item<false, float, false>(W.step, *L, &W.step.model->tables, base + kLayoutFloats, env, env);
        }
        __syncwarp();
    }
}

}  // namespace

int mix_articulated_warp_floats(const WarpLayout& layout) { return kLayoutFloats + layout.total; }
int mix_scene_warp_floats() { return static_cast<int>(scene_step_smem_bytes(false) / sizeof(float)); }

cudaError_t configure_mix_kernel(size_t max_dynamic_smem) {
    return cudaFuncSetAttribute(mix_step_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(max_dynamic_smem));
}

cudaError_t mix_occupancy(int warps_per_block, size_t smem_per_block, int* blocks_per_sm) {
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, mix_step_kernel, 32 * warps_per_block, smem_per_block);
}

cudaError_t launch_mix_step(const MixWorld* worlds, const std::uint32_t* items, int item_count, unsigned* next_item,
                            int warps_per_block, int smem_floats_per_warp, int grid, cudaStream_t stream) {
    if (warps_per_block < 1 || warps_per_block > 4 || grid < 1 || smem_floats_per_warp < kLayoutFloats) return cudaErrorInvalidValue;
    const size_t smem = static_cast<size_t>(smem_floats_per_warp) * sizeof(float) * warps_per_block;
    mix_step_kernel<<<grid, 32 * warps_per_block, smem, stream>>>(worlds, items, item_count, next_item, smem_floats_per_warp);
    return cudaGetLastError();
}

}  // namespace numi
