// The heterogeneous batch kernel (mix.h): one persistent launch per horizon
// of control steps over the environments of several worlds.  Each warp claims items
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
// at most 170 registers.
//
// A claimed item is one environment for the whole horizon: environments are
// independent, so the warp runs its `steps` control steps back to back
// (step k reads the world's step-k descriptor) and no environment waits
// for any other between control steps -- one launch per horizon.
__global__ void __launch_bounds__(128, 3) mix_step_kernel(const MixWorld* __restrict__ worlds, int world_count, int steps,
                                                          const std::uint32_t* __restrict__ items, int item_count,
                                                          unsigned* next_item, int smem_floats_per_warp) {
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
        const int world = static_cast<int>(code >> kMixWorldShift);
        const int env = static_cast<int>(code & kMixEnvMask);
        const int kind = worlds[world].kind;
        if (kind != kMixScene) {
            // The layout is read in every inner loop: keep a copy beside the
            // warp's sections instead of reading the descriptor in HBM.
            WarpLayout* L = reinterpret_cast<WarpLayout*>(base);
            if (lane < static_cast<int>(sizeof(WarpLayout) / 4))
                reinterpret_cast<int*>(L)[lane] = reinterpret_cast<const int*>(&worlds[world].layout)[lane];
            __syncwarp();
        }
        for (int k = 0; k < steps; ++k) {
            const MixWorld& W = worlds[static_cast<size_t>(k) * world_count + world];
            if (kind == kMixScene)
                scene_step_item<false, false>(W.scene, base, env, env);
            else if (kind == kMixContact)
                control_step_item<true, float, false>(W.step, *reinterpret_cast<const WarpLayout*>(base), &W.step.model->tables,
                                                      base + kLayoutFloats, env, env);
            else
                control_step_item<false, float, false>(W.step, *reinterpret_cast<const WarpLayout*>(base), &W.step.model->tables,
                                                       base + kLayoutFloats, env, env);
            __syncwarp();
        }
    }
}

// Per-family variants: the same env-major claim loop over one family's
// items only, each compiled to its own register budget -- the articulated
// one like the articulated kernel (3 CTAs of 4 warps) here, the free-body
// one like the scene kernel (16 resident warps, at most 128 registers) in
// scene_step.cu, beside the per-world scene kernel -- so a batch can run
// each family at its own kernel's occupancy.
__global__ void __launch_bounds__(128, 3) mix_articulated_kernel(const MixWorld* __restrict__ worlds, int world_count, int steps,
                                                                 const std::uint32_t* __restrict__ items, int item_count,
                                                                 unsigned* next_item, int smem_floats_per_warp) {
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
        const int world = static_cast<int>(code >> kMixWorldShift);
        const int env = static_cast<int>(code & kMixEnvMask);
        WarpLayout* L = reinterpret_cast<WarpLayout*>(base);
        if (lane < static_cast<int>(sizeof(WarpLayout) / 4))
            reinterpret_cast<int*>(L)[lane] = reinterpret_cast<const int*>(&worlds[world].layout)[lane];
        __syncwarp();
        const bool contact = worlds[world].kind == kMixContact;
        for (int k = 0; k < steps; ++k) {
            const MixWorld& W = worlds[static_cast<size_t>(k) * world_count + world];
            if (contact)
                control_step_item<true, float, false>(W.step, *L, &W.step.model->tables, base + kLayoutFloats, env, env);
            else
                control_step_item<false, float, false>(W.step, *L, &W.step.model->tables, base + kLayoutFloats, env, env);
            __syncwarp();
        }
    }
}

template <typename F>
cudaError_t for_mix_kernel(int family, F&& f) {
    if (family == kMixFamilyArticulated) return f(mix_articulated_kernel);
    return f(mix_step_kernel);
}

bool scene_family(int family) { return family == kMixFamilyScene || family == kMixFamilySceneConvex; }

}  // namespace

int mix_articulated_warp_floats(const WarpLayout& layout) { return kLayoutFloats + layout.total; }
int mix_scene_warp_floats() { return static_cast<int>(scene_step_smem_bytes(false) / sizeof(float)); }

cudaError_t configure_mix_kernel(int family, size_t max_dynamic_smem) {
    if (scene_family(family)) return configure_mix_scene_kernel(family == kMixFamilySceneConvex, max_dynamic_smem);
    return for_mix_kernel(family, [&](auto kernel) {
        return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(max_dynamic_smem));
    });
}

cudaError_t mix_occupancy(int family, int warps_per_block, size_t smem_per_block, int* blocks_per_sm) {
    if (scene_family(family)) return mix_scene_occupancy(family == kMixFamilySceneConvex, warps_per_block, smem_per_block, blocks_per_sm);
    return for_mix_kernel(family, [&](auto kernel) {
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, kernel, 32 * warps_per_block, smem_per_block);
    });
}

cudaError_t launch_mix_horizon(int family, const MixWorld* worlds, int world_count, int steps, const std::uint32_t* items,
                               int item_count, unsigned* next_item, int warps_per_block, int smem_floats_per_warp, int grid,
                               cudaStream_t stream) {
    const int max_warps = family == kMixFamilyScene || family == kMixFamilySceneConvex ? 1 : 4;
    if (warps_per_block < 1 || warps_per_block > max_warps || grid < 1 || steps < 1 || world_count < 1 ||
        smem_floats_per_warp < kLayoutFloats || (smem_floats_per_warp & 3) != 0)
        return cudaErrorInvalidValue;
    if (scene_family(family))
        return launch_mix_scene(family == kMixFamilySceneConvex, worlds, world_count, steps, items, item_count, next_item,
                                warps_per_block, smem_floats_per_warp, grid, stream);
    const size_t smem = static_cast<size_t>(smem_floats_per_warp) * sizeof(float) * warps_per_block;
    return for_mix_kernel(family, [&](auto kernel) {
        kernel<<<grid, 32 * warps_per_block, smem, stream>>>(worlds, world_count, steps, items, item_count, next_item,
                                                              smem_floats_per_warp);
        return cudaGetLastError();
    });
}

}  // namespace numi
