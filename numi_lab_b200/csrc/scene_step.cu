// Per-world free-body control-step kernel, the heterogeneous batch's
// free-body family kernels, and their host launchers; the device code lives
// in scene_step.cuh.
#include "mix.h"
#include "scene_step.cuh"

#include <cstdlib>

namespace numi {
namespace {

// The FP32 control step of a world with support-mapped pairs, compiled once
// out of line: the per-world kernel and the batch's free-body family both
// call this body, so the two produce the same bits (inlined into two
// kernels, the compiler's floating-point contractions may differ).
__device__ __noinline__ void scene_step_convex(const SceneParams& p, float* smem, int item, int env) {
    scene_step_item<false, true>(p, smem, item, env);
}

// At most 128 registers: 16 resident warps per SM.  More warps (96
// registers) ran slower: their narrowphase scratch no longer fits the L1.
template <bool kComp, bool kConvex>
__global__ void __launch_bounds__(32, 16) scene_step_kernel(SceneParams p) {
    extern __shared__ float4 smem4[];
    const int item = blockIdx.x;
    if (item >= p.env_count) return;
    const int env = p.env_index != nullptr ? p.env_index[item] : item;
    if constexpr (!kComp && kConvex)
        scene_step_convex(p, reinterpret_cast<float*>(smem4), item, env);
    else
        scene_step_item<kComp, kConvex>(p, reinterpret_cast<float*>(smem4), item, env);
}

// The batch's free-body family (mix_step.cu): the per-family claim loop over
// free-body items.  It sits in this translation unit so that it and the
// per-world kernel run one compiled copy of the out-of-line narrowphase
// (support_mapped_contacts): a batch reproduces each world alone bit for
// bit.  A world without support-mapped pairs runs the instance its own
// kernel runs.
template <bool kConvex>
__global__ void __launch_bounds__(32, 16) mix_scene_kernel(const MixWorld* __restrict__ worlds, int world_count, int steps,
                                                           const std::uint32_t* __restrict__ items, int item_count,
                                                           unsigned* next_item, int smem_floats_per_warp) {
    extern __shared__ float4 smem4[];
    const int lane = threadIdx.x & 31;
    float* base = reinterpret_cast<float*>(smem4) + static_cast<size_t>(threadIdx.x >> 5) * smem_floats_per_warp;
    for (;;) {
        unsigned claimed = 0u;
        if (lane == 0) claimed = atomicAdd(next_item, 1u);
        claimed = __shfl_sync(0xffffffffu, claimed, 0);
        if (claimed >= static_cast<unsigned>(item_count)) break;
        const std::uint32_t code = items[claimed];
        const int world = static_cast<int>(code >> kMixWorldShift);
        const int env = static_cast<int>(code & kMixEnvMask);
        for (int k = 0; k < steps; ++k) {
            const SceneParams& sp = worlds[static_cast<size_t>(k) * world_count + world].scene;
            if constexpr (kConvex) {
                if (sp.support_mapped)
                    scene_step_convex(sp, base, env, env);
                else
                    scene_step_item<false, false>(sp, base, env, env);
            } else {
                scene_step_item<false, false>(sp, base, env, env);
            }
            __syncwarp();
        }
    }
}

// The FP64 audit of the bodies each environment committed in the launch with
// the same parameters.
__global__ void __launch_bounds__(32) scene_audit_kernel(SceneParams p) {
    const int item = blockIdx.x;
    if (item >= p.env_count || p.audit == nullptr) return;
    const int env = p.env_index != nullptr ? p.env_index[item] : item;
    const SceneModel& M = *p.model;
    const bool reset = p.reset_masks != nullptr && p.reset_masks[item] != 0u;
    audit_scene(M, p.q + static_cast<size_t>(env) * M.nb * 7, p.v + static_cast<size_t>(env) * M.nb * 6,
                p.audit + static_cast<size_t>(env) * kAuditWords, reset, static_cast<int>(threadIdx.x));
}

}  // namespace

size_t scene_step_smem_bytes(bool compensated) {
    return static_cast<size_t>(compensated ? kSceneSmemWordsComp : kSceneSmemWords) * sizeof(float);
}

namespace {

// Resident environments per SM of the per-world launch (0: as many as the
// registers allow).  NUMI_B200_SCENE_RESIDENT, read once, overrides it; a
// lower count is reached by asking each one-warp CTA for more shared memory.
int scene_resident_limit() {
    static const int limit = [] {
        const char* env = std::getenv("NUMI_B200_SCENE_RESIDENT");
        const int v = env ? std::atoi(env) : 0;
        return v > 0 && v <= 32 ? v : 0;
    }();
    return limit;
}

size_t scene_launch_smem(bool compensated) {
    size_t smem = scene_step_smem_bytes(compensated);
    if (const int limit = scene_resident_limit()) {
        int dev = 0, per_sm = 0;
        if (cudaGetDevice(&dev) == cudaSuccess &&
            cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) == cudaSuccess && per_sm > 0) {
            const size_t padded = static_cast<size_t>(per_sm / limit) - 1024;  // 1 KB reserved per CTA
            if (padded > smem) smem = padded;
        }
    }
    return smem;
}

}  // namespace
size_t scene_workspace_words() { return static_cast<size_t>(kWsWords); }

namespace {

template <typename F>
cudaError_t for_scene_kernel(bool compensated, bool convex, F&& f) {
    if (compensated) return convex ? f(scene_step_kernel<true, true>) : f(scene_step_kernel<true, false>);
    return convex ? f(scene_step_kernel<false, true>) : f(scene_step_kernel<false, false>);
}

}  // namespace

cudaError_t configure_scene_step_kernel() {
    // The driver's default carveout keeps most of the unified L1 as cache,
    // which the narrowphase scratch and contact records rely on.
    cudaError_t e = cudaSuccess;
    for (const bool compensated : {false, true})
        for (const bool convex : {false, true})
            if (e == cudaSuccess)
                e = for_scene_kernel(compensated, convex, [&](auto kernel) {
                    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                static_cast<int>(scene_launch_smem(compensated)));
                });
    return e;
}

cudaError_t configure_mix_scene_kernel(bool convex, size_t max_dynamic_smem) {
    const int bytes = static_cast<int>(max_dynamic_smem);
    return convex ? cudaFuncSetAttribute(mix_scene_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes)
                  : cudaFuncSetAttribute(mix_scene_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

cudaError_t mix_scene_occupancy(bool convex, int warps_per_block, size_t smem_per_block, int* blocks_per_sm) {
    return convex ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, mix_scene_kernel<true>, 32 * warps_per_block,
                                                                  smem_per_block)
                  : cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, mix_scene_kernel<false>, 32 * warps_per_block,
                                                                  smem_per_block);
}

cudaError_t launch_mix_scene(bool convex, const MixWorld* worlds, int world_count, int steps, const std::uint32_t* items,
                             int item_count, unsigned* next_item, int warps_per_block, int smem_floats_per_warp, int grid,
                             cudaStream_t stream) {
    const size_t smem = static_cast<size_t>(smem_floats_per_warp) * sizeof(float) * warps_per_block;
    if (convex)
        mix_scene_kernel<true><<<grid, 32 * warps_per_block, smem, stream>>>(worlds, world_count, steps, items, item_count, next_item,
                                                                             smem_floats_per_warp);
    else
        mix_scene_kernel<false><<<grid, 32 * warps_per_block, smem, stream>>>(worlds, world_count, steps, items, item_count, next_item,
                                                                              smem_floats_per_warp);
    return cudaGetLastError();
}

cudaError_t launch_scene_audit(const SceneParams& p, cudaStream_t stream) {
    scene_audit_kernel<<<p.env_count, 32, 0, stream>>>(p);
    return cudaGetLastError();
}

cudaError_t launch_scene_step(const SceneParams& p, cudaStream_t stream) {
    const bool compensated = p.q_comp != nullptr;
    const size_t smem = scene_launch_smem(compensated);
    return for_scene_kernel(compensated, p.support_mapped != 0, [&](auto kernel) {
        kernel<<<p.env_count, 32, smem, stream>>>(p);
        return cudaGetLastError();
    });
}

}  // namespace numi
