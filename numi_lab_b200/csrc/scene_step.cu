// Per-world free-body control-step kernel and its host launchers; the
// device code lives in scene_step.cuh.
#include "scene_step.cuh"

#include <cstdlib>

namespace numi {
namespace {

// At most 128 registers: 16 resident warps per SM.  More warps (96
// registers) ran slower: their narrowphase scratch no longer fits the L1.
template <bool kComp, bool kConvex>
__global__ void __launch_bounds__(32, 16) scene_step_kernel(SceneParams p) {
    extern __shared__ float4 smem4[];
    const int item = blockIdx.x;
    if (item >= p.env_count) return;
    const int env = p.env_index != nullptr ? p.env_index[item] : item;
    scene_step_item<kComp, kConvex>(p, reinterpret_cast<float*>(smem4), item, env);
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
