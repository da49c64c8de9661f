// Per-world articulated control-step kernel and its host launchers; the
// device code lives in world_step.cuh.
#include "world_step.cuh"

#include <type_traits>

namespace numi {
namespace {

// The FP32 temporalCone instance may run up to kMaxStepWarpsPerBlock
// environments per CTA (one copy of the topology tables for all of them);
// the FP64 and quality instances keep CTAs of at most 4 warps and their
// larger register budgets.
template <typename R, bool kQuality>
constexpr bool kWideStepBlock = std::is_same<R, float>::value && !kQuality;

template <bool kContact, typename R, bool kComp, bool kQuality>
__global__ void __launch_bounds__(kWideStepBlock<R, kQuality> ? 32 * kMaxStepWarpsPerBlock : 128, kWideStepBlock<R, kQuality> ? 1 : 3)
    control_step_kernel(StepParams p, WarpLayout layout, int warps_per_block) {
    extern __shared__ float4 smem4[];
    // Topology tables: one copy per CTA.
    {
        const uint4* src = reinterpret_cast<const uint4*>(&p.model->tables);
        uint4* dst = reinterpret_cast<uint4*>(smem4);
        for (int i = threadIdx.x; i < static_cast<int>(sizeof(DeviceTables) / 16); i += blockDim.x) dst[i] = src[i];
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5;
    // Work item (compact index of this launch's outputs) and the resident
    // environment slot it advances.
    const int item = blockIdx.x * warps_per_block + warp;
    if (item >= p.env_count) return;
    const int env = p.env_index != nullptr ? p.env_index[item] : item;
    control_step_item<kContact, R, kComp, kQuality>(p, layout, reinterpret_cast<const DeviceTables*>(smem4),
                                          reinterpret_cast<float*>(smem4) + sizeof(DeviceTables) / sizeof(float) + warp * layout.total,
                                          item, env);
}

// The FP64 audit of the state each environment committed in the launch
// with the same parameters (one warp per environment, like that launch).
template <typename R>
__global__ void __launch_bounds__(32 * kMaxStepWarpsPerBlock) audit_step_kernel(StepParams p, WarpLayout layout, int warps_per_block) {
    extern __shared__ float4 smem4[];
    {
        const uint4* src = reinterpret_cast<const uint4*>(&p.model->tables);
        uint4* dst = reinterpret_cast<uint4*>(smem4);
        for (int i = threadIdx.x; i < static_cast<int>(sizeof(DeviceTables) / 16); i += blockDim.x) dst[i] = src[i];
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5;
    const int item = blockIdx.x * warps_per_block + warp;
    if (item >= p.env_count || p.audit == nullptr) return;
    const int env = p.env_index != nullptr ? p.env_index[item] : item;
    const int lane = threadIdx.x & 31;
    const DeviceModel& M = *p.model;
    Warp w;
    w.lane = lane;
    w.T = reinterpret_cast<const DeviceTables*>(smem4);
    w.s = reinterpret_cast<float*>(smem4) + sizeof(DeviceTables) / sizeof(float) + warp * layout.total;
    w.L = &layout;
    w.M = p.model;
    const float* q = p.q + static_cast<size_t>(env) * M.nq;
    const float* v = p.v + static_cast<size_t>(env) * M.nv;
    for (int i = lane; i < M.nq; i += 32) w.s[layout.q + i] = q[i];
    for (int i = lane; i < M.nv; i += 32) w.s[layout.v + i] = v[i];
    if (lane == 0) w.s[layout.misc] = 0.0f;
    BodyConst bc;
    if (lane < M.nb) load_body(M, lane, bc);
    __syncwarp();
    const bool reset = p.reset_masks != nullptr && p.reset_masks[item] != 0u;
    audit_articulated<R>(w, bc, p.audit + static_cast<size_t>(env) * kAuditWords, reset);
}

}  // namespace

cudaError_t launch_audit_step(const StepParams& p, const WarpLayout& layout, bool fp64_inertia, int warps_per_block,
                              cudaStream_t stream) {
    const int blocks = (p.env_count + warps_per_block - 1) / warps_per_block;
    const size_t smem = sizeof(DeviceTables) + static_cast<size_t>(layout.total) * sizeof(float) * warps_per_block;
    if (fp64_inertia)
        audit_step_kernel<double><<<blocks, 32 * warps_per_block, smem, stream>>>(p, layout, warps_per_block);
    else
        audit_step_kernel<float><<<blocks, 32 * warps_per_block, smem, stream>>>(p, layout, warps_per_block);
    return cudaGetLastError();
}

size_t control_step_table_bytes() { return sizeof(DeviceTables); }

int control_step_max_warps_per_block(std::uint32_t precision, bool quality) {
    return precision == MR_PRECISION_FP32 && !quality ? kMaxStepWarpsPerBlock : 4;
}

namespace {

// The kernel instance of (contact, precision, quality solver); the quality
// solver runs in contact worlds only.
template <typename F>
cudaError_t for_kernel(bool contact, std::uint32_t precision, bool quality, F&& f) {
    if (contact && quality) {
        if (precision == MR_PRECISION_COMPENSATED) return f(control_step_kernel<true, double, true, true>);
        if (precision == MR_PRECISION_FP64_ARTICULATED_INERTIA) return f(control_step_kernel<true, double, false, true>);
        return f(control_step_kernel<true, float, false, true>);
    }
    if (contact) {
        if (precision == MR_PRECISION_COMPENSATED) return f(control_step_kernel<true, double, true, false>);
        if (precision == MR_PRECISION_FP64_ARTICULATED_INERTIA) return f(control_step_kernel<true, double, false, false>);
        return f(control_step_kernel<true, float, false, false>);
    }
    if (precision == MR_PRECISION_COMPENSATED) return f(control_step_kernel<false, double, true, false>);
    if (precision == MR_PRECISION_FP64_ARTICULATED_INERTIA) return f(control_step_kernel<false, double, false, false>);
    return f(control_step_kernel<false, float, false, false>);
}

}  // namespace

// Host launcher: one control step of `env_count` environments.
// `precision` (MRPrecisionModeC) selects the kernel instance: FP32, FP64
// articulated inertia, or FP64 articulated inertia with compensated sums;
// `quality` the converged contact solve in place of the temporalCone sweeps
// (the layout must carry its workspace).
cudaError_t launch_control_step(const StepParams& p, const WarpLayout& layout, bool contact, std::uint32_t precision, bool quality,
                                int warps_per_block, cudaStream_t stream) {
    const int blocks = (p.env_count + warps_per_block - 1) / warps_per_block;
    const size_t smem = sizeof(DeviceTables) + static_cast<size_t>(layout.total) * sizeof(float) * warps_per_block;
    const int threads = 32 * warps_per_block;
    if (precision == MR_PRECISION_COMPENSATED && p.q_comp == nullptr) return cudaErrorInvalidValue;
    if (quality && (!contact || layout.quality >= layout.total)) return cudaErrorInvalidValue;
    return for_kernel(contact, precision, quality, [&](auto kernel) {
        kernel<<<blocks, threads, smem, stream>>>(p, layout, warps_per_block);
        return cudaGetLastError();
    });
}

cudaError_t control_step_occupancy(bool contact, std::uint32_t precision, bool quality, int warps_per_block, size_t smem,
                                   int* blocks_per_sm) {
    const int threads = 32 * warps_per_block;
    return for_kernel(contact, precision, quality, [&](auto kernel) {
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, kernel, threads, smem);
    });
}

cudaError_t configure_control_step_kernels(size_t max_dynamic_smem) {
    const int bytes = static_cast<int>(max_dynamic_smem);
    cudaError_t e = cudaSuccess;
    for (const bool contact : {true, false})
        for (const bool quality : {false, true})
            for (const std::uint32_t precision :
                 {std::uint32_t(MR_PRECISION_FP32), std::uint32_t(MR_PRECISION_FP64_ARTICULATED_INERTIA), std::uint32_t(MR_PRECISION_COMPENSATED)})
                if (e == cudaSuccess && (contact || !quality))
                    e = for_kernel(contact, precision, quality, [&](auto kernel) {
                        return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
                    });
    if (e == cudaSuccess) e = cudaFuncSetAttribute(audit_step_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(audit_step_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    return e;
}

}  // namespace numi
