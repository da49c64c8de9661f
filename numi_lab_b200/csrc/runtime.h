// Host-runtime pieces shared by the task-rollout handle (rollout.cu) and the
// continuous-batching server (serve.cu): CUDA error checks, owning device /
// pinned buffers, the C-ABI error convention, and the launch plan of the
// control-step kernel for a compiled model.
#pragma once

#include "device_model.h"
#include "layout.h"
#include "model.h"
#include "scene.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <stdexcept>
#include <string>

namespace numi {

// `precision` is an MRPrecisionModeC value; MR_PRECISION_COMPENSATED needs
// p.q_comp and the layout made with its compensation section.
// `quality` selects the instances with the converged contact solve
// (quality.cuh) in place of the temporalCone sweeps; their layout carries
// the solver's workspace.
cudaError_t control_step_occupancy(bool contact, std::uint32_t precision, bool quality, int warps_per_block, size_t smem,
                                   int* blocks_per_sm);
cudaError_t launch_control_step(const StepParams& p, const WarpLayout& layout, bool contact, std::uint32_t precision, bool quality,
                                int warps_per_block, cudaStream_t stream);
cudaError_t configure_control_step_kernels(size_t max_dynamic_smem);
// FP64 energy / momentum audit (audit.cuh) of the state the control-step
// launch with the same parameters committed; p.audit must be set.
cudaError_t launch_audit_step(const StepParams& p, const WarpLayout& layout, bool fp64_inertia, int warps_per_block,
                              cudaStream_t stream);
size_t control_step_table_bytes();
// Largest CTA (in warps) the control-step instance for (precision, quality) is built for.
int control_step_max_warps_per_block(std::uint32_t precision, bool quality);

namespace rt {

inline void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

template <typename T>
struct DeviceBuffer {
    T* ptr = nullptr;
    size_t count = 0;
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    ~DeviceBuffer() { if (ptr) cudaFree(ptr); }
    void reset() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        count = 0;
    }
    void resize(size_t n) {
        if (n <= count && ptr) return;
        if (ptr) { cudaFree(ptr); ptr = nullptr; }
        check(cudaMalloc(&ptr, std::max<size_t>(n, 1) * sizeof(T)), "cudaMalloc");
        count = n;
    }
};

template <typename T>
struct PinnedBuffer {
    T* ptr = nullptr;
    size_t count = 0;
    PinnedBuffer() = default;
    PinnedBuffer(const PinnedBuffer&) = delete;
    PinnedBuffer& operator=(const PinnedBuffer&) = delete;
    ~PinnedBuffer() { if (ptr) cudaFreeHost(ptr); }
    void resize(size_t n) {
        if (n <= count && ptr) return;
        if (ptr) { cudaFreeHost(ptr); ptr = nullptr; }
        check(cudaMallocHost(&ptr, std::max<size_t>(n, 1) * sizeof(T)), "cudaMallocHost");
        count = n;
    }
};

// The C ABI's error convention: thread-local message, 0 / -1 returns.
void set_last_error(const std::string& message);
const char* last_error();

template <typename F>
int guarded(F&& f) {
    try {
        f();
        return 0;
    } catch (const std::exception& e) {
        set_last_error(e.what());
    } catch (...) {
        set_last_error("unknown native error");
    }
    return -1;
}

// Everything the control-step kernel needs to know about a compiled model
// at one substep length: the packed device record, the per-warp
// shared-memory layout and the launch shape per (solver, precision mode).
constexpr int kPrecisionModes = 3;       // indexed by MRPrecisionModeC
constexpr int kSolverModes = 2;          // 0 temporalCone, 1 quality (contact worlds)
struct KernelPlan {
    DeviceModel dmodel{};
    // [solver]: FP32 and FP64 articulated inertia; compensated adds the q
    // compensation section.  The quality layouts add the solver workspace.
    WarpLayout layout[kSolverModes]{};
    WarpLayout layout_comp[kSolverModes]{};
    bool contact = false;
    int warps_per_block[kSolverModes][kPrecisionModes] = {{1, 1, 1}, {1, 1, 1}};
    int resident_warps_per_sm[kSolverModes][kPrecisionModes] = {{0, 0, 0}, {0, 0, 0}};
    const WarpLayout& layout_for(std::uint32_t precision, bool quality = false) const {
        return precision == MR_PRECISION_COMPENSATED ? layout_comp[quality] : layout[quality];
    }
};

DeviceModel pack_model(const CompiledModel& m, float h);
// Builds the plan for the current device; throws when the model does not fit.
void make_plan(const CompiledModel& m, float h, KernelPlan& plan);
// Packs a pile (scene) world for the free-body kernel at substep length h.
SceneModel pack_scene(const CompiledModel& m, float h);
// MRQualitySolverConfigC (null: all defaults) with its defaults applied;
// throws on out-of-range settings.
QualityConfig quality_config(const MRQualitySolverConfigC* c);

}  // namespace rt
}  // namespace numi
