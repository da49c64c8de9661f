// Pile / stack control steps for callers that cannot allocate device memory
// (mr_pile_step_no_alloc in numi_b200.h).
//
// Some hosts own all of the GPU's memory through their own allocator or a
// fixed budget and forbid a library from calling cudaMalloc (or from
// triggering the device-wide synchronisation it can cause in the middle of a
// latency-bound loop).  The rollout handle allocates its state and its
// per-environment workspace; this entry point instead runs the same
// free-body kernel on buffers the caller already owns, with the kernel's
// workspace, its launch counters and the packed world record in file-scope
// device arrays of fixed size.  Every GPU that loads the library holds those
// arrays (about 8 MB) until the process exits.
#include "numi_b200.h"
#include "runtime.h"
#include "device_model.h"
#include "scene.h"

#include <cstdint>
#include <cstring>
#include <mutex>
#include <stdexcept>
#include <string>

namespace {

using numi::rt::check;
using numi::rt::guarded;

// Workspace of MR_B200_NO_ALLOC_MAX_ENVS environments (each needs
// scene_workspace_words() floats; checked at set-up).
constexpr std::size_t kScratchBytes = std::size_t(8) << 20;
constexpr std::size_t kStatWords = 16;

static __device__ __align__(256) float g_scratch[kScratchBytes / sizeof(float)];
static __device__ __align__(256) std::uint32_t g_stats[kStatWords];
static __device__ __align__(256) numi::SceneModel g_model;

constexpr int kMaxDevices = 64;

// Device addresses of the arrays (host code may not use the array names as
// addresses) and the world record they currently hold, per device.
struct DeviceState {
    bool ready = false;
    float* scratch = nullptr;
    std::uint32_t* stats = nullptr;
    numi::SceneModel* model = nullptr;
    bool have_model = false;
    std::uint32_t source = 0;
    std::uint64_t seed = 0;
    float h = 0.0f;
    // Tag of the record in g_model: bumped by every upload, stored in the
    // record and passed with every launch, so a launch recorded for one
    // world (a captured graph, say) and run after another world's upload
    // reports a mismatch instead of stepping the wrong world.
    std::uint32_t generation = 0;
    numi::SceneModel host_model{};  // source of the last model upload
};

std::mutex g_mutex;
DeviceState g_devices[kMaxDevices];

// One-time set-up on the current device: resolve the arrays' device
// addresses (must run with that device current).
DeviceState& device_state() {
    int dev = 0;
    check(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) throw std::runtime_error("device index outside the supported range");
    DeviceState& d = g_devices[dev];
    if (!d.ready) {
        if (static_cast<std::size_t>(MR_B200_NO_ALLOC_MAX_ENVS) * numi::scene_workspace_words() * sizeof(float) > kScratchBytes)
            throw std::runtime_error("no-allocation scratch is smaller than the stated environment maximum");
        check(cudaGetSymbolAddress(reinterpret_cast<void**>(&d.scratch), g_scratch), "cudaGetSymbolAddress(scratch)");
        check(cudaGetSymbolAddress(reinterpret_cast<void**>(&d.stats), g_stats), "cudaGetSymbolAddress(stats)");
        check(cudaGetSymbolAddress(reinterpret_cast<void**>(&d.model), g_model), "cudaGetSymbolAddress(model)");
        check(numi::configure_scene_step_kernel(), "scene kernel attributes");
        d.ready = true;
    }
    return d;
}

}  // namespace

extern "C" {

MR_API int mr_pile_step_no_alloc(uint32_t source, uint64_t model_seed, uint32_t environment_count, float* q, float* v,
                                 float* manifolds, uint32_t* manifold_counts, const float* friction_scale,
                                 uint32_t* status_codes, uint32_t control_step_count, float control_timestep_seconds,
                                 uint32_t physics_substeps, uint32_t velocity_iterations, uint32_t final_velocity_iterations,
                                 uint64_t cuda_stream) {
    return guarded([&] {
        if (source != MR_RUN_SOURCE_SYNTHETIC_PILE && source != MR_RUN_SOURCE_SYNTHETIC_STACK)
            throw std::invalid_argument("mr_pile_step_no_alloc runs pile and stack worlds only (MR_RUN_SOURCE_SYNTHETIC_PILE, _STACK)");
        if (environment_count == 0 || environment_count > MR_B200_NO_ALLOC_MAX_ENVS)
            throw std::invalid_argument("environment_count " + std::to_string(environment_count) +
                                        " is outside [1, " + std::to_string(MR_B200_NO_ALLOC_MAX_ENVS) +
                                        "], the most environments the fixed no-allocation workspace holds");
        if (!q || !v || !manifolds || !manifold_counts || !friction_scale)
            throw std::invalid_argument("q, v, manifolds, manifold_counts and friction_scale must be non-null device pointers");
        if (physics_substeps == 0 || physics_substeps > MR_B200_MAX_SUBSTEPS)
            throw std::invalid_argument("physics_substeps must be in [1, 64]");
        if (!(control_timestep_seconds > 0.0f)) throw std::invalid_argument("control_timestep_seconds must be positive");
        if (velocity_iterations == 0 && final_velocity_iterations == 0)
            throw std::invalid_argument("contact worlds need at least one velocity iteration");
        cudaStream_t stream = reinterpret_cast<cudaStream_t>(cuda_stream);

        std::lock_guard<std::mutex> lock(g_mutex);
        DeviceState& d = device_state();
        const float h = control_timestep_seconds / static_cast<float>(physics_substeps);
        if (!d.have_model || d.source != source || d.seed != model_seed || d.h != h) {
            const numi::CompiledModel m = source == MR_RUN_SOURCE_SYNTHETIC_PILE ? numi::build_pile(model_seed)
                                                                                 : numi::build_stack(model_seed);
            d.host_model = numi::rt::pack_scene(m, h);
            d.generation = d.generation == 0xffffffffu ? 1u : d.generation + 1u;
            d.host_model.world_tag = d.generation;
            check(cudaMemcpyAsync(d.model, &d.host_model, sizeof(numi::SceneModel), cudaMemcpyHostToDevice, stream),
                  "world record upload");
            d.have_model = true;
            d.source = source;
            d.seed = model_seed;
            d.h = h;
        }
        check(cudaMemsetAsync(d.stats, 0, kStatWords * sizeof(std::uint32_t), stream), "clear counters");
        check(cudaMemsetAsync(d.stats + numi::kStatFirstFailEnv, 0xff, sizeof(std::uint32_t), stream), "clear counters");
        for (std::uint32_t k = 0; k < control_step_count; ++k) {
            numi::SceneParams p{};
            p.model = d.model;
            p.q = q;
            p.v = v;
            p.manifolds = manifolds;
            p.manifold_count = manifold_counts;
            p.friction_scale = friction_scale;
            p.status_codes = status_codes ? status_codes + static_cast<std::size_t>(k) * environment_count : nullptr;
            p.stats = d.stats;
            p.workspace = d.scratch;
            p.env_count = static_cast<int>(environment_count);
            p.substeps = static_cast<int>(physics_substeps);
            p.velocity_iterations = static_cast<int>(velocity_iterations);
            p.final_velocity_iterations = static_cast<int>(final_velocity_iterations);
            p.support_mapped = d.host_model.support_mapped;
            p.world_tag = d.generation;
            check(numi::launch_scene_step(p, stream), "scene step launch");
        }
    });
}

MR_API int mr_pile_step_no_alloc_counters(uint32_t* counters, uint32_t count, uint64_t cuda_stream) {
    return guarded([&] {
        if (!counters) throw std::invalid_argument("counters must be a non-null host pointer");
        if (count == 0 || count > kStatWords)
            throw std::invalid_argument("count must be in [1, " + std::to_string(kStatWords) + "]");
        cudaStream_t stream = reinterpret_cast<cudaStream_t>(cuda_stream);
        std::lock_guard<std::mutex> lock(g_mutex);
        DeviceState& d = device_state();
        // Pageable host memory: the copy completes before the call returns.
        check(cudaMemcpyAsync(counters, d.stats, count * sizeof(std::uint32_t), cudaMemcpyDeviceToHost, stream),
              "counter read-back");
        check(cudaStreamSynchronize(stream), "counter read-back");
    });
}

}  // extern "C"
