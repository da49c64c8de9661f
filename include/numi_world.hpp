// C++ world API of the B200 microstep: the shape of the reference's lower
// C++ boundary, `metalrobo::MetalWorldContext` (include/metalrobo/MetalWorld.hpp),
// over this library's C ABI (numi_b200.h).  Header-only, C++17.
//
//   reference                                   here
//   MetalWorldBatch        MetalWorld.hpp:245-276   numi::WorldBatch
//   MetalWorldStepConfig   MetalWorld.hpp:380-452   numi::WorldStepConfig
//   MetalWorldResult       MetalWorld.hpp:620-656   numi::WorldResult
//   MetalWorldDiagnostics  MetalWorld.hpp:658-675   numi::WorldDiagnostics
//   MetalWorldContext::initializeResidentState / submitResident / run
//                          MetalWorld.hpp:779-805   numi::WorldContext (same names)
//
// A CompiledWorld of the reference is a compiled robot/scene; here it names
// one of the library's seeded synthetic worlds.  The resident state stays on
// the device between submissions, as in the reference; a submission is
// synchronous (the reference's submit + wait pair collapses into one call).
#pragma once

#include "numi_b200.h"

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace numi {

// A seeded synthetic world (MR_RUN_SOURCE_SYNTHETIC_*).
struct CompiledWorld {
    std::uint32_t source = MR_RUN_SOURCE_SYNTHETIC_TREE29;
    std::uint64_t seed = 0;
};

// One submission: `control_step_count` control steps of `environment_count`
// environments.  Spans are (pointer, count) pairs, packed like the
// reference's: efforts / actions [control step][environment][action],
// reset masks [control step][environment].  initial_q / initial_v
// ([environment][nq] / [nv]) replace the sampled reset state when given.
struct WorldBatch {
    std::size_t environment_count = 0;
    std::size_t control_step_count = 0;
    const float* initial_q = nullptr;
    const float* initial_v = nullptr;
    const float* actions = nullptr;
    std::size_t action_count = 0;
    const std::uint32_t* reset_masks = nullptr;
    std::size_t reset_mask_count = 0;
};

enum class PrecisionMode : std::uint32_t {
    fp32 = MR_PRECISION_FP32,
    fp64_articulated_inertia = MR_PRECISION_FP64_ARTICULATED_INERTIA,
    compensated = MR_PRECISION_COMPENSATED
};

struct WorldStepConfig {
    float timestep_seconds = 0.02f;  // control period
    std::uint32_t physics_substeps = 4;
    std::uint32_t velocity_iterations = 8;
    std::uint32_t final_velocity_iterations = 0;
    PrecisionMode precision = PrecisionMode::fp32;
    bool publish_final_state = true;  // final q and per-step observations
};

struct WorldDiagnostics {
    bool succeeded = true;                 // every environment-step succeeded
    std::uint32_t successful_step_count = 0;
    std::uint32_t failed_step_count = 0;
    std::uint32_t first_failing_environment = MR_INVALID_INDEX;
    std::uint32_t first_failing_control_step = MR_INVALID_INDEX;
    std::uint32_t first_status = MR_STEP_SUCCESS;
    std::uint32_t maximum_active_contacts = 0;
    double gpu_milliseconds = 0.0;
};

struct WorldResult {
    std::uint32_t nq = 0, nv = 0;
    std::vector<float> final_q;       // [environment][nq]
    std::vector<float> observations;  // [control step][environment][q then v]
    std::vector<std::uint32_t> statuses;         // [control step][environment]
    std::vector<std::uint32_t> active_contacts;  // [control step][environment]
    std::vector<float> final_scene_bodies;       // [environment][body][13] (piles, stacks)
};

// Device-resident state of one world batch between submissions.
class WorldResidentState {
public:
    WorldResidentState() = default;
    WorldResidentState(const WorldResidentState&) = delete;
    WorldResidentState& operator=(const WorldResidentState&) = delete;
    WorldResidentState(WorldResidentState&& o) noexcept : handle_(std::exchange(o.handle_, nullptr)), layout_(o.layout_) {}
    WorldResidentState& operator=(WorldResidentState&& o) noexcept {
        if (this != &o) {
            reset();
            handle_ = std::exchange(o.handle_, nullptr);
            layout_ = o.layout_;
        }
        return *this;
    }
    ~WorldResidentState() { reset(); }

    bool initialized() const { return handle_ != nullptr; }
    const MRTaskRolloutLayoutC& layout() const { return layout_; }
    MRTaskRolloutHandle* handle() const { return handle_; }
    void reset() {
        if (handle_) mr_task_rollout_destroy(handle_);
        handle_ = nullptr;
    }

private:
    friend class WorldContext;
    MRTaskRolloutHandle* handle_ = nullptr;
    MRTaskRolloutLayoutC layout_{};
};

class WorldContext {
public:
    // Creates the resident state for `batch.environment_count` environments
    // and runs the batch's control steps from it.
    WorldDiagnostics initializeResidentState(const CompiledWorld& world, const WorldBatch& batch, const WorldStepConfig& config,
                                             WorldResidentState& state, WorldResult* result = nullptr) {
        state.reset();
        MRRunManifestC manifest{};
        manifest.source = world.source;
        manifest.profile.environment_count = static_cast<std::uint32_t>(batch.environment_count);
        manifest.profile.physics_substeps = config.physics_substeps;
        manifest.profile.velocity_iterations = config.velocity_iterations;
        manifest.profile.final_velocity_iterations = config.final_velocity_iterations;
        manifest.profile.control_timestep_seconds = config.timestep_seconds;
        manifest.profile.seed = world.seed;
        state.handle_ = mr_create_task_rollout(&manifest);
        if (!state.handle_) throw std::runtime_error(std::string("mr_create_task_rollout: ") + mr_last_error());
        state.layout_ = mr_task_rollout_layout(state.handle_);
        check(mr_task_rollout_set_precision(state.handle_, static_cast<MRPrecisionModeC>(config.precision)), "set_precision");
        if (batch.initial_q || batch.initial_v) {
            if (!batch.initial_q || !batch.initial_v) throw std::invalid_argument("initial_q and initial_v go together");
            check(mr_task_rollout_set_state(state.handle_, batch.initial_q, batch.initial_v, nullptr, 1u), "set_state");
        }
        if (batch.control_step_count == 0) return WorldDiagnostics{};
        return submitResident(world, batch, config, state, result);
    }

    // Continues an initialized resident state by the batch's control steps
    // (initial state spans must be empty).
    WorldDiagnostics submitResident(const CompiledWorld&, const WorldBatch& batch, const WorldStepConfig& config,
                                    WorldResidentState& state, WorldResult* result = nullptr) {
        if (!state.initialized()) throw std::invalid_argument("resident state is not initialized");
        if (batch.environment_count != state.layout_.environment_count)
            throw std::invalid_argument("environment_count differs from the resident state's");
        check(mr_task_rollout_set_state_readback(state.handle_, config.publish_final_state ? 1u : 0u), "set_state_readback");
        MRTaskRolloutAdvanceC out{};
        const int rc = mr_task_rollout_advance(state.handle_, batch.actions, batch.action_count, batch.reset_masks, batch.reset_mask_count,
                                               static_cast<std::uint32_t>(batch.control_step_count), 0, 0, &out);
        // A failed environment-step is reported in the counters and as -1
        // (c_api.cpp:3983-3988); anything else is an error of the call.
        if (rc != 0 && out.failed_environment_steps == 0) throw std::runtime_error(std::string("advance: ") + mr_last_error());
        WorldDiagnostics d;
        d.succeeded = out.failed_environment_steps == 0;
        d.successful_step_count = out.successful_environment_steps;
        d.failed_step_count = out.failed_environment_steps;
        d.first_failing_environment = out.first_failing_environment;
        d.first_failing_control_step = out.first_failing_control_step;
        d.first_status = out.first_gpu_status_code;
        d.maximum_active_contacts = out.maximum_active_contacts;
        d.gpu_milliseconds = out.gpu_milliseconds;
        if (result) publish(state, batch, config, *result);
        return d;
    }

    // One self-contained rollout: initialize, run, publish, release.
    WorldDiagnostics run(const CompiledWorld& world, const WorldBatch& batch, const WorldStepConfig& config, WorldResult& result) {
        WorldResidentState state;
        return initializeResidentState(world, batch, config, state, &result);
    }

private:
    static void check(int rc, const char* what) {
        if (rc != 0) throw std::runtime_error(std::string(what) + ": " + mr_last_error());
    }

    static void publish(const WorldResidentState& state, const WorldBatch& batch, const WorldStepConfig& config, WorldResult& r) {
        const MRTaskRolloutLayoutC& L = state.layout_;
        const std::size_t envs = L.environment_count, steps = batch.control_step_count;
        r.nq = L.nq;
        r.nv = L.nv;
        const std::uint32_t* st = mr_task_rollout_status_codes(state.handle_);
        const std::uint32_t* ac = mr_task_rollout_active_contacts(state.handle_);
        r.statuses.assign(st, st + steps * envs);
        r.active_contacts.assign(ac, ac + steps * envs);
        if (config.publish_final_state) {
            const float* q = mr_task_rollout_final_q(state.handle_);
            const float* obs = mr_task_rollout_actor_observations(state.handle_);
            if (q) r.final_q.assign(q, q + envs * L.nq);
            if (obs) r.observations.assign(obs, obs + steps * envs * (L.nq + L.nv));
        }
        if (L.scene_body_count) {
            r.final_scene_bodies.resize(envs * L.scene_body_count * 13);
            check(mr_task_rollout_copy_final_scene_states(state.handle_, r.final_scene_bodies.data(), r.final_scene_bodies.size()),
                  "copy_final_scene_states");
        }
    }
};

}  // namespace numi
