// The task layer on either side of the control step (reference:
// src/metal/LocomotionTask.metal: mr_locomotion_task_observe :2184,
// mr_locomotion_task_apply_actions :3442, mr_locomotion_task_complete
// :3904): launch parameters of its three kernels (task.cu) and the
// per-environment records they keep in HBM.
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

#include "device_model.h"
#include "numi_b200.h"

namespace numi {

constexpr int kTaskMaxActions = 64;
constexpr int kTaskMaxGroups = 8;          // contact groups
constexpr int kTaskGroupMetrics = 12;      // per group: force, slip, air time, clearance, CoP x, y; wrench force xyz, torque xyz
constexpr int kTaskMaxObservations = 256;  // the policy's widest input
constexpr int kTaskMaxHistory = 8;

// Per-environment task state (the reference's MRTaskStateGPU, the lanes the
// evaluated subset uses).
struct alignas(16) TaskEnvState {
    std::uint32_t episode_step;  // control steps completed in this episode
    std::uint32_t episode;       // episodes started; keys the episode's draws
    std::uint32_t command_steps; // control steps until the next command draw
    std::uint32_t initialized;
    std::uint32_t pending_reset; // the last step ended the episode
    std::uint32_t last_reason;
    std::uint32_t action_delay;       // raw actions of delay this episode
    std::uint32_t observation_delay;  // frames of delay this episode
    float command[3];            // x, y velocity and yaw rate
    float phase;                 // gait phase in [0, 2 pi)
    float previous_height;       // root height at the last step's end
    float episode_return;
    float episode_tracking;      // sum of the linear tracking scores
    float reserved2;
    std::uint32_t band;          // the episode's difficulty band
    std::uint32_t reserved3[3];
};
static_assert(sizeof(TaskEnvState) == 80, "task state layout");

// The installed program: tables in one device arena plus its constants.
struct TaskProgramDevice {
    const MRTaskActionBindingC* actions;
    const MRTaskObservationOperatorC* actor;
    const MRTaskObservationOperatorC* critic;
    const MRTaskRewardOperatorC* rewards;
    const MRTaskTerminationOperatorC* terminations;
    const MRTaskRandomizationOperatorC* randomization;
    const MRTaskIndexGroupC* groups;
    const std::uint32_t* members;
    const float* default_q;    // [nq]
    const float* limit_lower;  // [na]: position limits of each action's DoF
    const float* limit_upper;
    const MRTaskContactGroupC* contact_groups;
    const std::uint32_t* contact_members;
    const DeviceModel* model;  // the world (body tree, shapes, pairs) for the contact groups' kinematics
    std::int32_t ncontact_groups;
    float support_force_threshold, clearance_target, physics_dt, ground_height;
    std::int32_t na, nobs, nrewards, nterminations, nrandom, ngroups;
    std::int32_t history, delay, max_episode_steps, nq, nv;
    std::int32_t frames;       // actor frames stacked in an observation (oldest first)
    std::int32_t max_observation_delay;
    std::int32_t ncritic;      // critic operators (0: the critic reads the actor history)
    std::int32_t fixed_root;   // the root is welded to the world: root sources read zero
    float dt;                  // control step, seconds
    float base_height, gait_period, standing_probability, duration_min, duration_max;
    float root_reference[3];
    float command_lower[3], command_upper[3];
    float command_limit_lower[3], command_limit_upper[3], command_step[3];
    std::int32_t bands, band_min, band_max;  // band count; the rollout's sampled band range
    float band_exponent;
    unsigned long long seed;
};

// One launch over environments [env_base, env_base + env_count) of one
// control step.  Per-environment pointers are offset to env_base.
struct TaskParams {
    TaskProgramDevice prog;
    TaskEnvState* state;           // [env]
    float* action_history;         // [env][history][na]: raw slots 0..history-2, filter slot history-1
    float* previous_joint;         // [env][2][na]: joint velocity, joint position at the last step's end
    float* frame;                  // [env][frames][nobs]: the actor history of the next decision, oldest first
    float* critic_frame;           // [env][ncritic]: the critic's frame of the next decision
    float* reset_q;                // [env][nq]
    float* reset_v;                // [env][nv]
    const float* q;                // [env][nq]
    const float* v;                // [env][nv]
    const std::uint32_t* masks_in; // caller's reset masks of this step [env], or null
    std::uint32_t* masks_out;      // [env]: the step's resets
    float* observations;           // [env][frames * nobs] of this step, or null
    const float* actions;          // [env][na] of this step
    float* targets;                // [env][na]: drive targets for the control step
    const std::uint32_t* status;   // [env] of this step
    const float* manifolds;        // [env][pair][56]: the step's committed contacts (contact groups)
    float* air_time;               // [env][kTaskMaxGroups]
    MRTaskTransitionC* transitions;// [env] of this step
    unsigned long long policy_revision;
    std::int32_t env_count, env_base;
};

cudaError_t launch_task_observe(const TaskParams& p, cudaStream_t stream);
cudaError_t launch_task_apply(const TaskParams& p, cudaStream_t stream);
cudaError_t launch_task_complete(const TaskParams& p, cudaStream_t stream);

}  // namespace numi
