// PolicyPack files: numi-lab's persisted policy artifact (reference:
// include/metalrobo/PolicyProgram.hpp:56-76 for the record,
// src/core/LearningPacks.cpp for the container and its wire encoding).
//
// A pack file is a 32-byte little-endian header -- magic "MRLEARN\0",
// format version (u32), artifact kind (u32, 2 for a policy), payload bytes
// (u64), payload hash (u64, FNV-1a 64 with a zero result mapped to one) --
// followed by the payload: the policy id (u64 length + bytes), revision
// (u64), the actor's observation mean and inverse standard deviation
// (u64 count + FP32 values each), the actor layers (u64 count; per layer
// input count, output count, activation as u32, weights [output][input] and
// bias as counted FP32 vectors), the critic's normalisation and layers in the
// same encoding, the action log standard deviation, bias and scale vectors,
// the observation and action clips (FP32), and, from format version 4, the
// semantic contract (version, world, task, observation and action
// fingerprints, u64 each).  Version 3 packs end after the clips.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "numi_b200.h"

namespace numi {

constexpr std::uint32_t kPolicyPackKind = 2u;
constexpr std::uint32_t kPolicyPackVersion = 4u;        // written
constexpr std::uint32_t kPolicyPackOldestVersion = 3u;  // read

struct PolicyPackLayer {
    std::uint32_t input_count = 0, output_count = 0, activation = 0;
    std::vector<float> weights, bias;
};

// An owned PolicyPack (the fields of MRPolicyPackC).
struct PolicyPackData {
    std::uint32_t format_version = kPolicyPackVersion;
    std::string id;
    std::uint64_t revision = 0;
    std::uint64_t contract_version = 0, world_fingerprint = 0, task_fingerprint = 0, observation_fingerprint = 0,
                  action_fingerprint = 0;
    std::vector<float> observation_mean, observation_inverse_std;
    std::vector<PolicyPackLayer> layers;
    std::vector<float> critic_observation_mean, critic_observation_inverse_std;
    std::vector<PolicyPackLayer> critic_layers;
    std::vector<float> action_log_std, action_bias, action_scale;
    float observation_clip = 100.0f, action_clip = 0.0f;
    std::uint64_t content_hash = 0;  // of the payload read or written
};

// FNV-1a 64 of a payload, zero mapped to one.
std::uint64_t learning_pack_hash(const void* bytes, std::size_t count);

// The C record <-> the owned record (spans copied).
PolicyPackData policy_pack_from_c(const MRPolicyPackC& c);
// A view of `d` (valid while `d` and `storage` live).
MRPolicyPackC policy_pack_view(const PolicyPackData& d, std::vector<MRPolicyDenseLayerC>& storage);

// Throws std::invalid_argument with a message on an invalid pack (the
// artifact rules of the reference's writer: identity, non-zero revision, an
// exact contract, positive finite clips, layer shapes, finite values, a
// critic for a stochastic actor).
void validate_policy_pack(const PolicyPackData& d);

// Atomically writes a version-4 pack (sibling temporary, fsync, rename).
void write_policy_pack(const PolicyPackData& d, const std::string& path);
// Reads and checks a version 3 or 4 pack; throws with a message.
PolicyPackData read_policy_pack(const std::string& path);
// FNV-1a 64 of a pack's payload as this library encodes it (version 4):
// the installed policy's fingerprint.
std::uint64_t policy_pack_payload_hash(const PolicyPackData& d);

// PolicyRolloutPack files (reference: include/metalrobo/LearningPacks.hpp:54-105,
// src/core/LearningPacks.cpp:726-918 rules, :1818-1867 payload): the same
// container with artifact kind 3, format version 7, and a payload of the id,
// task and policy fingerprints and revision (u64), environment, control-step,
// actor-observation, critic-observation, action and motion-feature counts
// (u32), eight counted FP32 tables (actor and critic observations, motion
// features, teacher actions, latents, log-probabilities, values, bootstrap
// values), the outcome schema (u64 count; id, unit, direction u32 each), the
// outcome values and the learning transitions (u64 count + 64-byte records).
constexpr std::uint32_t kPolicyRolloutPackKind = 3u;
constexpr std::uint32_t kPolicyRolloutPackVersion = 7u;

// MRLearningTransitionGPU (task_program_types.h:633-643).
struct LearningTransition {
    float reward, timeout_bootstrap_value, reserved0, reserved1;
    std::uint32_t done, timeout, physics_error, termination_reason;
    std::uint32_t difficulty_band, terrain_level, impact_sequence_index, impact_event_flags;
    std::uint64_t policy_revision, reserved;
};
static_assert(sizeof(LearningTransition) == 64, "learning transition layout");

struct PolicyOutcome {
    std::string id, unit;
    std::uint32_t direction = 0;
};

struct PolicyRolloutPackData {
    std::string id;
    std::uint64_t task_fingerprint = 0, policy_fingerprint = 0, policy_revision = 0;
    std::uint32_t environment_count = 0, control_step_count = 0, actor_observation_count = 0, critic_observation_count = 0,
                  action_count = 0, motion_feature_count = 0;
    std::vector<float> actor_observations, critic_observations, motion_features, teacher_actions, latents, log_probabilities, values,
        bootstrap_values;
    std::vector<PolicyOutcome> outcomes;
    std::vector<float> outcome_values;  // [sample][outcome]
    std::vector<LearningTransition> transitions;
    std::uint64_t content_hash = 0;
};

// TaskPack files (reference: include/metalrobo/TaskProgram.hpp:211-500,
// src/core/LearningPacks.cpp:81-258 rules, :1127-1262 payload): the same
// container with artifact kind 1, format version 17.  The authored task is
// name-based (actuators, bodies, joints are strings resolved against a robot
// when compiled); the payload keeps the reference's field order and
// encodings: strings and string lists as u64 counts + bytes, enums as u32,
// booleans as u8, four-float records as 16 bytes, the capacity profile as
// its 27 u32 fields.
constexpr std::uint32_t kTaskPackKind = 1u;
constexpr std::uint32_t kTaskPackVersion = 17u;
constexpr std::size_t kCapacityProfileWords = 27;

struct TaskPackOutcome {
    std::string id, unit;
    std::uint32_t source = 2u, direction = 0u, reward_operation = 2u;
};
struct TaskPackContactGroup {
    std::string id;
    std::vector<std::string> bodies;
    std::uint8_t support = 0, forbidden = 0;
    std::string reference_body;
    float local_reference[4] = {};
    float gait_phase_offset = 0.0f, stance_fraction = 0.5f;
    float support_patch_bounds[4] = {};
    std::uint32_t support_patch_width = 0, support_patch_height = 0;
};
struct TaskPackJointGroup {
    std::string id;
    std::vector<std::string> joints;
};
struct TaskPackReward {
    std::uint32_t operation = 2u;
    std::string source_group, target;
    float weight = 0.0f;
    float parameters[4] = {};
};
struct TaskPackTermination {
    std::uint32_t operation = 0u;
    std::string source_group;
    std::uint32_t reason = 1u, priority = 0u;
    float threshold = 0.0f, failure_penalty = 0.0f;
    std::uint32_t minimum_band = 0u, maximum_band = 0xffffffffu;
};

struct TaskPackData {
    std::string id;
    std::uint32_t capacities[kCapacityProfileWords] = {};
    std::vector<std::string> actions;
    std::vector<TaskPackOutcome> outcomes;
    std::vector<TaskPackContactGroup> contact_groups;
    std::vector<TaskPackJointGroup> joint_groups;
    std::vector<TaskPackReward> rewards;
    std::vector<TaskPackTermination> terminations;
    // Commands: lower, upper, limit lower, limit upper, difficulty step (xyzw each).
    float commands[5][4] = {};
    float standing_probability = 0.0f, difficulty_sampling_exponent = 2.0f, command_duration[2] = {5.0f, 10.0f};
    // Pushes: maximum velocity, interval minimum / maximum, projectile standing
    // probability, target radius, horizontal speed lower / upper, target height lower / upper.
    float pushes[9] = {0.0f, 2.0f, 5.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    std::string terrain_body;
    std::vector<float> terrain_sample_offsets, terrain_reset_translations;  // xyzw each
    std::string threat_protected_group;
    // Activation speed, horizon, safety margin, CBF alpha, step-over / sidestep /
    // lean maximum heights, urgency, desired-velocity horizon, projection epsilon.
    float threat[10] = {0.5f, 2.0f, 0.05f, 2.0f, 0.35f, 0.75f, 1.10f, 0.35f, 0.20f, 1.0e-5f};
    std::string motion_anchor;
    std::vector<std::string> motion_tracked;
    std::uint32_t maximum_episode_steps = 1000u, difficulty_band_count = 1u;
    float interaction_student_authority = 0.1f, interaction_reset_phase_fraction = 0.0f;
    std::vector<float> initial_action_positions;
    std::uint8_t interaction_control_reference = 1, interaction_initialize_from_reference = 1, interaction_align_reference_yaw = 0;
    float base_height_target = 0.0f, gait_period = 0.8f, clearance_target = 0.1f, success_tracking_threshold = 0.8f,
          support_force_threshold = 1.0f;
    std::uint64_t content_hash = 0;
};

// Throws std::invalid_argument on a pack the reference's writer refuses.
void validate_task_pack(const TaskPackData& d);
void write_task_pack(const TaskPackData& d, const std::string& path);
TaskPackData read_task_pack(const std::string& path);

// A task transition as the learner's record (c_api.cpp's publication).
LearningTransition learning_transition(const MRTaskTransitionC& t);
// The C record -> the owned record (spans copied, transitions converted).
PolicyRolloutPackData policy_rollout_pack_from_c(const MRPolicyRolloutPackC& c);
// Throws std::invalid_argument on a pack the reference's writer refuses.
void validate_policy_rollout_pack(const PolicyRolloutPackData& d);
void write_policy_rollout_pack(const PolicyRolloutPackData& d, const std::string& path);
PolicyRolloutPackData read_policy_rollout_pack(const std::string& path);

}  // namespace numi
