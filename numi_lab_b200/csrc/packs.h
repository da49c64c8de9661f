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

// A task transition as the learner's record (c_api.cpp's publication).
LearningTransition learning_transition(const MRTaskTransitionC& t);
// The C record -> the owned record (spans copied, transitions converted).
PolicyRolloutPackData policy_rollout_pack_from_c(const MRPolicyRolloutPackC& c);
// Throws std::invalid_argument on a pack the reference's writer refuses.
void validate_policy_rollout_pack(const PolicyRolloutPackData& d);
void write_policy_rollout_pack(const PolicyRolloutPackData& d, const std::string& path);
PolicyRolloutPackData read_policy_rollout_pack(const std::string& path);

}  // namespace numi
