// Native policy evaluation between control steps (the reference's dense
// policy operator and action sampler, PolicyInference.metal): launch
// parameters of the fused actor / critic kernel (policy.cu).
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

namespace numi {

constexpr int kPolicyMaxLayers = 8;
constexpr int kPolicyMaxWidth = 256;  // widest layer (inputs and outputs)
constexpr int kPolicyTile = 8;        // environments per CTA

struct PolicyLayer {
    std::int32_t in, out, activation, reserved;
    const float* weights_t;  // [in][out] (the reference's [out][in], transposed at install)
    const float* bias;       // [out]
};

struct PolicyParams {
    PolicyLayer actor[kPolicyMaxLayers];
    PolicyLayer critic[kPolicyMaxLayers];
    std::int32_t actor_layers, critic_layers;
    const float* obs_mean;      // [observation count] or null (no normalisation)
    const float* obs_inv_std;
    const float* critic_mean;   // [observation count] or null
    const float* critic_inv_std;
    float obs_clip, action_clip;
    const float* log_std;       // [na] or null (deterministic)
    const float* action_bias;   // [na]
    const float* action_scale;  // [na]
    // Observation source: the task layer's actor frames ([env][frame_count])
    // when `frame` is set, else the resident state [q, v].
    const float* q;
    const float* v;
    const float* frame;
    std::int32_t frame_count;
    const float* critic_frame;  // the critic's own frames ([env][critic_frame_count]), or null: it reads `frame`
    std::int32_t critic_frame_count;
    std::int32_t nq, nv, envs, na;
    // Outputs of this control step (per env), any of them null to skip.
    float* actions;    // [env][na]: fed to the control step
    float* latents;    // [env][na]
    float* log_prob;   // [env]
    float* values;     // [env]
    // Draw key: seed and revision mixed; the control-step index is
    // *step_base + step_offset.
    const unsigned long long* step_base;
    std::int32_t step_offset;
    unsigned long long key;
    std::int32_t env_base;  // slot of this launch's environment 0 (state and outputs start there): keys the draws
};

cudaError_t configure_policy_kernel();
cudaError_t launch_policy(const PolicyParams& p, cudaStream_t stream);
// *counter += steps (one thread), after an advance's last evaluation.
cudaError_t launch_policy_counter(unsigned long long* counter, unsigned long long steps, cudaStream_t stream);

}  // namespace numi
