// Native policy on the device: the reference's dense layer operator
// (mr_policy_dense_layer, PolicyInference.metal:80-160) and action sampler
// (mr_policy_sample_and_score, :162-268) fused into one kernel per control
// step.  A CTA takes kPolicyTile (8) environments through every actor layer
// (and the critic), the activations of the tile living in shared memory;
// thread j owns output neuron j and keeps one accumulator per environment,
// so each weight is read once per CTA and used kPolicyTile times.  Weights
// are stored [input][output] so a warp's weight loads are contiguous; the
// environment's input value is a shared-memory broadcast.  Each output
// starts from its bias and accumulates inputs in ascending order with FMA,
// the reference's order.  FP32 throughout, as the reference evaluates: at
// 4096 environments a 71-256-128-29 actor plus a 71-64-1 critic take 85 us
// per launch against 1.22 ms for the contact control step it feeds, so
// tensor-core operands (bf16 / tf32) would change the actions to save at
// most 7 % of a step.
#include "policy.h"

#include <cstdint>

#include "numi_b200.h"

namespace numi {
namespace {

constexpr int kThreads = kPolicyMaxWidth;

__device__ __forceinline__ float activate(int op, float x) {
    switch (op) {
        case MR_POLICY_ACTIVATION_C_IDENTITY: return x;
        case MR_POLICY_ACTIVATION_C_RELU: return fmaxf(x, 0.0f);
        case MR_POLICY_ACTIVATION_C_TANH: return tanhf(x);
        case MR_POLICY_ACTIVATION_C_ELU: return x >= 0.0f ? x : expf(x) - 1.0f;
        case MR_POLICY_ACTIVATION_C_SILU: return x / (1.0f + expf(-x));
        default: return 0.0f;
    }
}

// SplitMix64's output function (Steele, Lea and Flood 2014): the counter-based
// generator of the policy's Gaussian draws.
__device__ __forceinline__ unsigned long long mix64(unsigned long long x) {
    x += 0x9e3779b97f4a7c15ull;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}
// Uniform in (0, 1) from the top 24 bits.
__device__ __forceinline__ float uniform01(unsigned long long key) {
    return (static_cast<float>(static_cast<unsigned>(mix64(key) >> 40)) + 0.5f) * (1.0f / 16777216.0f);
}
// Standard normal for (env key, action): Box-Muller on two draws.
__device__ __forceinline__ float normal_draw(unsigned long long key, int action) {
    const unsigned long long base = key + 2ull * static_cast<unsigned long long>(action);
    const float u1 = uniform01(base), u2 = uniform01(base + 1ull);
    return sqrtf(-2.0f * logf(u1)) * cospif(2.0f * u2);
}

// Observation feature i of the tile's environment e into x (normalised).
__device__ __forceinline__ void load_observation(const PolicyParams& p, const float* mean, const float* inv_std, int env0,
                                                 float* x, bool critic = false) {
    const float* frame = critic && p.critic_frame ? p.critic_frame : p.frame;
    const int nobs = critic && p.critic_frame ? p.critic_frame_count : (p.frame ? p.frame_count : p.nq + p.nv);
    for (int idx = threadIdx.x; idx < kPolicyTile * nobs; idx += blockDim.x) {
        const int e = idx / nobs, i = idx - e * nobs;
        const int env = env0 + e;
        float value = 0.0f;
        if (env < p.envs) {
            if (frame)
                value = frame[static_cast<size_t>(env) * nobs + i];
            else
                value = i < p.nq ? p.q[static_cast<size_t>(env) * p.nq + i] : p.v[static_cast<size_t>(env) * p.nv + (i - p.nq)];
            if (mean) value = fminf(fmaxf((value - mean[i]) * inv_std[i], -p.obs_clip), p.obs_clip);
        }
        x[e * kPolicyMaxWidth + i] = value;
    }
}

// Dense layers in place over the two tile buffers; returns the buffer that
// holds the last layer's outputs.
__device__ float* forward(const PolicyLayer* layers, int count, float* x, float* y) {
    for (int l = 0; l < count; ++l) {
        __syncthreads();
        const PolicyLayer L = layers[l];
        const int j = threadIdx.x;
        if (j < L.out) {
            float acc[kPolicyTile];
            const float b = L.bias[j];
#pragma unroll
            for (int e = 0; e < kPolicyTile; ++e) acc[e] = b;
            const float* w = L.weights_t + j;
            // Four inputs per shared-memory load (rows are 16-byte aligned),
            // still accumulated in ascending input order.
            const int in4 = L.in & ~3;
            for (int k = 0; k < in4; k += 4) {
                const float w0 = w[static_cast<size_t>(k) * L.out], w1 = w[static_cast<size_t>(k + 1) * L.out],
                            w2 = w[static_cast<size_t>(k + 2) * L.out], w3 = w[static_cast<size_t>(k + 3) * L.out];
#pragma unroll
                for (int e = 0; e < kPolicyTile; ++e) {
                    const float4 xv = *reinterpret_cast<const float4*>(x + e * kPolicyMaxWidth + k);
                    float a = acc[e];
                    a = __fmaf_rn(w0, xv.x, a);
                    a = __fmaf_rn(w1, xv.y, a);
                    a = __fmaf_rn(w2, xv.z, a);
                    acc[e] = __fmaf_rn(w3, xv.w, a);
                }
            }
            for (int k = in4; k < L.in; ++k) {
                const float wk = w[static_cast<size_t>(k) * L.out];
#pragma unroll
                for (int e = 0; e < kPolicyTile; ++e) acc[e] = __fmaf_rn(wk, x[e * kPolicyMaxWidth + k], acc[e]);
            }
#pragma unroll
            for (int e = 0; e < kPolicyTile; ++e) y[e * kPolicyMaxWidth + j] = activate(L.activation, acc[e]);
        }
        float* t = x;
        x = y;
        y = t;
    }
    __syncthreads();
    return x;
}

__global__ void __launch_bounds__(kThreads) policy_kernel(PolicyParams p) {
    extern __shared__ float tile[];
    float* a = tile;
    float* b = tile + kPolicyTile * kPolicyMaxWidth;
    const int env0 = blockIdx.x * kPolicyTile;

    // Actor: mean, then latent, action and log-probability per environment
    // (one thread per environment, actions in order: the reference's
    // accumulation order of the log-probability).
    load_observation(p, p.obs_mean, p.obs_inv_std, env0, a);
    const float* mean = forward(p.actor, p.actor_layers, a, b);
    const int e = threadIdx.x;
    if (e < kPolicyTile && env0 + e < p.envs) {
        const int env = env0 + e;
        const unsigned long long step = *p.step_base + static_cast<unsigned long long>(p.step_offset);
        const unsigned long long slot = static_cast<unsigned long long>(env + p.env_base);
        const unsigned long long key = mix64(p.key ^ mix64((slot << 32) ^ step));
        float log_prob = 0.0f;
        constexpr float kHalfLogTwoPi = 0.91893853320467274178f;
        for (int act = 0; act < p.na; ++act) {
            const float m = mean[e * kPolicyMaxWidth + act];
            float latent = m;
            if (p.log_std) {
                const float ls = p.log_std[act];
                const float n = normal_draw(key, act);
                latent = __fmaf_rn(expf(ls), n, m);
                log_prob += -0.5f * n * n - ls - kHalfLogTwoPi;
            }
            const float action = fminf(fmaxf(__fmaf_rn(p.action_scale[act], latent, p.action_bias[act]), -p.action_clip), p.action_clip);
            const size_t o = static_cast<size_t>(env) * p.na + act;
            if (p.actions) p.actions[o] = action;
            if (p.latents) p.latents[o] = latent;
        }
        if (p.log_prob) p.log_prob[env] = log_prob;
    }
    if (p.values == nullptr) return;
    if (p.critic_layers == 0) {
        if (e < kPolicyTile && env0 + e < p.envs) p.values[env0 + e] = 0.0f;
        return;
    }
    __syncthreads();
    load_observation(p, p.critic_mean, p.critic_inv_std, env0, a, true);
    const float* value = forward(p.critic, p.critic_layers, a, b);
    if (e < kPolicyTile && env0 + e < p.envs) p.values[env0 + e] = value[e * kPolicyMaxWidth];
}

__global__ void counter_kernel(unsigned long long* counter, unsigned long long steps) { *counter += steps; }

constexpr size_t kSmemBytes = 2ull * kPolicyTile * kPolicyMaxWidth * sizeof(float);

}  // namespace

cudaError_t configure_policy_kernel() {
    return cudaFuncSetAttribute(policy_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kSmemBytes));
}

cudaError_t launch_policy(const PolicyParams& p, cudaStream_t stream) {
    const int blocks = (p.envs + kPolicyTile - 1) / kPolicyTile;
    policy_kernel<<<blocks, kThreads, kSmemBytes, stream>>>(p);
    return cudaGetLastError();
}

cudaError_t launch_policy_counter(unsigned long long* counter, unsigned long long steps, cudaStream_t stream) {
    counter_kernel<<<1, 1, 0, stream>>>(counter, steps);
    return cudaGetLastError();
}

}  // namespace numi
