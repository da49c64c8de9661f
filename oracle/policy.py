"""FP64 restatement of the native policy (test infrastructure only: the
checker of numi_lab_b200/csrc/policy.cu, never a product path).

Follows the reference's dense layer operator and action sampler,
src/metal/PolicyInference.metal: each output starts from its bias and
accumulates weight x input over the inputs in order (:124-151), inputs
normalised as clamp((x - mean) * inv_std, +-clip) when a mean is given
(:131-146), activations identity / relu / tanh / elu / silu (:20-37);
latent = mean (+ exp(log sigma) x standard normal), action =
clamp(scale x latent + bias, +-action_clip), log-probability
sum(-n^2 / 2 - log sigma - log(2 pi) / 2) (:214-259).

The Gaussian draws follow this library's counter-based key (the reference
keys its draws on task episodes, which these synthetic worlds do not have):
SplitMix64's output function mixes (seed, revision) into the policy key
and (env, control-step index) into the draw key; action a's standard normal
is Box-Muller on the uniforms of keys 2a and 2a + 1 (top 24 bits).
"""

from __future__ import annotations

import math

import numpy as np

MASK = (1 << 64) - 1
ACTIVATIONS = {
    "identity": lambda x: x,
    "relu": lambda x: np.maximum(x, 0.0),
    "tanh": np.tanh,
    "elu": lambda x: np.where(x >= 0.0, x, np.expm1(np.minimum(x, 0.0))),
    "silu": lambda x: x / (1.0 + np.exp(-x)),
}


def mix64(x: int) -> int:
    x = (x + 0x9E3779B97F4A7C15) & MASK
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & MASK
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & MASK
    return x ^ (x >> 31)


def policy_key(seed: int, revision: int) -> int:
    return mix64(seed & MASK) ^ mix64((revision ^ 0x5BD1E995) & MASK)


def uniform01(key: int) -> float:
    return ((mix64(key) >> 40) + 0.5) / 16777216.0


def standard_normal(policy_key_: int, env: int, step: int, action: int) -> float:
    key = mix64(policy_key_ ^ mix64(((env << 32) ^ step) & MASK))
    base = (key + 2 * action) & MASK
    u1, u2 = uniform01(base), uniform01((base + 1) & MASK)
    return math.sqrt(-2.0 * math.log(u1)) * math.cos(2.0 * math.pi * u2)


def forward(x: np.ndarray, layers, mean=None, inv_std=None, clip: float = 0.0) -> np.ndarray:
    """Dense network on observations x [env][features] (float64)."""
    h = np.asarray(x, np.float64)
    if mean is not None:
        h = np.clip((h - np.asarray(mean, np.float64)) * np.asarray(inv_std, np.float64), -clip, clip)
    for w, b, act in layers:
        w = np.asarray(w, np.float64)
        bias = np.zeros(w.shape[0]) if b is None else np.asarray(b, np.float64)
        h = ACTIVATIONS[act](h @ w.T + bias)
    return h


def act(obs: np.ndarray, layers, *, action_clip: float, key: int, step: int, mean=None, inv_std=None, obs_clip: float = 0.0,
        log_std=None, action_bias=None, action_scale=None):
    """(actions, latents, log-probabilities) for observations [env][features]."""
    mu = forward(obs, layers, mean, inv_std, obs_clip)
    envs, na = mu.shape
    bias = np.zeros(na) if action_bias is None else np.asarray(action_bias, np.float64)
    scale = np.ones(na) if action_scale is None else np.asarray(action_scale, np.float64)
    latents = mu.copy()
    log_prob = np.zeros(envs)
    if log_std is not None:
        ls = np.asarray(log_std, np.float64)
        for e in range(envs):
            n = np.array([standard_normal(key, e, step, a) for a in range(na)])
            latents[e] = mu[e] + np.exp(ls) * n
            log_prob[e] = float(np.sum(-0.5 * n * n - ls - 0.5 * math.log(2.0 * math.pi)))
    actions = np.clip(scale * latents + bias, -action_clip, action_clip)
    return actions, latents, log_prob
