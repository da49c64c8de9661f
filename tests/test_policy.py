"""Native policy (mr_task_rollout_set_policy): the device's fused dense
actor / critic and action sampler (numi_lab_b200/csrc/policy.cu) against
the FP64 restatement (oracle/policy.py) of the reference's
PolicyInference.metal, and the closed loop against an open-loop rollout
fed the same actions.

Tolerances: the device evaluates in FP32 with FMA in the reference's
order; over layers of <= 256 inputs the actor's mean agrees with FP64 to
~1e-6 relative, held at 1e-4 absolute on the tanh-bounded means and
latents (the Gaussian draw's log / cos in FP32 add ~1e-6).
"""

from __future__ import annotations

import numpy as np
import pytest

import numi_lab_b200 as nb
from oracle import policy as ref

TOL = 1e-4
SEED = 5


def _network(rng, sizes, acts):
    layers = []
    for (n_in, n_out), a in zip(zip(sizes[:-1], sizes[1:]), acts):
        layers.append((rng.normal(0.0, 1.0 / np.sqrt(n_in), (n_out, n_in)).astype(np.float32),
                       rng.normal(0.0, 0.1, n_out).astype(np.float32), a))
    return layers


def _policy(world, rng, stochastic: bool):
    nobs, na = world.observation_count, world.action_count
    actor = _network(rng, [nobs, 256, 128, na], ["elu", "silu", "tanh"])
    critic = _network(rng, [nobs, 64, 1], ["relu", "identity"])
    spec = dict(
        layers=actor, critic_layers=critic, revision=7, action_clip=2.5,
        observation_mean=rng.normal(0.0, 0.1, nobs).astype(np.float32),
        observation_inverse_std=rng.uniform(0.5, 2.0, nobs).astype(np.float32), observation_clip=5.0,
        critic_observation_mean=np.zeros(nobs, np.float32), critic_observation_inverse_std=np.ones(nobs, np.float32),
        action_bias=rng.normal(0.0, 0.05, na).astype(np.float32), action_scale=rng.uniform(0.3, 0.6, na).astype(np.float32),
        action_log_std=np.full(na, -1.0, np.float32) if stochastic else None,
    )
    return spec


def test_policy_oracle_restates_the_layer_order_and_sampler():
    """CPU: the restatement's pieces -- normalisation clamp, activation
    set, the sampler's law (unit-variance draws, log-probability of a
    Gaussian) -- on a small hand-made network."""
    rng = np.random.default_rng(1)
    w = np.array([[1.0, -2.0], [0.5, 0.25]])
    layers = [(w, np.array([0.1, -0.1]), "identity")]
    x = np.array([[0.3, -0.4], [10.0, 0.0]])
    out = ref.forward(x, layers, mean=np.zeros(2), inv_std=np.ones(2), clip=1.0)
    np.testing.assert_allclose(out[0], w @ x[0] + [0.1, -0.1])
    np.testing.assert_allclose(out[1], w @ [1.0, 0.0] + [0.1, -0.1])  # clipped input
    for name, f in ref.ACTIVATIONS.items():
        assert np.isfinite(f(np.linspace(-3, 3, 7))).all(), name
    key = ref.policy_key(3, 7)
    draws = np.array([ref.standard_normal(key, e, s, a) for e in range(40) for s in range(5) for a in range(10)])
    assert abs(draws.mean()) < 0.1 and abs(draws.std() - 1.0) < 0.1
    actions, latents, lp = ref.act(np.zeros((3, 2)), layers, action_clip=1.0, key=key, step=0, log_std=np.array([-1.0, 0.0]))
    n = (latents - ref.forward(np.zeros((3, 2)), layers)) / np.exp([-1.0, 0.0])
    np.testing.assert_allclose(lp, np.sum(-0.5 * n * n - np.array([-1.0, 0.0]) - 0.5 * np.log(2 * np.pi), axis=1))
    assert (np.abs(actions) <= 1.0).all()
    del rng


@pytest.mark.gpu
@pytest.mark.parametrize("stochastic,chains", [(False, "1"), (True, "1"), (True, "3")])
def test_policy_actions_match_the_oracle(cuda_device, monkeypatch, stochastic, chains):
    """Three chains: each block's draws are keyed on the absolute slot."""
    monkeypatch.setenv("NUMI_B200_CHAINS", chains)
    rng = np.random.default_rng(11 if stochastic else 12)
    envs, steps = 64, 3
    with nb.World("tree29", envs, substeps=4, velocity_iterations=8, control_dt=0.02, seed=SEED) as world:
        spec = _policy(world, rng, stochastic)
        world.set_policy(**spec)
        assert world.policy_revision == 7
        key = ref.policy_key(SEED, 7)
        for k in range(steps):
            q0, v0, _ = world.state()
            _, status = world.step_policy(1)
            assert int(status.abs().sum()) == 0
            out = world.policy_outputs()
            obs = np.concatenate([q0, v0], axis=1).astype(np.float64)
            actions, latents, lp = ref.act(obs, spec["layers"], action_clip=spec["action_clip"], key=key, step=k,
                                           mean=spec["observation_mean"], inv_std=spec["observation_inverse_std"],
                                           obs_clip=spec["observation_clip"], log_std=spec["action_log_std"],
                                           action_bias=spec["action_bias"], action_scale=spec["action_scale"])
            assert float(np.max(np.abs(out["latents"][0] - latents))) <= TOL
            assert float(np.max(np.abs(out["log_probabilities"][0] - lp))) <= TOL * world.action_count
            values = ref.forward(obs, spec["critic_layers"], spec["critic_observation_mean"],
                                 spec["critic_observation_inverse_std"], spec["observation_clip"])[:, 0]
            assert float(np.max(np.abs(out["values"][0] - values))) <= TOL


@pytest.mark.gpu
@pytest.mark.parametrize("chains", ["1", "3"])
def test_policy_closed_loop_equals_open_loop_with_its_actions(cuda_device, monkeypatch, chains):
    """A policy-driven advance applies exactly the actions it reports: an
    open-loop rollout fed clamp(scale x latent + bias) ends bit-identical,
    and evaluate_final_policy gives the critic on the final state."""
    import torch

    monkeypatch.setenv("NUMI_B200_CHAINS", chains)  # three chains: each evaluates the policy on its own block
    rng = np.random.default_rng(3)
    envs, steps = 32, 6
    with nb.World("tree29", envs, substeps=4, velocity_iterations=8, control_dt=0.02, seed=SEED) as a, \
            nb.World("tree29", envs, substeps=4, velocity_iterations=8, control_dt=0.02, seed=SEED) as b:
        spec = _policy(a, rng, True)
        a.set_policy(**spec)
        res = a.advance_host(None, steps=steps, evaluate_final_policy=True, raise_on_failure=False)
        assert int(res["counters"].failed_environment_steps) == 0
        out = a.policy_outputs()
        acts = np.clip(spec["action_scale"] * out["latents"].astype(np.float64) + spec["action_bias"], -spec["action_clip"],
                       spec["action_clip"])
        # The device formed each action in FP32 with one FMA.
        acts32 = np.clip(np.float32(spec["action_scale"]) * out["latents"] + np.float32(spec["action_bias"]), -2.5, 2.5)
        assert float(np.max(np.abs(acts - acts32))) <= 1e-6
        fma = np.array([[[np.float32(np.float64(s) * np.float64(l) + np.float64(c)) for s, l, c in
                          zip(spec["action_scale"], out["latents"][k, e], spec["action_bias"])] for e in range(envs)]
                        for k in range(steps)], np.float32)
        b.step(torch.from_numpy(np.clip(fma, -2.5, 2.5)).cuda(), wait=True)
        qa, va, _ = a.state()
        qb, vb, _ = b.state()
        assert np.array_equal(qa, qb) and np.array_equal(va, vb)
        final = np.concatenate([qa, va], axis=1).astype(np.float64)
        values = ref.forward(final, spec["critic_layers"], spec["critic_observation_mean"], spec["critic_observation_inverse_std"],
                             spec["observation_clip"])[:, 0]
        assert float(np.max(np.abs(out["bootstrap_values"] - values))) <= TOL
        # Without the policy the rollout wants actions again.
        a.clear_policy()
        assert a.policy_revision == 0
        with pytest.raises(nb.MetalRoboError):
            a.advance_host(None, steps=1)


@pytest.mark.gpu
def test_policy_install_rejects_mismatched_networks(cuda_device):
    rng = np.random.default_rng(4)
    with nb.World("tree29", 4, seed=SEED) as world:
        spec = _policy(world, rng, False)
        bad = dict(spec, layers=spec["layers"][:-1])  # ends in 128 outputs, not the 29 actions
        with pytest.raises(nb.MetalRoboError, match="must end in"):
            world.set_policy(**bad)
        with pytest.raises(nb.MetalRoboError, match="revision"):
            world.set_policy(**dict(spec, revision=0))
        wide = _network(rng, [world.observation_count, 300, world.action_count], ["relu", "tanh"])
        with pytest.raises(nb.MetalRoboError, match="outputs"):
            world.set_policy(**dict(spec, layers=wide))
        assert world.policy_revision == 0


@pytest.mark.gpu
def test_policy_pack_file_drives_the_rollout_like_the_in_memory_policy(cuda_device, tmp_path):
    """A PolicyPack written by the reference's own writer (oracle/_ref) or by
    this library, loaded with mr_task_rollout_load_policy_pack, drives a
    rollout bit-identically to the same policy installed from memory; a
    failed load (a corrupt file) leaves the installed policy in place."""

    from test_packs import CONTRACT

    rng = np.random.default_rng(8)
    envs, steps = 32, 5
    kw = dict(substeps=4, velocity_iterations=8, control_dt=0.02, seed=SEED)
    with nb.World("tree29", envs, **kw) as a, nb.World("tree29", envs, **kw) as b:
        spec = dict(_policy(a, rng, True), policy_id="g1-walk", contract=CONTRACT, observation_clip=5.0)
        path = tmp_path / "policy.mrpolicy"
        try:
            from oracle import reference_write_policy_pack

            pk, keep = nb.world.policy_pack_c(**spec)
            reference_write_policy_pack(pk, path)
            del keep
        except FileNotFoundError:  # no reference core on this host: this library's writer (byte-identical)
            nb.write_policy_pack(path, **spec)
        a.set_policy(**{k: v for k, v in spec.items() if k != "contract"})
        b.load_policy_pack(path)
        assert a.policy_revision == b.policy_revision == spec["revision"]
        a.advance_host(None, steps=steps, raise_on_failure=False)
        b.advance_host(None, steps=steps, raise_on_failure=False)
        qa, va, _ = a.state()
        qb, vb, _ = b.state()
        assert np.array_equal(qa, qb) and np.array_equal(va, vb)
        assert np.array_equal(a.policy_outputs()["latents"], b.policy_outputs()["latents"])
        corrupt = tmp_path / "corrupt.mrpolicy"
        data = bytearray(path.read_bytes())
        data[-60] ^= 0x10
        corrupt.write_bytes(bytes(data))
        with pytest.raises(nb.MetalRoboError, match="hash"):
            b.load_policy_pack(corrupt)
        assert b.policy_revision == spec["revision"]
        b.advance_host(None, steps=1, raise_on_failure=False)  # the installed policy still drives it
