"""The task layer on the device (mr_task_rollout_set_task) against its
oracle (oracle/task.py), through the C ABI, on the 29-DoF contact world:

* step by step in lockstep: each step's actor frames, and its transitions
  (rewards and their breakdown, terminations, timeouts) computed by the
  oracle from the device's post-step state, over short episodes with
  observation noise, an action delay and a first-order response;
* the drive targets: a twin rollout without a task, put in the same state
  and given the oracle's targets, ends each step where the tasked one does;
* a native policy reads the actor frames;
* the installer refuses programs outside the evaluated subset, and
  clearing the task restores [q, v] observations.
"""

from __future__ import annotations

import numpy as np
import pytest

import numi_lab_b200 as nb
from numi_lab_b200 import task as T
from numi_lab_b200.native import MetalRoboError
from oracle.task import TaskOracle

pytestmark = pytest.mark.gpu

SEED = 5
DT = 0.02
OBS_TOL = 2e-5     # FP32 device vs FP64 oracle, same inputs, per value (absolute, scaled by max(1, |x|))
REWARD_TOL = 2e-5


def _default_q(world) -> np.ndarray:
    q, _, _ = nb.sample_reset("tree29", SEED, SEED, 0, 1)
    dq = np.zeros(world.nq, np.float32)
    dq[2], dq[6] = q[0, 2], 1.0
    return dq


def _program(world, **kw):
    return T.locomotion_task(world.model(), _default_q(world), **kw)


def _oracle(world, prog) -> TaskOracle:
    rec = world.model()
    lo = [float(np.float32(rec.dofs[b.dof].limits[0])) for b in prog.actions]
    hi = [float(np.float32(rec.dofs[b.dof].limits[1])) for b in prog.actions]
    return TaskOracle(prog, nq=world.nq, nv=world.nv, dt=DT, seed=world.seed, fixed_root=False, limit_lower=lo, limit_upper=hi)


def _close(a, b, tol) -> float:
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b) / np.maximum(1.0, np.abs(b)))) if a.size else 0.0


@pytest.mark.parametrize("contacts", [False, True])
def test_task_layer_matches_oracle_step_by_step(cuda_device, contacts):
    """With `contacts` the program also has the feet's support groups and a
    forbidden torso group: their metrics in the frames, the contact rewards
    and the contact termination, computed from the committed manifolds."""

    import torch

    from oracle import Oracle

    envs, steps = 16, 40
    bands = (1, 3) if contacts else None
    with nb.World("tree29", envs, substeps=4, velocity_iterations=8, control_dt=DT, seed=SEED, difficulty_bands=bands) as w:
        # Tight height and tilt limits: episodes end by timeout, height and
        # tilt within the run.
        groups = T.foot_contact_groups(w.model()) if contacts else None
        # The contact variant also stacks two actor frames.
        prog = _program(w, maximum_episode_steps=12, noise=0.05, response_time_seconds=0.04, action_history=4,
                        action_delay_steps=1, min_height_fraction=0.995, max_tilt=0.04, contact_groups=groups,
                        observation_history=2 if contacts else 1)
        if contacts:  # per-episode action and observation delays too
            prog.randomization += [T.Randomization(T.RANDOMIZE["action_delay"], (0.0, 2.0, 0.0, 0.0)),
                                   T.Randomization(T.RANDOMIZE["observation_delay"], (0.0, 1.0, 0.0, 0.0))]
            prog.maximum_observation_delay = 1
            # Difficulty bands: episodes draw bands 1-3 (of 4), each band
            # widens the command range; the velocity kick starts at band 2
            # and the tilt termination stops after band 2.
            prog.difficulty_band_count, prog.band_sampling_exponent = 4, 0.8
            prog.command_band_step = (0.2, 0.1, 0.2)
            prog.command_limit_lower, prog.command_limit_upper = (-1.0, -0.6, -1.0), (1.6, 0.6, 1.0)
            prog.randomization.append(T.Randomization(T.RANDOMIZE["velocity"], (-0.2, 0.2, 0.0, 0.0), minimum_band=2))
            prog.terminations[1].maximum_band = 2
        w.set_task(prog)
        assert w.observation_count == len(prog.actor) * prog.observation_history
        o = _oracle(w, prog)
        if contacts:
            o = TaskOracle(prog, nq=w.nq, nv=w.nv, dt=DT, seed=w.seed, fixed_root=False, limit_lower=o.lo, limit_upper=o.hi,
                           records=w.model(), world=Oracle(w.model(), DT / 4, 4, 8, 0), physics_dt=DT / 4, band_range=bands)
        band_seen = set()
        touched = 0
        states = [o.new_state() for _ in range(envs)]
        gen = torch.Generator(device="cuda").manual_seed(3)
        seen = {"reset": 0, "timeout": 0, "height": 0, "tilt": 0}
        worst_obs = worst_reward = 0.0
        for k in range(steps):
            acts = 0.6 * torch.randn((1, envs, w.action_count), device="cuda", generator=gen)
            obs, status, _ = w.step(acts, wait=True)
            obs = obs.cpu().numpy()[0]
            status = status.cpu().numpy()[0]
            q, v, mans = w.state()
            tr = w.transitions(1)
            a_np = acts.cpu().numpy()[0]
            for e in range(envs):
                reset, _, _, want = o.observe(e, states[e], None, None, False)
                seen["reset"] += reset
                worst_obs = max(worst_obs, _close(obs[e], want, OBS_TOL))
                assert _close(obs[e], want, OBS_TOL) <= OBS_TOL, (k, e, int(np.argmax(np.abs(obs[e] - want))))
                o.apply(states[e], a_np[e])
                env_mans = mans[e * w.pair_count:(e + 1) * w.pair_count] if contacts else None
                t = o.complete(e, states[e], q[e].astype(np.float64), v[e].astype(np.float64), int(status[e]), env_mans)
                if contacts:
                    touched += int(np.sum(t["contact_metrics"][:2, 0] > prog.support_force_threshold))
                for f in ("done", "timeout", "physics_error", "termination_reason", "difficulty_band"):
                    assert int(tr[f][0, e]) == t[f], (k, e, f)
                if contacts:
                    band_seen.add(t["difficulty_band"])
                for f in ("reward", "tracking_score", "root_height", "tilt", "task_reward", "base_reward", "joint_velocity_reward",
                          "joint_acceleration_reward", "control_reward", "posture_reward", "contact_reward", "episode_tracking_score"):
                    err = _close(tr[f][0, e], t[f], REWARD_TOL)
                    worst_reward = max(worst_reward, err)
                    assert err <= REWARD_TOL, (k, e, f, float(tr[f][0, e]), t[f])
                seen["timeout"] += t["timeout"]
                seen["height"] += t["termination_reason"] == 1
                seen["tilt"] += t["termination_reason"] == 2
        print(f"worst observation error {worst_obs:.2e}, worst transition error {worst_reward:.2e}; {seen}")
        # The run crossed episode boundaries of each kind it can.
        assert seen["reset"] > envs and seen["timeout"] > 0 and seen["height"] + seen["tilt"] > 0
        if contacts:
            assert touched > 0  # the feet carried load on some steps
            assert band_seen == {1, 2, 3}, band_seen


def test_drive_targets_match_the_oracle(cuda_device):
    """A twin rollout without a task, set to the tasked rollout's state and
    given the oracle's drive targets, lands where the tasked one does."""

    import torch

    envs, steps = 8, 10
    with nb.World("tree29", envs, substeps=4, velocity_iterations=8, control_dt=DT, seed=SEED) as a, \
            nb.World("tree29", envs, substeps=4, velocity_iterations=8, control_dt=DT, seed=SEED) as b:
        prog = _program(a, response_time_seconds=0.03, action_history=4, action_delay_steps=1)
        a.set_task(prog)
        o = _oracle(a, prog)
        states = [o.new_state() for _ in range(envs)]
        gen = torch.Generator(device="cuda").manual_seed(9)
        compared = 0
        for k in range(steps):
            qa, va, ma = a.state()
            acts = 0.8 * torch.randn((1, envs, a.action_count), device="cuda", generator=gen)
            _, status, _ = a.step(acts, wait=True)
            a_np = acts.cpu().numpy()[0]
            targets = np.zeros((envs, a.action_count), np.float32)
            fresh = []
            for e in range(envs):
                reset, _, _, _ = o.observe(e, states[e], None, None, False)
                fresh.append(reset)
                targets[e] = o.apply(states[e], a_np[e])
            qa1, va1, _ = a.state()
            for e in range(envs):
                o.complete(e, states[e], qa1[e].astype(np.float64), va1[e].astype(np.float64), int(status[0, e]))
            b.set_state(qa, va, ma)
            b.step(torch.tensor(targets[None], device="cuda"), wait=True)
            qb1, vb1, _ = b.state()
            for e in range(envs):
                if fresh[e]:
                    continue  # the tasked rollout started this step from its task's reset state
                assert _close(qb1[e], qa1[e], 1e-5) <= 1e-5, (k, e)
                assert _close(vb1[e], va1[e], 1e-4) <= 1e-4, (k, e)
                compared += 1
        assert compared >= envs * (steps - 2)


def test_policy_reads_the_actor_frames(cuda_device):
    from oracle import policy as ref

    rng = np.random.default_rng(4)
    envs, steps = 32, 4
    with nb.World("tree29", envs, substeps=4, velocity_iterations=8, control_dt=DT, seed=SEED) as w:
        prog = _program(w, noise=0.02)
        w.set_task(prog)
        nobs, na = w.observation_count, w.action_count
        layers = []
        for (n_in, n_out), act in zip(zip([nobs, 128, 64], [128, 64, na]), ["elu", "tanh", "identity"]):
            layers.append((rng.normal(0.0, 1.0 / np.sqrt(n_in), (n_out, n_in)).astype(np.float32),
                           rng.normal(0.0, 0.1, n_out).astype(np.float32), act))
        w.set_policy(layers=layers, revision=3, action_clip=1.0)
        obs, status = w.step_policy(steps)
        out = w.policy_outputs()
        tr = w.transitions(steps)
        frames = obs.cpu().numpy().astype(np.float64)
        for k in range(steps):
            want = ref.forward(frames[k], layers)
            assert float(np.max(np.abs(out["latents"][k] - want))) <= 1e-4
        assert np.all(tr["policy_revision"] == 3)
        # The advance published as a PolicyRolloutPack, read back by both readers.
        import tempfile
        from pathlib import Path

        with tempfile.TemporaryDirectory() as tmp:
            path = Path(tmp) / "batch.mrrollout"
            w.write_policy_rollout_pack(path, "task-batch", obs)
            info, params = nb.inspect_policy_rollout_pack(path)
            assert (info["environment_count"], info["control_step_count"], info["actor_observation_count"],
                    info["action_count"], info["policy_revision"], info["id"]) == (envs, steps, nobs, na, 3, "task-batch")
            assert info["task_fingerprint"] == prog.task_fingerprint and info["policy_fingerprint"] != 0
            want = np.concatenate([frames.astype(np.float32).reshape(-1), out["latents"].reshape(-1), out["log_probabilities"].reshape(-1),
                                   out["values"].reshape(-1), out["bootstrap_values"].reshape(-1)])
            np.testing.assert_array_equal(params, want)
            assert info["reward_sum"] == pytest.approx(float(tr["reward"].astype(np.float64).sum()), rel=1e-6)
            try:
                from oracle import reference_inspect_policy_rollout_pack
                ref_info, ref_params = reference_inspect_policy_rollout_pack(path, params.size)
            except FileNotFoundError:
                ref_info = None  # the reference build is absent where this runs
            if ref_info is not None:
                np.testing.assert_array_equal(ref_params, params)
                assert ref_info["transition_count"] == envs * steps


def test_critic_reads_its_own_frame(cuda_device):
    """A task with critic operators (privileged, noise-free: root height,
    linear velocity, joint velocities, command): the policy's critic values
    equal the critic network on the oracle's critic frames."""

    import torch

    from oracle import policy as ref

    rng = np.random.default_rng(6)
    envs, steps = 16, 3
    with nb.World("tree29", envs, substeps=4, velocity_iterations=8, control_dt=DT, seed=SEED) as w:
        prog = _program(w, noise=0.02)
        prog.critic = ([T.Observation(T.OBSERVE["root_height"])] +
                       [T.Observation(T.OBSERVE["root_linear_velocity_local"], 0, c) for c in range(3)] +
                       [T.Observation(T.OBSERVE["joint_velocity"], a) for a in range(w.action_count)] +
                       [T.Observation(T.OBSERVE["command"], 0, c) for c in range(3)])
        w.set_task(prog)
        nobs, ncrit, na = w.observation_count, len(prog.critic), w.action_count
        assert int(w.layout().critic_observation_count) == ncrit
        dense = lambda sizes, acts: [(rng.normal(0.0, 1.0 / np.sqrt(a), (b, a)).astype(np.float32),  # noqa: E731
                                      rng.normal(0.0, 0.1, b).astype(np.float32), f) for (a, b), f in zip(zip(sizes[:-1], sizes[1:]), acts)]
        critic = dense([ncrit, 32, 1], ["tanh", "identity"])
        w.set_policy(layers=dense([nobs, 64, na], ["elu", "identity"]), critic_layers=critic, revision=5, action_clip=1.0)
        o = _oracle(w, prog)
        states = [o.new_state() for _ in range(envs)]
        for k in range(steps):
            obs, status = w.step_policy(1)
            out = w.policy_outputs()
            q, v, _ = w.state()
            tr = w.transitions(1)
            for e in range(envs):
                o.observe(e, states[e], None, None, False)
                want = ref.forward(states[e].critic[None], critic)[0, 0]
                assert abs(float(out["values"][0, e]) - want) <= 1e-4, (k, e)
                o.apply(states[e], out["latents"][0, e].clip(-1.0, 1.0))
                o.complete(e, states[e], q[e].astype(np.float64), v[e].astype(np.float64), int(status[0, e]))
        del tr


def test_installer_refuses_programs_outside_the_subset(cuda_device):
    with nb.World("tree29", 4, seed=SEED) as w:
        base = _program(w)
        bad = [
            dict(actions=base.actions[:-1]),
            dict(actor=base.actor + [T.Observation(16)]),
            dict(actor=base.actor + [T.Observation(T.OBSERVE["joint_velocity"], source=99)]),
            dict(actor=base.actor + [T.Observation(T.OBSERVE["delayed_action"], source=0, component=5)]),
            dict(rewards=base.rewards + [T.Reward(11, -1.0)]),
            dict(rewards=base.rewards + [T.Reward(T.REWARD["joint_group_posture_squared"], -1.0, group=7)]),
            dict(terminations=[T.Termination(2, 3, 1, 0.5)]),
            dict(randomization=[T.Randomization(4)]),
            dict(action_history=2),
            dict(rewards=base.rewards + [T.Reward(T.REWARD["support_slip"], -1.0, group=0)]),  # no contact groups
            dict(contact_groups=[T.ContactGroup([99], T.CONTACT_SUPPORT, 0)]),
            dict(terminations=[T.Termination(T.TERMINATE["contact_group"], 3, 1, 0.5, group=0)]),
            dict(default_q=base.default_q[:-1]),
        ]
        for change in bad:
            prog = T.TaskProgram(**{**base.__dict__, **change})
            with pytest.raises(MetalRoboError, match="task program"):
                w.set_task(prog)
        w.set_task(base)
        assert w.observation_count == len(base.actor)
        w.clear_task()
        assert w.observation_count == w.nq + w.nv
        import torch

        obs, status, _ = w.step(torch.zeros((1, 4, w.action_count), device="cuda"), wait=True)
        q, v, _ = w.state()
        np.testing.assert_array_equal(obs.cpu().numpy()[0], np.concatenate([q, v], axis=1))


def test_reseed_starts_new_episodes_under_the_new_draws(cuda_device):
    """mr_task_rollout_reset with a new seed: every environment starts a new
    episode at the next step, its reset draws and commands keyed on the new
    seed (the first frame equals a fresh oracle's under that seed)."""

    import torch

    envs = 8
    with nb.World("tree29", envs, substeps=4, velocity_iterations=8, control_dt=DT, seed=SEED) as w:
        prog = _program(w, noise=0.03)
        w.set_task(prog)
        zeros = torch.zeros((1, envs, w.action_count), device="cuda")
        for _ in range(3):
            w.step(zeros, wait=True)
        w.reset(seed=11)
        obs, _, _ = w.step(zeros, wait=True)
        o = _oracle(w, prog)
        assert o.seed == 11
        for e in range(envs):
            st = o.new_state()
            reset, _, _, want = o.observe(e, st, None, None, False)
            assert reset
            assert _close(obs.cpu().numpy()[0, e], want, OBS_TOL) <= OBS_TOL, e
