"""CUDA microstep vs the oracle, one control step at a time from identical
FP32 input state (the CUDA path runs through the C ABI).

Tolerances, per control step, relative to max(1, |x|) of the oracle state:

* chain7 (no contact): q within 1e-5; qd within 1e-5 with FP64
  articulated inertias and 5e-5 in the all-FP32 mode (see CHAIN_V_TOL).
* tree29 (contact): every env-step within max(1e-5, K x sensitivity) for
  q and qd and max(1e-4, K x sensitivity) for impulses, where the
  sensitivity is the FP64 oracle's own response to rounding its FP32 inputs
  (tests/_sensitivity.py): contact targets divide FP32 positions by the
  substep (-sep / h), so some steps amplify input rounding and the bound
  follows that step's amplification, not a blanket loosening.
* Discrete decisions (contact sets, manifold feature ids, status codes,
  rollback) identical, except decisions the oracle took within its band of
  a threshold.
"""

from __future__ import annotations

import numpy as np
import pytest

import numi_lab_b200 as nb
from oracle import Oracle

pytestmark = pytest.mark.gpu

Q_TOL = 1e-5
V_TOL = 1e-5
IMPULSE_TOL = 1e-4


def _rel_err(a: np.ndarray, b: np.ndarray) -> float:
    """Largest per-step deviation relative to the state vector's scale."""

    return float(np.max(np.abs(a - b)) / max(1.0, float(np.max(np.abs(b)))))


def _manifold_features(manifolds, env: int, pairs: int) -> list[tuple[int, tuple[int, ...]]]:
    out = []
    for p in range(pairs):
        m = manifolds[env * pairs + p]
        out.append((int(m.count), tuple(int(m.points[i].feature_a) for i in range(m.count))))
    return out


def _oracle_features(man, pairs: int) -> list[tuple[int, tuple[int, ...]]]:
    return [(int(man[p].count), tuple(int(man[p].points[i].feature_a) for i in range(man[p].count))) for p in range(pairs)]


# FP32 articulated inertia: rounding the shifted child inertias to FP32
# alone moves the FP64 oracle's joint velocities by up to ~3e-5 relative on
# this chain (parallel-axis terms dwarf the distal pivots), so the FP32 mode
# is held to 5e-5 and the FP64 articulated-inertia modes to 1e-5.
CHAIN_V_TOL = {"fp32": 5e-5, "fp64-inertia": 1e-5, "compensated": 1e-5}


@pytest.mark.parametrize("precision", ["fp32", "fp64-inertia", "compensated"])
def test_chain7_free_motion_per_step(cuda_device, precision):
    import torch

    envs, steps, dt = 64, 25, 0.005
    with nb.World("chain7", envs, substeps=1, control_dt=dt, seed=3, precision=precision) as world:
        oracle = Oracle(world.model(), dt, 1, 0, 0)
        gen = torch.Generator(device="cuda").manual_seed(11)
        worst_q = worst_v = 0.0
        for k in range(steps):
            q0, v0, _ = world.state()
            actions = 5.0 * torch.randn((1, envs, world.action_count), device="cuda", generator=gen)
            _, status, _ = world.step(actions, wait=True)
            assert int(status.abs().sum()) == 0
            q1, v1, _ = world.state()
            acts = actions.cpu().numpy()[0]
            for e in range(envs):
                q = q0[e].astype(np.float64)
                v = v0[e].astype(np.float64)
                st, _ = oracle.control_step(q, v, None, acts[e], 1.0)
                assert st == 0
                worst_q = max(worst_q, _rel_err(q1[e], q))
                worst_v = max(worst_v, _rel_err(v1[e], v))
        print(f"chain7 {precision}: worst q {worst_q:.2e} qd {worst_v:.2e}")
        assert worst_q <= Q_TOL, worst_q
        assert worst_v <= CHAIN_V_TOL[precision], worst_v


def _tree_world(envs: int, seed: int = 5, precision: str = "fp32"):
    return nb.World("tree29", envs, substeps=4, velocity_iterations=8, final_velocity_iterations=0, control_dt=0.02, seed=seed,
                    precision=precision)


@pytest.mark.parametrize("precision", ["fp32", "fp64-inertia", "compensated"])
def test_tree29_contact_per_step(cuda_device, precision):
    """Per control step from identical FP32 state, every env-step held to
    max(base, K x the spread of the oracle's Monte Carlo FP32-rounding runs)
    (tests/_sensitivity.py): q and qd base 1e-5, impulses 1e-4."""

    import torch

    import _sensitivity as S

    envs, warm, steps, seed = 32, 20, 12, 5
    with _tree_world(envs, seed=seed, precision=precision) as world, S.pool() as ex:
        friction = world.friction_scales()
        pairs = world.pair_count
        gen = torch.Generator(device="cuda").manual_seed(21)
        warm_actions = 0.3 * torch.randn((warm, envs, world.action_count), device="cuda", generator=gen)
        _, status, _ = world.step(warm_actions, wait=True)
        assert int(status.abs().sum()) == 0
        failures, band_cases, contacts_seen, plain = [], 0, 0, 0
        for k in range(steps):
            q0, v0, m0 = world.state()
            actions = 0.3 * torch.randn((1, envs, world.action_count), device="cuda", generator=gen)
            _, status, _ = world.step(actions, wait=True)
            assert int(status.abs().sum()) == 0
            q1, v1, m1 = world.state()
            acts = actions.cpu().numpy()[0].astype(np.float64)
            jobs = [{"source": "tree29", "seed": seed, "h": 0.005, "substeps": 4, "iters": 8, "q": q0[e], "v": v0[e],
                     "manifolds": S.manifold_bytes(m0, e, pairs), "actions": acts[e], "friction": float(friction[e]),
                     "rng": 1000 * k + e} for e in range(envs)]
            for e, res in enumerate(ex.map(S.tree_env_step, jobs, chunksize=4)):
                assert res["status"] == 0
                imps, feats = [], []
                for p in range(pairs):
                    gm = m1[e * pairs + p]
                    feats.append((int(gm.count), tuple((int(gm.points[i].feature_a), int(gm.points[i].feature_b),
                                                        int(gm.points[i].life)) for i in range(gm.count))))
                    imps += [list(gm.points[i].impulses) for i in range(gm.count)]
                imp = np.array(imps, np.float64).reshape(-1, 3)
                same = tuple(feats) == res["features"]
                dq, dv = _rel_err(q1[e], res["q"]), _rel_err(v1[e], res["v"])
                di = (float(np.max(np.abs(imp - res["imp"]))) / max(1.0, float(np.max(np.abs(res["imp"]))))
                      if same and imp.size else 0.0)
                verdict, misses = S.judge(res, same, {"q": dq, "v": dv, "imp": di})
                if verdict == "band":
                    band_cases += 1
                    continue
                if verdict == "fail":
                    failures.append((k, e, misses))
                    continue
                contacts_seen += res["contacts"]
                plain += dq <= Q_TOL and dv <= V_TOL and di <= IMPULSE_TOL
        clean = envs * steps - band_cases
        print(f"tree29 {precision}: {plain}/{clean} clean env-steps within the plain tolerances, {band_cases} band cases")
        assert not failures, failures[:10]
        assert contacts_seen > 0, "the workload should produce contacts"
        assert band_cases <= envs * steps // 20, f"{band_cases} band cases"


def test_invalid_quaternion_rolls_back_only_that_env(cuda_device):
    import torch

    envs = 8
    with _tree_world(envs, seed=9) as world:
        q0, v0, m0 = world.state()
        bad = q0.copy()
        bad[3, 3:7] = [0.0, 0.0, 0.0, 2.0]  # norm 2: rejected quaternion
        world.set_state(bad, v0, m0)
        actions = torch.zeros((1, envs, world.action_count), device="cuda")
        _, status, _ = world.step(actions, wait=True)
        codes = status.cpu().numpy()[0]
        assert codes[3] == 2  # MR_STEP_NONFINITE_INPUT
        assert np.all(np.delete(codes, 3) == 0)
        q1, v1, _ = world.state()
        np.testing.assert_array_equal(q1[3], bad[3])  # transactional: checkpoint kept
        np.testing.assert_array_equal(v1[3], v0[3])
    with _tree_world(envs, seed=9) as clean:
        clean.set_state(q0, v0, m0)
        _, status, _ = clean.step(torch.zeros((1, envs, clean.action_count), device="cuda"), wait=True)
        q2, v2, _ = clean.state()
        keep = [e for e in range(envs) if e != 3]
        np.testing.assert_array_equal(q1[keep], q2[keep])  # isolation: other envs unaffected
        np.testing.assert_array_equal(v1[keep], v2[keep])


def test_reset_mask_restores_reset_state(cuda_device):
    import torch

    envs = 6
    with _tree_world(envs, seed=2) as world:
        q_reset, v_reset, _ = world.state()
        actions = 0.3 * torch.randn((5, envs, world.action_count), device="cuda")
        world.step(actions, wait=True)
        mask = torch.zeros((1, envs), dtype=torch.int32, device="cuda")
        mask[0, 4] = 1
        zero = torch.zeros((1, envs, world.action_count), device="cuda")
        world.step(zero, reset_mask=mask, wait=True)
        q1, _, _ = world.state()
    with _tree_world(envs, seed=2) as ref:
        ref.step(zero, wait=True)  # from the reset state, one step
        q2, _, _ = ref.state()
    np.testing.assert_array_equal(q1[4], q2[4])


def test_bitwise_replay_and_host_path(cuda_device):
    import torch

    envs, steps = 16, 6
    actions = 0.3 * torch.randn((steps, envs, 29), device="cuda", generator=torch.Generator(device="cuda").manual_seed(4))
    results = []
    for _ in range(2):
        with _tree_world(envs, seed=12) as world:
            obs, status, _ = world.step(actions, wait=True)
            results.append((obs.cpu().numpy(), world.state()[0]))
    np.testing.assert_array_equal(results[0][0], results[1][0])
    np.testing.assert_array_equal(results[0][1], results[1][1])
    with _tree_world(envs, seed=12) as world:
        world.set_state_readback(True)
        out = world.advance_host(actions.cpu().numpy())
        assert out["counters"].successful_environment_steps == steps * envs
        np.testing.assert_array_equal(out["observations"], results[0][0])
        np.testing.assert_array_equal(out["final_q"], results[0][1])
    # The host path again in uneven pieces (each advance its own captured
    # graph with per-step observation read-back on the copy stream), read
    # through views of the rollout's result memory.
    with _tree_world(envs, seed=12) as world:
        world.set_state_readback(True)
        host = actions.cpu().numpy()
        done = 0
        for n in (1, 3, 2):
            out = world.advance_host(host[done:done + n], copy=False)
            np.testing.assert_array_equal(out["observations"], results[0][0][done:done + n])
            done += n
        np.testing.assert_array_equal(out["final_q"], results[0][1])


def test_environment_chains_are_bitwise_equal_and_report_absolute_slots(cuda_device, monkeypatch):
    """An advance run as several environment chains (contiguous blocks on
    their own streams inside the graph) equals the single chain bit for bit,
    also for an uneven split, and counters name the absolute slot."""
    import torch

    envs, steps = 50, 4
    actions = 0.3 * torch.randn((steps, envs, 29), device="cuda", generator=torch.Generator(device="cuda").manual_seed(9))
    results = {}
    for chains in ("1", "3"):
        monkeypatch.setenv("NUMI_B200_CHAINS", chains)
        with _tree_world(envs, seed=21) as world:
            q0, v0, m0 = world.state()
            bad = q0.copy()
            bad[37, 3:7] = [0.0, 0.0, 0.0, 2.0]  # rejected quaternion in the third block
            world.set_state(bad, v0, m0)
            obs, status, counters = world.step(actions, wait=True)
            results[chains] = (obs.cpu().numpy(), status.cpu().numpy(), world.state()[0], counters.first_failing_environment)
    a, b = results["1"], results["3"]
    for x, y in zip(a[:3], b[:3]):
        np.testing.assert_array_equal(x, y)
    assert a[3] == b[3] == 37


def test_chain7_literal_configuration_latches_with_the_oracle(cuda_device):
    """The plain-ABA configuration as stated (tau ~ N(0, 5) N m, 5 ms steps,
    no episodes): the chain gains energy until its velocities overflow.
    From the device's FP32 state at the start of every control step, the
    FP64 oracle must take the same rollback decision -- the same status
    code on the same step -- as the device (the oracle latches when FP32
    arithmetic would overflow; magnitudes within 1e6 of FLT_MAX are band
    decisions, which may go either way).  A latched environment keeps its
    checkpoint: its state does not change."""

    import torch

    envs, steps, dt = 128, 400, 0.005
    with nb.World("chain7", envs, substeps=1, control_dt=dt, seed=2026) as world:
        oracle = Oracle(world.model(), dt, 1, 0, 0)
        gen = torch.Generator(device="cuda").manual_seed(2026)
        decided = {"fail": 0, "ok": 0, "band": 0}
        first_failure = {}
        for k in range(steps):
            q0, v0, _ = world.state()
            actions = 5.0 * torch.randn((1, envs, world.action_count), device="cuda", generator=gen)
            _, status, _ = world.step(actions, wait=True)
            st = status.cpu().numpy()[0]
            q1, v1, _ = world.state()
            acts = actions.cpu().numpy()[0]
            for e in range(envs):
                q = q0[e].astype(np.float64)
                v = v0[e].astype(np.float64)
                ost, trace = oracle.control_step(q, v, None, acts[e], 1.0)
                if int(st[e]) != ost:
                    assert trace.band_decisions > 0, (k, e, int(st[e]), ost)
                    decided["band"] += 1
                    continue
                decided["fail" if ost else "ok"] += 1
                if ost:
                    first_failure.setdefault(e, k)
                    np.testing.assert_array_equal(q1[e], q0[e])  # rolled back: the checkpoint stays
                    np.testing.assert_array_equal(v1[e], v0[e])
        print(f"chain7 tau ~ N(0, 5): {decided}; first latch steps {sorted(first_failure.values())[:5]}...")
        assert len(first_failure) > envs // 2  # the literal configuration does blow up within the horizon
        assert decided["band"] <= envs * steps // 100  # a latched checkpoint within 1e6 of FLT_MAX stays a band case
