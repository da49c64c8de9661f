"""Per-step parity on the contact benchmark's own configuration: 4096
environments of the 29-DoF floating tree (model and reset seed 2026, 20 ms
control = 4 x 5 ms microsteps, 8 temporalCone iterations, PD targets
~ N(0, 0.3)).  A seeded sample of 256 environments is replayed by the FP64
oracle for 25 control steps, each from the device's FP32 state at the start
of the step.

Every env-step is held to the per-step bound of tests/_sensitivity.py:
max(1e-5, K x the spread of the oracle's Monte Carlo FP32-rounding runs)
for q and qd and max(1e-4, K x that spread) for impulses.  Status codes and
manifold feature ids / lifetimes must be identical.  Only on env-steps
where the oracle took a decision within its band of a threshold, or where
rounding flipped a decision in one of its noisy runs, may the device differ
(band steps: counted, at most 5 %).
The test reports the fraction of env-steps that meet the plain 1e-5 / 1e-4
tolerances."""

from __future__ import annotations

import numpy as np
import pytest

import numi_lab_b200 as nb

import _sensitivity as S

pytestmark = pytest.mark.gpu

ENVS, SEED, SAMPLE, STEPS, WARM = 4096, 2026, 256, 25, 5
Q_TOL, V_TOL, IMP_TOL = 1e-5, 1e-5, 1e-4


def _gpu_impulses(manifolds, env: int, pairs: int):
    imps, feats = [], []
    for p in range(pairs):
        m = manifolds[env * pairs + p]
        feats.append((int(m.count), tuple((int(m.points[i].feature_a), int(m.points[i].feature_b), int(m.points[i].life))
                                          for i in range(m.count))))
        for i in range(m.count):
            imps.append(list(m.points[i].impulses))
    return np.array(imps, np.float64).reshape(-1, 3), tuple(feats)


def test_tree29_bench_configuration_per_step(cuda_device):
    import torch

    rng = np.random.default_rng(SEED)
    sample = np.sort(rng.choice(ENVS, SAMPLE, replace=False))
    stats = {"env_steps": 0, "band": 0, "plain_q": 0, "plain_v": 0, "plain_imp": 0, "imp_steps": 0, "contacts": 0}
    worst = {"q": 0.0, "v": 0.0, "imp": 0.0}
    failures = []
    with nb.World("tree29", ENVS, substeps=4, velocity_iterations=8, control_dt=0.02, seed=SEED) as world, S.pool() as ex:
        fr = world.friction_scales()
        pairs = world.pair_count
        gen = torch.Generator(device="cuda").manual_seed(SEED)
        _, status, _ = world.step(0.3 * torch.randn((WARM, ENVS, world.action_count), device="cuda", generator=gen), wait=True)
        assert int(status.abs().sum()) == 0
        for k in range(STEPS):
            q0, v0, m0 = world.state()
            actions = 0.3 * torch.randn((1, ENVS, world.action_count), device="cuda", generator=gen)
            _, status, _ = world.step(actions, wait=True)
            st = status.cpu().numpy()[0]
            q1, v1, m1 = world.state()
            acts = actions.cpu().numpy()[0].astype(np.float64)
            jobs = [{"source": "tree29", "seed": SEED, "h": 0.005, "substeps": 4, "iters": 8, "q": q0[e], "v": v0[e],
                     "manifolds": S.manifold_bytes(m0, int(e), pairs), "actions": acts[e], "friction": float(fr[e]),
                     "rng": int(SEED * 100003 + k * ENVS + e)} for e in sample]
            for e, res in zip(sample, ex.map(S.tree_env_step, jobs, chunksize=8)):
                stats["env_steps"] += 1
                assert int(st[e]) == res["status"] == 0, (k, e, int(st[e]), res["status"])
                imp, feats = _gpu_impulses(m1, int(e), pairs)
                same = feats == res["features"]
                dq, dv = S.rel_err(q1[e], res["q"]), S.rel_err(v1[e], res["v"])
                di = (float(np.max(np.abs(imp - res["imp"]))) / max(1.0, float(np.max(np.abs(res["imp"]))))
                      if same and imp.size else 0.0)
                verdict, misses = S.judge(res, same, {"q": dq, "v": dv, "imp": di})
                if verdict == "band":
                    stats["band"] += 1
                    continue
                if verdict == "fail":
                    failures.append((k, int(e), misses))
                    continue
                stats["contacts"] += res["contacts"]
                for name, err in (("q", dq), ("v", dv), ("imp", di)):
                    worst[name] = max(worst[name], err / S.bounded(err, res["sens"][name], S.BASES[name], res["k"])[1])
                stats["plain_q"] += dq <= Q_TOL
                stats["plain_v"] += dv <= V_TOL
                if imp.size:
                    stats["imp_steps"] += 1
                    stats["plain_imp"] += di <= IMP_TOL
    clean = stats["env_steps"] - stats["band"]
    print(f"tree29 bench config: {stats['env_steps']} env-steps, {stats['band']} band; plain-tolerance fractions "
          f"q {stats['plain_q'] / clean:.4f} qd {stats['plain_v'] / clean:.4f} impulses {stats['plain_imp'] / max(1, stats['imp_steps']):.4f}; "
          f"worst error / bound {worst}; contacts {stats['contacts']}")
    assert not failures, failures[:10]
    assert stats["contacts"] > 0
    assert stats["band"] <= stats["env_steps"] // 20
