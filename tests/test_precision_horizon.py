"""Horizon drift of the precision modes against the FP64 oracle.

The 29-DoF contact world is chaotic: any perturbation -- FP32 rounding
included -- grows over the horizon, so per-step parity (test_gpu_parity)
is the accuracy gate and this test reports how fast each precision mode
leaves the FP64 trajectory when both start from the same FP32 state and see
the same actions.  It also checks that every impulse the device publishes
satisfies its friction cone.
"""

from __future__ import annotations

import numpy as np
import pytest

import numi_lab_b200 as nb
from oracle import Oracle

pytestmark = pytest.mark.gpu

CHECKPOINTS = (1, 5, 10, 25, 50, 100)


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(1.0, float(np.max(np.abs(b)))))


def _cone_violation(manifolds, mu):
    worst = 0.0
    for env, m_env in enumerate(manifolds):
        for m in m_env:
            for i in range(m.count):
                n, t, b = m.points[i].impulses
                scale = max(1.0, abs(n))
                if n < 0.0:
                    worst = max(worst, -n / scale)
                lim = mu[env] * max(n, 0.0)
                tang = float(np.hypot(t, b))
                worst = max(worst, (tang - lim) / scale)
    return worst


def test_horizon_drift_and_cone_feasibility(cuda_device):
    import torch

    envs, steps, seed = 8, max(CHECKPOINTS), 5
    gen = torch.Generator(device="cuda").manual_seed(3)
    actions = 0.3 * torch.randn((steps, envs, 29), device="cuda", generator=gen)
    acts = actions.cpu().numpy()
    report = {}
    oracle_q = None
    for precision in ("fp32", "fp64-inertia", "compensated"):
        with nb.World("tree29", envs, substeps=4, velocity_iterations=8, control_dt=0.02, seed=seed,
                      precision=precision) as world:
            if oracle_q is None:
                # FP64 reference trajectory from the same FP32 start state.
                oracle = Oracle(world.model(), 0.005, 4, 8, 0)
                q0, v0, m0 = world.state()
                fr = world.friction_scales()
                qs = [q0[e].astype(np.float64) for e in range(envs)]
                vs = [v0[e].astype(np.float64) for e in range(envs)]
                mans = [oracle.env_manifolds(m0, e) for e in range(envs)]
                oracle_q = {}
                for k in range(steps):
                    for e in range(envs):
                        st, _ = oracle.control_step(qs[e], vs[e], mans[e], acts[k, e], float(fr[e]))
                        assert st == 0
                    if k + 1 in CHECKPOINTS:
                        oracle_q[k + 1] = [q.copy() for q in qs]
            drift = {}
            cone = 0.0
            mu = world.friction_scales()
            for k in range(steps):
                _, status, _ = world.step(actions[k:k + 1], wait=True)
                assert int(status.abs().sum()) == 0
                q, _, m = world.state()
                per_env = [[m[e * world.pair_count + p] for p in range(world.pair_count)] for e in range(envs)]
                cone = max(cone, _cone_violation(per_env, mu))
                if k + 1 in CHECKPOINTS:
                    d = [_rel(q[e], oracle_q[k + 1][e]) for e in range(envs)]
                    drift[k + 1] = (float(np.median(d)), float(np.max(d)))
            report[precision] = {"drift_median_max": drift, "cone_violation": cone}
    for precision, r in report.items():
        print(f"{precision}: cone violation {r['cone_violation']:.2e}")
        for k, (med, mx) in r["drift_median_max"].items():
            print(f"  after {k:4d} control steps: q deviation from FP64 median {med:.2e} max {mx:.2e}")
    for r in report.values():
        # Published impulses satisfy the elliptic cone to FP32 rounding.
        assert r["cone_violation"] <= 1e-6
        # One control step stays at FP32-rounding level of the state.
        assert r["drift_median_max"][1][0] <= 1e-5
