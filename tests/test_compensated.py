"""Compensated precision (MR_PRECISION_COMPENSATED): FP64 articulated
inertia plus Kahan-compensated FP32 sums for the position integration and
the cone solve's impulse accumulation.

Per-step parity of the mode against the FP64 oracle runs with the other
modes in test_gpu_parity.py and test_scene_parity.py.  This file checks
what the compensation is for and how its state behaves:

* on a contact-free 7-DoF chain (5 ms steps, PD targets N(0, 0.5)) the
  position sums' rounding dominates the short-horizon error of the FP64
  articulated-inertia mode, and the compensated sums cut the median q
  deviation from the FP64 oracle after 10 and 25 control steps to well
  under the uncompensated mode's (measured ~0.4x; gated at 0.7x);
* the compensation terms belong to the resident state: set_state clears
  them, so a world given a state continues exactly like a fresh world given
  the same state, while a world that keeps its terms ends elsewhere in the
  last bits.
"""

from __future__ import annotations

import numpy as np
import pytest

import numi_lab_b200 as nb
from oracle import Oracle

pytestmark = pytest.mark.gpu

CHECKPOINTS = (10, 25)
GAIN = 0.7  # compensated median drift <= GAIN x the uncompensated mode's


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(1.0, float(np.max(np.abs(b)))))


def test_compensated_sums_reduce_chain_drift(cuda_device):
    import torch

    envs, dt = 64, 0.005
    steps = max(CHECKPOINTS)
    gen = torch.Generator(device="cuda").manual_seed(5)
    with nb.World("chain7", envs, substeps=1, control_dt=dt, seed=3) as world:
        actions = 0.5 * torch.randn((steps, envs, world.action_count), device="cuda", generator=gen)
        q0, v0, _ = world.state()
        oracle = Oracle(world.model(), dt, 1, 0, 0)
    acts = actions.cpu().numpy().astype(np.float64)
    qs = [q0[e].astype(np.float64) for e in range(envs)]
    vs = [v0[e].astype(np.float64) for e in range(envs)]
    reference = {}
    for k in range(steps):
        for e in range(envs):
            st, _ = oracle.control_step(qs[e], vs[e], None, acts[k, e], 1.0)
            assert st == 0
        if k + 1 in CHECKPOINTS:
            reference[k + 1] = [q.copy() for q in qs]
    drift = {}
    for precision in ("fp64-inertia", "compensated"):
        with nb.World("chain7", envs, substeps=1, control_dt=dt, seed=3, precision=precision) as world:
            done = 0
            for cp in CHECKPOINTS:
                _, status, _ = world.step(actions[done:cp].contiguous(), wait=True)
                assert int(status.abs().sum()) == 0
                done = cp
                q, _, _ = world.state()
                drift[(precision, cp)] = float(np.median([_rel(q[e], reference[cp][e]) for e in range(envs)]))
    print({f"{p} @{k}": f"{d:.2e}" for (p, k), d in drift.items()})
    for cp in CHECKPOINTS:
        assert drift[("compensated", cp)] <= GAIN * drift[("fp64-inertia", cp)], drift


def test_set_state_clears_the_compensation_terms(cuda_device):
    import torch

    envs = 16
    gen = torch.Generator(device="cuda").manual_seed(1)
    actions = 0.3 * torch.randn((20, envs, 29), device="cuda", generator=gen)

    def world():
        return nb.World("tree29", envs, substeps=4, velocity_iterations=8, control_dt=0.02, seed=5, precision="compensated")

    with world() as a, world() as b, world() as c:
        a.step(actions[:10].contiguous(), wait=True)
        state = a.state()
        a.set_state(*state)
        b.set_state(*state)
        c.step(actions[:10].contiguous(), wait=True)  # same trajectory as a, terms kept
        for w in (a, b, c):
            _, status, _ = w.step(actions[10:].contiguous(), wait=True)
            assert int(status.abs().sum()) == 0
        qa, va, _ = a.state()
        qb, vb, _ = b.state()
        qc, _, _ = c.state()
        assert np.array_equal(qa, qb) and np.array_equal(va, vb)
        assert int((qc != qa).sum()) > 0
