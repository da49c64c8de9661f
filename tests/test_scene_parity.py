"""Free-body piles: CUDA control step vs the oracle, one control step at a
time from identical FP32 input state (the CUDA path runs through the C ABI).

Each environment is a pile of 8-64 boxes and spheres dropped onto a plane.
The oracle restates the device stage order in FP64 (oracle/oracle.c).
Discrete decisions -- manifold pair keys, point features and lifetimes,
status codes -- must agree exactly, except at steps where the oracle took a
decision within its band of a threshold (5e-5 for piles: within a control
step the device trajectory departs from the oracle's by up to ~5e-6 in
position, and later substeps decide on the departed state).  Continuous state is compared
relative to max(1, |x|) of the oracle state: q within 1e-5 at every clean
env-step; body velocities within 2e-5 at the median and 1e-3 at the worst
clean env-step; impulses within 1e-4 at the median and 1e-2 at the worst.
The velocity bounds are set by FP32 conditioning: the FP64 oracle's own
response to a perturbation of its inputs by eight FP32 roundings is ~5e-6 at
the median (tests/test_conditioning.py), and contact stacks compound it.
"""

from __future__ import annotations

import numpy as np
import pytest

import numi_lab_b200 as nb
from oracle import SceneOracle

pytestmark = pytest.mark.gpu

# Per control step tolerances (relative to max(1, |x|)).
Q_TOL = 1e-5
V_MEDIAN_TOL = 2e-5
V_WORST_TOL = 1e-3
IMPULSE_MEDIAN_TOL = 1e-4
IMPULSE_WORST_TOL = 1e-2


def _counts(table: np.ndarray) -> list[int]:
    out = []
    for e in range(table.shape[0]):
        c = 0
        while c < table.shape[1] and int(table[e, c, 7].view(np.uint32)) != 0:
            c += 1
        out.append(c)
    return out


def _keys(table: np.ndarray, env: int, count: int) -> list[int]:
    return [int(table[env, i, 56].view(np.uint32)) for i in range(count)]


def _compare_run(seed: int, envs: int, steps: int, precision: str = "fp32", source: str = "pile"):
    import torch

    substeps, iters = 4, 8
    rows = []
    with nb.World(source, envs, substeps=substeps, velocity_iterations=iters, control_dt=0.02, seed=seed,
                  precision=precision) as world:
        oracle = SceneOracle(world.model(), 0.02 / substeps, substeps, iters, 0)
        fr = world.friction_scales()
        acts = torch.zeros((1, envs, 0), device="cuda")
        for _ in range(steps):
            q0, v0, t0 = world.state()
            c0 = _counts(t0)
            _, status, _ = world.step(acts, wait=True)
            st = status.cpu().numpy()[0]
            q1, v1, t1 = world.state()
            c1 = _counts(t1)
            for e in range(envs):
                q = q0[e].astype(np.float64)
                v = v0[e].astype(np.float64)
                table = oracle.table_from_device(t0[e], c0[e])
                ost, trace = oracle.step(q, v, table, float(fr[e]))
                row = {
                    "status": (int(st[e]), ost),
                    "band": int(trace.band_decisions),
                    "dq": float(np.max(np.abs(q1[e] - q)) / max(1.0, float(np.max(np.abs(q))))),
                    "dv": float(np.max(np.abs(v1[e] - v)) / max(1.0, float(np.max(np.abs(v))))),
                    "keys": (_keys(t1, e, c1[e]), table.keys()),
                    "features_equal": True,
                    "dimp": 0.0,
                    "contacts": int(trace.contact_count),
                }
                if row["keys"][0] == row["keys"][1]:
                    dev = oracle.table_from_device(t1[e], c1[e])
                    for i in range(c1[e]):
                        md, mo = dev.slots[i].m, table.slots[i].m
                        if md.count != mo.count:
                            row["features_equal"] = False
                            break
                        for p in range(md.count):
                            pd, po = md.points[p], mo.points[p]
                            if (pd.feature_a, pd.feature_b, pd.life) != (po.feature_a, po.feature_b, po.life):
                                row["features_equal"] = False
                            scale = max(1.0, abs(po.impulses[0]))
                            row["dimp"] = max(row["dimp"], max(abs(pd.impulses[j] - po.impulses[j]) for j in range(3)) / scale)
                rows.append(row)
    return rows


@pytest.mark.parametrize("seed,precision", [(3, "fp32"), (10, "fp32"), (13, "fp32"), (1, "fp32"),  # 10, 8, 17, 50 bodies
                                            (13, "compensated"), (1, "compensated")])
def test_pile_control_steps_match_oracle(cuda_device, seed, precision):
    rows = _compare_run(seed, 8, 60, precision)
    assert all(r["status"][0] == r["status"][1] == 0 for r in rows)
    clean = [r for r in rows if r["band"] == 0]
    assert len(clean) >= len(rows) // 2, "too many band steps for a meaningful comparison"
    assert max(r["contacts"] for r in rows) > 0
    for r in clean:
        assert r["keys"][0] == r["keys"][1]
        assert r["features_equal"]
        assert r["dq"] <= Q_TOL
        assert r["dv"] <= V_WORST_TOL
        assert r["dimp"] <= IMPULSE_WORST_TOL
    assert float(np.median([r["dv"] for r in clean])) <= V_MEDIAN_TOL
    assert float(np.median([r["dimp"] for r in clean])) <= IMPULSE_MEDIAN_TOL


def test_pile_failed_step_keeps_state_and_reset_restores(cuda_device):
    import torch

    envs = 4
    with nb.World("pile", envs, seed=7) as world:
        acts = torch.zeros((1, envs, 0), device="cuda")
        for _ in range(3):
            world.step(acts, wait=True)
        q, v, t = world.state()
        bad = q.copy()
        bad[1, 3:7] = np.nan  # non-finite orientation of env 1's first body
        world.set_state(bad, v, t)
        _, status, _ = world.step(acts, wait=True)
        st = status.cpu().numpy()[0]
        assert st[1] == 2  # MR_STEP_NONFINITE_INPUT
        assert st[0] == st[2] == st[3] == 0
        q2, v2, t2 = world.state()
        np.testing.assert_array_equal(np.isnan(q2[1]), np.isnan(bad[1]))
        np.testing.assert_array_equal(v2[1], v[1])
        # A reset of env 1 publishes its reset state stepped once.
        rq, rv, _ = nb.sample_reset("pile", 7, 7, 0, envs)
        mask = torch.tensor([[0, 1, 0, 0]], dtype=torch.int32, device="cuda")
        _, status, _ = world.step(acts, reset_mask=mask, wait=True)
        assert int(status.cpu().numpy()[0][1]) == 0
        q3, v3, t3 = world.state()
        oracle = SceneOracle(world.model(), 0.005, 4, 8, 0)
        qo, vo = rq[1].astype(np.float64), rv[1].astype(np.float64)
        from oracle import SceneTable

        table = SceneTable()
        ost, _ = oracle.step(qo, vo, table, float(world.friction_scales()[1]))
        assert ost == 0
        assert np.max(np.abs(q3[1] - qo)) <= Q_TOL * max(1.0, np.max(np.abs(qo)))


@pytest.mark.parametrize("seed", [3, 11, 5])  # 10, 25 and 49 bodies, one quarter cylinders
def test_cylinder_pile_control_steps_match_oracle(cuda_device, seed):
    """Piles with cylinders: the support-mapped narrowphase (GJK, EPA, MPR,
    the cylinder patch) and cylinder-on-plane contacts on the device against
    the oracle's FP64 restatement, under the pile tolerances.  A support
    point or witness feature picked within rounding of a tie (a box face
    across the normal, near-equal barycentric weights) is a band decision."""
    rows = _compare_run(seed, 8, 60, "fp32", "cylinder_pile")
    assert all(r["status"][0] == r["status"][1] == 0 for r in rows)
    clean = [r for r in rows if r["band"] == 0]
    print(f"cylinder pile seed {seed}: {len(clean)} clean of {len(rows)} env-steps")
    # Resting contact of a box face on a cylinder picks the box's support
    # vertex by the sign of a rounding-level component every substep, so a
    # large pile has few env-steps without any band decision.
    assert len(clean) >= max(40, len(rows) // 10), "too many band steps for a meaningful comparison"
    assert max(r["contacts"] for r in rows) > 0
    for r in clean:
        assert r["keys"][0] == r["keys"][1]
        assert r["features_equal"]
        assert r["dq"] <= Q_TOL
        assert r["dv"] <= V_WORST_TOL
        assert r["dimp"] <= IMPULSE_WORST_TOL
    assert float(np.median([r["dv"] for r in clean])) <= V_MEDIAN_TOL
    assert float(np.median([r["dimp"] for r in clean])) <= IMPULSE_MEDIAN_TOL

