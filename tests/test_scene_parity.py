"""Free-body piles: CUDA control step vs the oracle, one control step at a
time from identical FP32 input state (the CUDA path runs through the C ABI).

Each environment is a pile of 8-64 boxes and spheres dropped onto a plane.
The oracle restates the device stage order in FP64 (oracle/oracle.c).
Discrete decisions -- manifold pair keys, point features and lifetimes,
island partitions, status codes -- must agree exactly, except at steps
where the oracle took a decision within its band of a threshold (5e-5 for
piles: within a control step the device trajectory departs from the
oracle's by up to ~5e-6 in position, and later substeps decide on the
departed state) or where rounding the inputs flips a decision in the oracle
itself.  Continuous state is compared relative to max(1, |x|) of the oracle
state, every clean env-step against its own bound: max(1e-5, K x the FP64
oracle's sensitivity to rounding its FP32 inputs) for q and body velocities
and max(1e-4, K x sensitivity) for impulses (tests/_sensitivity.py).
"""

from __future__ import annotations

import numpy as np
import pytest

import numi_lab_b200 as nb
from oracle import SceneOracle

pytestmark = pytest.mark.gpu

# Per control step base tolerances (relative to max(1, |x|)); each env-step
# is held to max(base, K x the oracle's FP32-input sensitivity).
Q_TOL = 1e-5
V_TOL = 1e-5
IMPULSE_TOL = 1e-4


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
    """Per control step from identical FP32 state: one row per env-step with
    the device's and the oracle's decisions, the errors and their per-step
    bounds (tests/_sensitivity.py)."""

    import torch

    import _sensitivity as S

    substeps, iters = 4, 8
    rows = []
    with nb.World(source, envs, substeps=substeps, velocity_iterations=iters, control_dt=0.02, seed=seed,
                  precision=precision) as world, S.pool() as ex:
        world.set_island_labels(True)
        fr = world.friction_scales()
        acts = torch.zeros((1, envs, 0), device="cuda")
        for k in range(steps):
            q0, v0, t0 = world.state()
            c0 = _counts(t0)
            _, status, _ = world.step(acts, wait=True)
            st = status.cpu().numpy()[0]
            q1, v1, t1 = world.state()
            labels = world.island_labels()
            c1 = _counts(t1)
            jobs = [{"source": source, "seed": seed, "h": 0.02 / substeps, "substeps": substeps, "iters": iters, "q": q0[e],
                     "v": v0[e], "table": t0[e], "count": c0[e], "friction": float(fr[e]), "rng": 1000 * k + e}
                    for e in range(envs)]
            for e, res in enumerate(ex.map(S.scene_env_step, jobs, chunksize=2)):
                row = {
                    "status": (int(st[e]), res["status"]),
                    "res": res,
                    "contacts": res["contacts"],
                    "keys": (_keys(t1, e, c1[e]), [f[0] for f in res["features"]]),
                    "features_equal": True,
                    "islands_equal": True,
                    "dq": S.rel_err(q1[e], res["q"]),
                    "dv": S.rel_err(v1[e], res["v"]),
                    "dimp": 0.0,
                    "sens": res["sens"],
                }
                if row["keys"][0] == row["keys"][1]:
                    dev_imps, dev_feats = [], []
                    for i in range(c1[e]):
                        w = t1[e, i]
                        count = int(w[7].view(np.uint32))
                        pts = []
                        for p in range(count):
                            pw = w[8 + 12 * p: 20 + 12 * p]
                            pts.append((int(pw[6].view(np.uint32)), int(pw[7].view(np.uint32)), int(pw[8].view(np.uint32))))
                            dev_imps.append([float(x) for x in pw[9:12]])
                        dev_feats.append((int(w[56].view(np.uint32)), tuple(pts)))
                    row["features_equal"] = tuple(dev_feats) == res["features"]
                    imp = np.array(dev_imps, np.float64).reshape(-1, 3)
                    if row["features_equal"] and imp.size:
                        row["dimp"] = float(np.max(np.abs(imp - res["imp"]))) / max(1.0, float(np.max(np.abs(res["imp"]))))
                    nbod = labels.shape[1]
                    want = np.where(res["island_of"][:nbod] == 0xFFFFFFFF, 255, res["island_of"][:nbod]).astype(np.uint8)
                    row["islands_equal"] = res["contacts"] == 0 or np.array_equal(labels[e], want)
                rows.append(row)
    return rows


def _check_rows(rows, min_clean: int) -> list:
    """Every env-step: identical decisions and island partitions, continuous
    state within its per-step bound -- except band steps (tests/_sensitivity.py),
    which must leave at least `min_clean` matched env-steps."""

    import _sensitivity as S

    assert all(r["status"][0] == r["status"][1] == 0 for r in rows)
    assert max(r["contacts"] for r in rows) > 0
    matched, band, failures, plain = 0, 0, [], 0
    for r in rows:
        same = r["keys"][0] == r["keys"][1] and r["features_equal"] and r["islands_equal"]
        verdict, misses = S.judge(r["res"], same, {"q": r["dq"], "v": r["dv"], "imp": r["dimp"]})
        if verdict == "fail":
            failures.append(misses)
        elif verdict == "band":
            band += 1
        else:
            matched += 1
            plain += r["dq"] <= Q_TOL and r["dv"] <= V_TOL and r["dimp"] <= IMPULSE_TOL
    print(f"{matched} matched, {band} band of {len(rows)} env-steps; {plain} within the plain tolerances")
    assert not failures, failures[:10]
    assert matched >= min_clean, "too many band steps for a meaningful comparison"
    return rows


@pytest.mark.parametrize("seed,precision", [(3, "fp32"), (10, "fp32"), (13, "fp32"), (1, "fp32"),  # 10, 8, 17, 50 bodies
                                            (13, "compensated"), (1, "compensated")])
def test_pile_control_steps_match_oracle(cuda_device, seed, precision):
    rows = _compare_run(seed, 8, 60, precision)
    _check_rows(rows, len(rows) // 2)


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


def _overflow_states(world) -> np.ndarray:
    """Four states of the 64-body pile (seed 31: 14 spheres, 24 capsules,
    26 boxes), each the first substep of a capacity limit in the oracle:
    every body at one point (2016 overlapping body pairs for 512 candidate
    slots ->
    MR_STEP_PAIR_CAPACITY_OVERFLOW), the bodies 4 cm apart on a line (more
    touching pairs than the 128 manifold slots -> MANIFOLD), boxes face to
    face in a row, spheres in a row and capsules apart, all resting 1 mm
    deep on the plane (283 contact points for 256 solver rows -> CONTACT),
    and a settled state that fits."""

    model = world.model()
    n = int(model.world.body_count) - 1
    types = [int(model.shapes[i].shape_type) for i in range(n)]
    dims = [np.array(model.shapes[i].dimensions[:3], np.float64) for i in range(n)]
    q = np.zeros((4, n, 7))
    q[..., 6] = 1.0
    q[0, :, 2] = 0.5
    q[1, :, 0] = 0.04 * np.arange(n)
    q[1, :, 2] = 0.2
    pen, end = 0.001, {0: None, 2: None}
    for i, t in enumerate(types):
        if t in end:  # spheres and boxes in rows, each 1 mm into the previous one
            half = dims[i][0]
            q[2, i, 0] = 0.0 if end[t] is None else end[t] + half - pen
            end[t] = q[2, i, 0] + half
            q[2, i, 1] = 0.0 if t == 2 else 1.0
            q[2, i, 2] = (dims[i][2] if t == 2 else dims[i][0]) - pen
        else:  # capsules lie along their local y axis, apart
            q[2, i, :3] = [0.5 * i, 2.0, dims[i][0] - pen]
    return q


def test_pile_capacity_overflows_latch_like_the_oracle(cuda_device):
    """Capacity limits are statuses, not truncations: an environment whose
    candidate pairs, manifolds or solver contacts exceed their capacity
    reports the same status code as the oracle and keeps its state
    bit for bit; the other environments step on."""

    import torch

    from oracle import SceneTable

    envs = 4
    with nb.World("pile", envs, seed=31) as world:
        acts = torch.zeros((1, envs, 0), device="cuda")
        for _ in range(5):
            world.step(acts, wait=True)
        q0, v0, _ = world.state()
        n = q0.shape[1] // 7
        states = _overflow_states(world)
        q = q0.copy()
        v = np.zeros_like(v0)
        for e in range(3):
            q[e] = states[e].reshape(-1)
        v[3] = v0[3]
        empty = np.zeros((envs,) + world.state()[2].shape[1:], np.float32)
        world.set_state(q, v, empty)
        q_in, v_in, _ = world.state()
        oracle = SceneOracle(world.model(), 0.005, 4, 8, 0)
        friction = world.friction_scales()
        want = []
        for e in range(envs):
            qo, vo = q_in[e].astype(np.float64), v_in[e].astype(np.float64)
            st, _ = oracle.step(qo, vo, SceneTable(), float(friction[e]))
            want.append((st, qo))
        assert [w[0] for w in want] == [4, 6, 5, 0]
        for k in range(2):  # the failed environments fail again from the kept state
            _, status, _ = world.step(acts, wait=True)
            st = status.cpu().numpy()[0].tolist()
            assert st[:3] == [w[0] for w in want[:3]] and st[3] == 0
            q1, v1, _ = world.state()
            np.testing.assert_array_equal(q1[:3], q_in[:3])
            np.testing.assert_array_equal(v1[:3], v_in[:3])
            if k == 0:
                qo = want[3][1]
                assert np.max(np.abs(q1[3] - qo)) <= Q_TOL * max(1.0, np.max(np.abs(qo)))
        assert n == 64


@pytest.mark.parametrize("seed", [3, 11, 5])  # 10, 25 and 49 bodies, one quarter cylinders
def test_cylinder_pile_control_steps_match_oracle(cuda_device, seed):
    """Piles with cylinders: the support-mapped narrowphase (GJK, EPA, MPR,
    the cylinder patch) and cylinder-on-plane contacts on the device against
    the oracle's FP64 restatement, under the pile tolerances.  A support
    point or witness feature picked within rounding of a tie (a box face
    across the normal, near-equal barycentric weights) is a band decision."""
    rows = _compare_run(seed, 8, 60, "fp32", "cylinder_pile")
    # Resting contact of a box face on a cylinder picks the box's support
    # vertex by the sign of a rounding-level component every substep, so a
    # large pile has few env-steps without any band decision.
    _check_rows(rows, max(40, len(rows) // 10))


@pytest.mark.parametrize("seed", [3, 7, 5])  # one quarter convex hulls of 12 vertices
def test_hull_pile_control_steps_match_oracle(cuda_device, seed):
    """Piles with convex hulls (MR_RUN_SOURCE_SYNTHETIC_HULL_PILE): the hull
    path of the support-mapped narrowphase -- GJK distance, the
    support-axis penetration witness, the sampled patch, the deepest vertex
    on the plane -- on the device against the oracle's FP64 restatement,
    under the pile tolerances.  A hull vertex or witness axis picked within
    rounding of a tie is a band decision."""
    rows = _compare_run(seed, 8, 60, "fp32", "hull_pile")
    _check_rows(rows, max(40, len(rows) // 10))


@pytest.mark.parametrize("seed", [3, 13, 1])  # 10, 17 and 50 bodies
def test_gjk_capsule_box_pile_control_steps_match_oracle(cuda_device, seed):
    """Piles whose capsule-box pairs take the support-mapped narrowphase
    (GJK, EPA with MPR fallback; MR_RUN_SOURCE_SYNTHETIC_PILE_GJK) on the
    device against the oracle's FP64 restatement of the same query."""
    rows = _compare_run(seed, 8, 60, "fp32", "pile_gjk")
    _check_rows(rows, len(rows) // 4)
