"""The pile oracle (oracle/oracle.c, free-body scene restatement) against
the reference's FP64 CPU collision -- from golden fixtures
(tests/golden/pile_collision.npz) and, where the reference-core library is
built, live over longer runs -- plus physical sanity checks of the whole
control step.  CPU only."""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

import numi_lab_b200 as nb
from oracle import SceneOracle, SceneTable

import _pile

GOLDEN = Path(__file__).resolve().parent / "golden" / "pile_collision.npz"
H = 0.005


@pytest.fixture(scope="module")
def golden():
    if not GOLDEN.is_file():
        pytest.skip("golden fixture missing")
    return np.load(GOLDEN)


@pytest.mark.parametrize("seed", [3, 13, 14])
def test_pile_collision_matches_reference_golden(golden, seed):
    p = f"seed{seed}_"
    rec = nb.compile_model("pile", seed)
    fp = np.frombuffer(bytes(rec.bodies) + bytes(rec.shapes), np.uint8)
    assert np.array_equal(fp, golden[p + "fingerprint"]), "pile model drifted from the fixture"
    oracle = SceneOracle(rec, H, 4, 8, 0)
    table = SceneTable()
    tainted: set = set()
    raw_at = np.concatenate([[0], np.cumsum(golden[p + "raw_rows"])])
    man_at = np.concatenate([[0], np.cumsum(golden[p + "manifold_rows"])])
    matched = checked = 0
    for k, q in enumerate(golden[p + "q"]):
        status, raw = oracle.collide(q, table)
        assert status == 0
        r = _pile.compare_raw(rec, raw, golden[p + "raw"][raw_at[k]:raw_at[k + 1]], tainted)
        matched += r["matched"]
        checked += _pile.compare_manifolds(table, golden[p + "manifolds"][man_at[k]:man_at[k + 1]], tainted)
    assert matched > 0 and checked > 0


@pytest.mark.reference
@pytest.mark.parametrize("seed", [1, 6, 9, 14, 17])
def test_pile_collision_matches_reference_live(reference_available, seed):
    from oracle import ReferenceScene

    rec = nb.compile_model("pile", seed)
    oracle = SceneOracle(rec, H, 4, 8, 0)
    q, v, f = nb.sample_reset("pile", seed, 1, 0, 1)
    q = q[0].astype(np.float64)
    v = v[0].astype(np.float64)
    table, ctable, ref = SceneTable(), SceneTable(), ReferenceScene(rec)
    tainted: set = set()
    matched = checked = 0
    for _ in range(100):
        status, _ = oracle.step(q, v, table, float(f[0]))
        assert status == 0
        s1, raw = oracle.collide(q, ctable)
        s2, raw_ref, man_ref = ref.collide(q)
        assert s1 == 0 and s2 == 0
        matched += _pile.compare_raw(rec, raw, raw_ref, tainted)["matched"]
        checked += _pile.compare_manifolds(ctable, man_ref, tainted)
    assert matched > 1000 and checked > 100
    assert len(tainted) <= 3


def test_resting_pile_settles_on_the_plane():
    # After two simulated seconds every body rests on the plane or on other
    # bodies: nothing below the plane beyond the rest slop, nothing moving.
    seed = 10
    rec = nb.compile_model("pile", seed)
    oracle = SceneOracle(rec, H, 4, 8, 0)
    q, v, f = nb.sample_reset("pile", seed, 1, 0, 1)
    q = q[0].astype(np.float64)
    v = v[0].astype(np.float64)
    table = SceneTable()
    for _ in range(100):
        status, trace = oracle.step(q, v, table, float(f[0]))
        assert status == 0
    n = rec.world.body_count - 1
    pos = q.reshape(n, 7)[:, :3]
    for b in range(n):
        sh = rec.shapes[b]
        lowest = float(sh.dimensions[0]) if sh.shape_type == 0 else 0.0
        if sh.shape_type == 0:
            assert pos[b, 2] >= lowest - 2e-3
    assert np.max(np.abs(v)) < 0.05
    assert trace.contact_count > n  # every body touches something


def test_sphere_on_plane_rest_height_and_zero_impulse_drift():
    # A lone sphere dropped on the plane comes to rest with its lowest point
    # within the depenetration slop of the plane, and its normal impulse per
    # substep settles to m g h.
    seed = 10
    rec = nb.compile_model("pile", seed)
    n = rec.world.body_count - 1
    spheres = [b for b in range(n) if rec.shapes[b].shape_type == 0]
    assert spheres
    oracle = SceneOracle(rec, H, 4, 8, 0)
    q = np.zeros(7 * n)
    v = np.zeros(6 * n)
    for b in range(n):  # spread far apart so only the plane is touched
        q[7 * b: 7 * b + 3] = [3.0 * b, 0.0, 0.5]
        q[7 * b + 6] = 1.0
    table = SceneTable()
    for _ in range(150):
        status, _ = oracle.step(q, v, table, 1.0)
        assert status == 0
    for b in spheres:
        r = float(rec.shapes[b].dimensions[0])
        assert abs(q[7 * b + 2] - r) < 2e-3
    keys = table.keys()
    mass = {b: float(rec.bodies[b].mass_inverse_mass[0]) for b in range(n)}
    for i, key in enumerate(keys):
        a = key // 65
        if a in spheres:
            m = table.slots[i].m
            assert m.count == 1
            assert abs(m.points[0].impulses[0] - mass[a] * 9.81 * H) < 1e-3 * mass[a] * 9.81 * H + 1e-9


def test_failed_step_publishes_nothing():
    seed = 3
    rec = nb.compile_model("pile", seed)
    oracle = SceneOracle(rec, H, 4, 8, 0)
    q, v, f = nb.sample_reset("pile", seed, 1, 0, 1)
    q = q[0].astype(np.float64)
    v = v[0].astype(np.float64)
    table = SceneTable()
    for _ in range(40):
        assert oracle.step(q, v, table, float(f[0]))[0] == 0
    q[3:7] = np.nan
    q0, v0, keys0 = q.copy(), v.copy(), table.keys()
    status, trace = oracle.step(q, v, table, float(f[0]))
    assert status == 2 and trace.failing_index == 0
    np.testing.assert_array_equal(np.isnan(q), np.isnan(q0))
    np.testing.assert_array_equal(v, v0)
    assert table.keys() == keys0


CYLINDER, CONVEX_CLASS = 4, 11
RIM_FEATURES = (10, 11)  # general rim points of a cylinder (Collision.metal:26-27)


def _rim_conditioning(rec, q):
    """Rounding bound of a cylinder's general-rim point on the plane: the
    rim azimuth is -radial / |radial| of the plane normal in the disk basis,
    so a normal perturbation of ~2e-7 (FP32 plane rotation) moves the point
    by radius x 2e-7 / |radial| -- large when the cylinder stands nearly
    upright on its cap."""
    body = q.reshape(-1, 7)

    def bound(pair, feat, row):
        a = pair[0]
        if (feat[0] >> 28) != CYLINDER:
            return 0.0
        x, y, z, w = body[a, 3:]
        u = np.array([x, y, z])
        v = np.array([0.0, 1.0, 0.0])
        axis = v + 2.0 * np.cross(u, np.cross(u, v) + w * v)
        axial = abs(float(np.dot(axis / np.linalg.norm(axis), row[2:5])))
        radial = np.sqrt(max(1e-30, 1.0 - axial * axial))
        # The cap-ring and side-rim classes are taken at |axial| or
        # |radial| <= 1e-6 (Collision.metal:21): within rounding of that
        # threshold either side may take the other class.
        if axial <= 1e-5 or radial <= 1e-5:
            return np.inf
        if (feat[0] & 0x0FFFFFFF) not in RIM_FEATURES:
            return 0.0
        radius = float(rec.shapes[a].dimensions[0])
        return 4.0 * radius * 2e-7 / radial

    return bound


@pytest.mark.reference
@pytest.mark.parametrize("seed", [5, 8, 11])
def test_cylinder_pile_collision_matches_reference_live(reference_available, seed):
    """Piles with cylinders: every class the reference's CPU collision
    handles -- cylinder on the plane among them -- against the oracle; the
    reference's CPU skips cylinder-finite pairs (no CPU GJK), so the
    oracle's support-mapped pairs are left out (they are pinned in
    tests/test_support_mapped_oracle.py)."""
    from oracle import ReferenceScene

    rec = nb.compile_model("cylinder_pile", seed)
    cls = {(int(rec.pairs[i].shape_a), int(rec.pairs[i].shape_b)): int(rec.pairs[i].pair_class)
           for i in range(int(rec.world.pair_count))}
    oracle = SceneOracle(rec, H, 4, 8, 0)
    q, v, f = nb.sample_reset("cylinder_pile", seed, 1, 0, 1)
    q = q[0].astype(np.float64)
    v = v[0].astype(np.float64)
    table, ctable, ref = SceneTable(), SceneTable(), ReferenceScene(rec)
    tainted: set = set()
    matched = checked = cylinder_plane = 0
    for _ in range(100):
        status, _ = oracle.step(q, v, table, float(f[0]))
        assert status == 0
        s1, raw = oracle.collide(q, ctable)
        s2, raw_ref, man_ref = ref.collide(q)
        assert s1 == 0 and s2 == 0
        keep = np.array([cls[(int(r[0]), int(r[1]))] != CONVEX_CLASS for r in raw], bool)
        tainted |= {(int(r[0]), int(r[1])) for r in raw[~keep]}
        matched += _pile.compare_raw(rec, raw[keep], raw_ref, tainted, _rim_conditioning(rec, q))["matched"]
        cylinder_plane += sum(1 for r in raw_ref if cls[(int(r[0]), int(r[1]))] == 5)
        checked += _pile.compare_manifolds(ctable, man_ref, tainted)
    assert matched > 1000 and checked > 100
    assert cylinder_plane > 50


@pytest.mark.parametrize("seed", [5, 11])
def test_cylinder_pile_collision_matches_reference_golden(golden, seed):
    """The fixture's cylinder piles: the reference's CPU contacts (cylinder
    on the plane included) against the oracle's, support-mapped pairs left
    out as in the live test."""
    p = f"cylinder_seed{seed}_"
    rec = nb.compile_model("cylinder_pile", seed)
    fp = np.frombuffer(bytes(rec.bodies) + bytes(rec.shapes), np.uint8)
    assert np.array_equal(fp, golden[p + "fingerprint"]), "cylinder pile model drifted from the fixture"
    cls = {(int(rec.pairs[i].shape_a), int(rec.pairs[i].shape_b)): int(rec.pairs[i].pair_class)
           for i in range(int(rec.world.pair_count))}
    oracle = SceneOracle(rec, H, 4, 8, 0)
    table = SceneTable()
    tainted: set = set()
    raw_at = np.concatenate([[0], np.cumsum(golden[p + "raw_rows"])])
    man_at = np.concatenate([[0], np.cumsum(golden[p + "manifold_rows"])])
    matched = checked = cylinder_plane = 0
    for k, q in enumerate(golden[p + "q"]):
        status, raw = oracle.collide(q, table)
        assert status == 0
        keep = np.array([cls[(int(r[0]), int(r[1]))] != CONVEX_CLASS for r in raw], bool)
        tainted |= {(int(r[0]), int(r[1])) for r in raw[~keep]}
        ref_raw = golden[p + "raw"][raw_at[k]:raw_at[k + 1]]
        matched += _pile.compare_raw(rec, raw[keep], ref_raw, tainted, _rim_conditioning(rec, q))["matched"]
        cylinder_plane += sum(1 for r in ref_raw if cls[(int(r[0]), int(r[1]))] == 5)
        checked += _pile.compare_manifolds(table, golden[p + "manifolds"][man_at[k]:man_at[k + 1]], tainted)
    assert matched > 0 and checked > 0 and cylinder_plane > 0

