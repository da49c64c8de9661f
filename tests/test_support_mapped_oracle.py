"""The oracle's support-mapped narrowphase -- GJK, then EPA on overlap
with MPR as the fallback: the reference's primitive-GJK class,
Collision.metal:2298-3193 and 3434-3620 -- pinned to exact geometry, on the
CPU.

The reference has no CPU GJK, so the restatement is checked where the
answer is known independently:

* on shape pairs an analytic class also handles (sphere-sphere,
  sphere-capsule, capsule-capsule, sphere-box, capsule-box, box-box) the
  support-mapped query is forced through MR_COLLISION_PAIR_CONVEX and held
  to what each of its paths guarantees: a GJK distance bounds the analytic
  distance from above within GJK's own stopping gap; an EPA depth and
  normal match the analytic ones; an MPR witness (EPA out of iterations,
  typical of two curved supports) is conservative -- at least as deep as
  the analytic penetration, along a normal in the same half-space;
* a sphere against a cylinder has a closed-form distance;
* every support-mapped contact's witness points must be `separation`
  apart along its normal (GJK's exactly on the normal line).

EPA stops within 64 FLT_EPSILON x (scale + 1) of the depth (about 1.5e-5 m
at these scales); a curved support converges more slowly in direction than
in depth, so EPA normals are held to 5e-2 on curved pairs (about sqrt(2 tol / R)
for a 0.2 m summed radius, with margin) and 1e-3 on
box-box.
"""

from __future__ import annotations

import numpy as np
import pytest

import numi_lab_b200 as nb
from oracle import SceneOracle

SPHERE, CAPSULE, BOX, PLANE, CYLINDER = 0, 1, 2, 3, 4
CONVEX = 11
ANALYTIC = {(SPHERE, SPHERE): 1, (SPHERE, CAPSULE): 6, (CAPSULE, SPHERE): 6, (CAPSULE, CAPSULE): 7, (SPHERE, BOX): 8,
            (BOX, SPHERE): 8, (CAPSULE, BOX): 9, (BOX, CAPSULE): 9, (BOX, BOX): 10}
SEP_TOL = 1e-4
# Overlaps shallower than this compare depths exactly: there every analytic
# class's witness is the minimum translation.  Deeper, an analytic witness
# (a segment through a box, say) need not be, while EPA's still is.
SHALLOW = -0.01
NORMAL_TOL = {"curved": 5e-2, "flat": 1e-3}


@pytest.fixture(scope="module")
def scene():
    rec = nb.compile_model("cylinder_pile", 5)
    oracle = SceneOracle(rec, 0.005, 4, 8, 0)
    types = [int(rec.shapes[i].shape_type) for i in range(oracle.nb)]
    dims = [tuple(float(x) for x in rec.shapes[i].dimensions[:3]) for i in range(oracle.nb)]
    return oracle, types, dims


def _random_quat(rng) -> np.ndarray:
    q = rng.normal(size=4)
    return q / np.linalg.norm(q)


def _parked(n: int) -> np.ndarray:
    q = np.zeros((n, 7))
    q[:, 0] = 10.0 * np.arange(n)
    q[:, 2] = 5.0
    q[:, 6] = 1.0
    return q


def _extent(t: int, d) -> float:
    if t == SPHERE:
        return d[0]
    if t == CAPSULE:
        return d[0] + d[1]
    if t == BOX:
        return float(np.linalg.norm(d))
    return float(np.hypot(d[0], d[1]))


def _configs(scene, ta: int, tb: int, count: int, seed: int):
    """Poses of one body of type ta and one of tb, from well apart to deep overlap."""
    oracle, types, dims = scene
    a = types.index(ta)
    b = [i for i, t in enumerate(types) if t == tb and i != a][0]
    lo, hi = (a, b) if a < b else (b, a)
    rng = np.random.default_rng(seed)
    reach = _extent(types[lo], dims[lo]) + _extent(types[hi], dims[hi])
    for _ in range(count):
        q = _parked(oracle.nb)
        q[lo, :3] = [0.3, -0.2, 1.0]
        q[lo, 3:] = _random_quat(rng)
        direction = rng.normal(size=3)
        direction /= np.linalg.norm(direction)
        q[hi, :3] = q[lo, :3] + direction * reach * rng.uniform(0.35, 1.1)
        q[hi, 3:] = _random_quat(rng)
        yield lo, hi, q.reshape(-1)


def _unit(v):
    return v / np.linalg.norm(v)


def _gjk_gap(distance: float, q: np.ndarray, a: int, b: int) -> float:
    """Bound on GJK's distance error at its stopping test: it stops once the
    support advance along the unit direction -closest is within tol =
    32 FLT_EPSILON x (scale + 1), so the reported distance exceeds the true
    one by at most tol (the reference measures the advance along the
    unnormalised direction, Collision.metal:2372-2376, which lets the gap
    grow to tol / distance below 1 m)."""
    body = q.reshape(-1, 7)
    scale = max(np.abs(body[a, :3]).max(), np.abs(body[b, :3]).max()) + 0.5 + 1.0
    tol = 32.0 * 1.1920929e-7 * scale
    return tol + SEP_TOL


@pytest.mark.parametrize("ta,tb", [(SPHERE, SPHERE), (SPHERE, CAPSULE), (CAPSULE, CAPSULE), (SPHERE, BOX), (CAPSULE, BOX),
                                   (BOX, BOX)])
def test_gjk_epa_matches_the_analytic_classes(scene, ta, tb):
    oracle = scene[0]
    flat = ta == BOX and tb == BOX
    overlapping = by_epa = 0
    for a, b, q in _configs(scene, ta, tb, 200, 17 + 5 * ta + tb):
        cls = ANALYTIC[(scene[1][a], scene[1][b])]
        st_g, g, path = oracle.pair_query(q, a, b, CONVEX)
        st_a, r, _ = oracle.pair_query(q, a, b, cls)
        assert st_g == 0 and st_a == 0
        if len(r) == 0:
            # Beyond the accepted distance analytically: GJK's distance is an
            # upper bound, so it must not accept either.
            assert len(g) == 0, (ta, tb, g[0, 3])
            continue
        deepest = float(r[:, 3].min())
        if path == 0:
            # GJK found them apart: its distance bounds the analytic one from
            # above within its stopping gap (touching pairs included).
            if len(g):
                gap = _gjk_gap(max(g[0, 3], 1e-9), q, a, b)
                assert deepest - 1e-9 <= g[0, 3] <= max(deepest, 0.0) + gap, (ta, tb, g[0, 3], deepest)
            else:
                assert deepest + _gjk_gap(0.004, q, a, b) >= 0.004
            continue
        assert len(g) > 0
        overlapping += 1
        cos = float(np.dot(_unit(g[0, :3]), _unit(r[0, :3])))
        if path == 3:
            if deepest >= SHALLOW:
                assert abs(g[0, 3] - deepest) <= SEP_TOL, (ta, tb, g[0, 3], deepest)
                if deepest < -2 * SEP_TOL:
                    angle = float(np.arccos(np.clip(cos, -1.0, 1.0)))
                    assert angle <= NORMAL_TOL["flat" if flat else "curved"], (ta, tb, angle, deepest)
            by_epa += 1
        else:
            assert path == 1, path
            assert g[0, 3] <= min(deepest, 0.0) + SEP_TOL, (ta, tb, g[0, 3], deepest)
            assert cos > 0.0, (ta, tb, cos)
    assert overlapping >= 40
    # EPA resolves most overlaps that involve a flat face.
    if ta == BOX or tb == BOX:
        assert by_epa >= overlapping // 2, (by_epa, overlapping)


def _cylinder_distance(p, c, axis, radius, half_length):
    d = p - c
    a = float(np.dot(d, axis))
    rho = float(np.linalg.norm(d - a * axis))
    da, dr = abs(a) - half_length, rho - radius
    if da <= 0.0 and dr <= 0.0:
        return max(da, dr)  # inside: distance to the nearer face (negative)
    return float(np.hypot(max(da, 0.0), max(dr, 0.0)))


def _rotate(q, v):
    x, y, z, w = q
    u = np.array([x, y, z])
    return v + 2.0 * np.cross(u, np.cross(u, v) + w * v)


def test_sphere_cylinder_distance_is_the_closed_form(scene):
    oracle, types, dims = scene
    checked = 0
    for a, b, q in _configs(scene, SPHERE, CYLINDER, 200, 3):
        body = q.reshape(-1, 7)
        st, g, path = oracle.pair_query(q, a, b, CONVEX)
        s, c = (a, b) if types[a] == SPHERE else (b, a)
        radius, half = dims[c][0], dims[c][1]
        axis = _rotate(body[c, 3:], np.array([0.0, 1.0, 0.0]))
        dist = _cylinder_distance(body[s, :3], body[c, :3], axis, radius, half) - dims[s][0]
        assert st == 0
        if dist > 0.004 + 2e-4:
            assert len(g) == 0
            continue
        if len(g) == 0:
            assert dist + _gjk_gap(0.004, q, a, b) >= 0.004  # GJK's distance is an upper bound
            continue
        if path == 0:
            assert dist - 1e-9 <= g[0, 3] <= max(dist, 0.0) + _gjk_gap(max(g[0, 3], 1e-9), q, a, b), (g[0, 3], dist)
        elif path == 3:
            # Inside the cylinder's radius and slab the closed form is the
            # distance to the nearer face, which is EPA's minimum translation.
            assert abs(g[0, 3] - dist) <= SEP_TOL, (g[0, 3], dist)
        else:
            assert g[0, 3] <= min(dist, 0.0) + SEP_TOL, (g[0, 3], dist)
        checked += 1
    assert checked >= 40


@pytest.mark.parametrize("ta,tb", [(CYLINDER, CYLINDER), (CYLINDER, BOX), (CAPSULE, CYLINDER), (SPHERE, CYLINDER)])
def test_support_mapped_witnesses_are_consistent_and_mirror(scene, ta, tb):
    oracle, types, _ = scene
    contacts = 0
    for a, b, q in _configs(scene, ta, tb, 150, 29 + ta + 7 * tb):
        st, g, path = oracle.pair_query(q, a, b, CONVEX)
        assert st == 0
        for row in g:
            n, sep, pa, pb = row[:3], row[3], row[4:7], row[7:10]
            assert abs(np.linalg.norm(n) - 1.0) <= 1e-9
            if path == 1:
                # MPR's conservative witness: never reported as separation.
                assert sep <= 0.0
            else:
                # GJK and EPA witnesses (and the patch points taken from
                # them) sit `sep` apart along the normal.  GJK's lie on the
                # normal line; EPA's weighted supports may slide across a flat
                # contact face (any point of it is a witness).
                d = pb - pa
                assert abs(float(np.dot(d, n)) - sep) <= SEP_TOL, (float(np.dot(d, n)), sep)
                if path == 0:
                    assert float(np.linalg.norm(d - np.dot(d, n) * n)) <= SEP_TOL
        contacts += len(g)
    assert contacts >= 50


def test_cylinder_patch_gives_a_ring_on_a_flat_cap(scene):
    """A cylinder standing on a box face: the query point plus the four
    patch samples of the cap rim (Collision.metal:3363-3375)."""
    oracle, types, dims = scene
    c = types.index(CYLINDER)
    bx = types.index(BOX)
    lo, hi = min(c, bx), max(c, bx)
    q = _parked(oracle.nb)
    q[bx, :3] = [0.0, 0.0, 1.0]
    q[c, :3] = [0.0, 0.0, 1.0 + dims[bx][2] + dims[c][1] - 0.001]
    q[c, 3:] = [np.sqrt(0.5), 0.0, 0.0, np.sqrt(0.5)]  # local +Y (the axis) -> world +Z
    st, g, _ = oracle.pair_query(q.reshape(-1), lo, hi, CONVEX)
    assert st == 0
    assert len(g) == 5
    np.testing.assert_allclose(g[:, 3], -0.001, atol=SEP_TOL)
    cyl_points = g[:, 4:7] if lo == c else g[:, 7:10]
    # Patch points lie on the cap rim.
    rim = np.linalg.norm(cyl_points[1:, :2] - q[c, :2], axis=1)
    np.testing.assert_allclose(rim, dims[c][0], atol=1e-3)


@pytest.mark.reference
@pytest.mark.parametrize("seed", [1, 13])
def test_gjk_capsule_box_pile_matches_reference_witness(reference_available, seed):
    """A pile whose capsule-box pairs take the support-mapped query
    (pile_gjk): over a settling run, every capsule-box pair the reference's
    CPU collision (analytic capsule-box witness, Collision.cpp:1462) puts in
    contact, the oracle's GJK / EPA query puts in contact too, with the
    deepest separation within SEP_TOL and, for overlaps deeper than that,
    the normal within the curved-shape angle."""
    import numi_lab_b200 as nb
    from oracle import ReferenceScene, SceneOracle, SceneTable

    rec = nb.compile_model("pile_gjk", seed)
    types = [int(rec.shapes[i].shape_type) for i in range(rec.world.shape_count)]
    oracle = SceneOracle(rec, 0.005, 4, 8, 0)
    q, v, f = nb.sample_reset("pile_gjk", seed, 1, 0, 1)
    q, v = q[0].astype(np.float64), v[0].astype(np.float64)
    table, ctable, ref = SceneTable(), SceneTable(), ReferenceScene(rec)
    compared = 0
    for _ in range(80):
        assert oracle.step(q, v, table, float(f[0]))[0] == 0
        s1, raw = oracle.collide(q, ctable)
        s2, raw_ref, _ = ref.collide(q)
        assert s1 == 0 and s2 == 0
        ours = {}
        for r in raw:
            ours.setdefault((int(r[0]), int(r[1])), []).append(r)
        seen = set()
        for r in raw_ref:
            a, b = int(r[0]), int(r[1])
            if (a, b) in seen or b >= len(types) - 1 or {types[a], types[b]} != {CAPSULE, BOX}:
                continue
            seen.add((a, b))
            rows = [x for x in raw_ref if int(x[0]) == a and int(x[1]) == b]
            deepest = min(float(x[5]) for x in rows)
            accept = float(rec.shapes[a].contact_rest_bound[0]) + float(rec.shapes[b].contact_rest_bound[0])
            if (a, b) not in ours:
                # Only a contact within the acceptance band may be missing here.
                assert deepest >= accept - 5e-5, (a, b, deepest, accept)
                continue
            g = ours[(a, b)][0]
            if deepest <= 0.0:
                # Overlap: EPA's depth equals the analytic one.
                assert abs(float(g[5]) - deepest) <= SEP_TOL, (a, b, float(g[5]), deepest)
                if deepest < -2 * SEP_TOL:
                    ref_n = min(rows, key=lambda x: float(x[5]))[2:5]
                    cos = float(np.dot(_unit(g[2:5]), _unit(ref_n)))
                    assert float(np.arccos(np.clip(cos, -1.0, 1.0))) <= NORMAL_TOL["curved"], (a, b, cos)
            else:
                # Apart: GJK's distance bounds the analytic one from above
                # within its stopping gap (the reference publishes FP32).
                assert deepest - 2e-6 <= float(g[5]) <= deepest + _gjk_gap(max(float(g[5]), 1e-9), q, a, b), (a, b, g[5], deepest)
            compared += 1
    assert compared > 20
