"""The oracle's hull path of the support-mapped narrowphase -- a convex hull
(MR_SHAPE_CONVEX) against the plane, a primitive or another hull:
Collision.metal:1899-1936 (hull support), 3129-3260 (support-axis witness),
3327-3432 (patch), 3623-3720 (the hull query) -- checked on the CPU where
the answer is known independently (the reference has no CPU hull query):

* a hull on the plane: its deepest vertex, at its signed height;
* a hull apart from a sphere: GJK's distance equals the distance from the
  sphere's centre to the hull (a small quadratic program over the
  vertices) less the radius, within GJK's stopping gap;
* overlapping hulls: the separation and normal are the best of the
  witness's seven candidate axes, recomputed here from the vertices;
* every hull contact's witness points are `separation` apart along its
  normal, and a flat hull face on a hull gives a patch of several points.
"""

from __future__ import annotations

import numpy as np
import pytest
from scipy.optimize import minimize

import numi_lab_b200 as nb
from oracle import SceneOracle

SPHERE, CAPSULE, BOX, PLANE, CONVEX_SHAPE = 0, 1, 2, 3, 5
CONVEX_CLASS = 11
SEP_TOL = 1e-4


@pytest.fixture(scope="module")
def scene():
    rec = nb.compile_model("hull_pile", 7)
    oracle = SceneOracle(rec, 0.005, 4, 8, 0)
    types = [int(rec.shapes[i].shape_type) for i in range(oracle.nb)]
    dims = [np.array(rec.shapes[i].dimensions[:3], np.float64) for i in range(oracle.nb)]
    hulls = {}
    for i in range(oracle.nb):
        if types[i] == CONVEX_SHAPE:
            s = rec.shapes[i]
            v = rec.hull_vertices[s.hull_first:s.hull_first + s.hull_count, :3].astype(np.float64)
            hulls[i] = v * dims[i]
    return oracle, types, dims, hulls


def _rot(q: np.ndarray) -> np.ndarray:
    x, y, z, w = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def _random_quat(rng) -> np.ndarray:
    q = rng.normal(size=4)
    return q / np.linalg.norm(q)


def _parked(n: int) -> np.ndarray:
    q = np.zeros((n, 7))
    q[:, 0] = 10.0 * np.arange(n)
    q[:, 2] = 5.0
    q[:, 6] = 1.0
    return q


def _world_vertices(hulls, i, pose) -> np.ndarray:
    return pose[:3] + hulls[i] @ _rot(pose[3:]).T


def test_hull_on_the_plane_is_its_deepest_vertex(scene):
    oracle, types, dims, hulls = scene
    rng = np.random.default_rng(2)
    plane = oracle.nb
    for i in list(hulls)[:4]:
        for _ in range(10):
            q = _parked(oracle.nb)
            q[i, :3] = [0.0, 0.0, rng.uniform(-0.05, 0.2)]
            q[i, 3:] = _random_quat(rng)
            st, rows, _ = oracle.pair_query(q.reshape(-1), i, plane, CONVEX_CLASS)
            assert st == 0
            w = _world_vertices(hulls, i, q[i])
            k = int(np.argmin(w[:, 2]))
            depth = w[k, 2]
            if depth > 0.002 + SEP_TOL:  # beyond the contact offset: no contact
                assert len(rows) == 0
                continue
            assert len(rows) == 1
            normal, sep, pa = rows[0, :3], rows[0, 3], rows[0, 4:7]
            # The plane's normal comes from its FP32 rotation (3e-8 off +Z).
            np.testing.assert_allclose(normal, [0.0, 0.0, -1.0], atol=1e-7)
            assert abs(sep - depth) <= 1e-7
            np.testing.assert_allclose(pa, w[k], atol=1e-9)
            assert int(rows[0, 10]) & 0x0fffffff == k  # vertex feature


def _point_to_hull(p: np.ndarray, verts: np.ndarray) -> float:
    n = len(verts)
    res = minimize(lambda w: float(np.sum((w @ verts - p) ** 2)), np.full(n, 1.0 / n), method="SLSQP",
                   jac=lambda w: 2.0 * verts @ (w @ verts - p), bounds=[(0.0, 1.0)] * n,
                   constraints=[{"type": "eq", "fun": lambda w: np.sum(w) - 1.0, "jac": lambda w: np.ones(n)}],
                   options={"ftol": 1e-16, "maxiter": 500})
    return float(np.sqrt(max(res.fun, 0.0)))


def test_hull_sphere_distance_is_the_point_to_hull_distance(scene):
    oracle, types, dims, hulls = scene
    rng = np.random.default_rng(4)
    h = next(iter(hulls))
    s = types.index(SPHERE)
    lo, hi = min(h, s), max(h, s)
    checked = 0
    for _ in range(40):
        q = _parked(oracle.nb)
        q[h, :3] = [0.3, -0.2, 1.0]
        q[h, 3:] = _random_quat(rng)
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        reach = np.linalg.norm(hulls[h], axis=1).max() + dims[s][0]
        q[s, :3] = q[h, :3] + d * reach * rng.uniform(1.05, 1.4)
        # A 1 m speculative margin makes every separated pose report its distance.
        rows = oracle.raw_contacts(q.reshape(-1), lo, hi, 1.0, 0.0)
        exact = _point_to_hull(q[s, :3], _world_vertices(hulls, h, q[h])) - dims[s][0]
        assert len(rows) >= 1 and exact > 0.0
        # GJK stops within 32 FLT_EPSILON x (scale + 1) of the distance.
        assert abs(rows[0, 3] - exact) <= 32 * 1.1920929e-7 * 3.0 + 1e-7
        checked += 1
    for _ in range(40):  # overlapping: at least as deep as the exact depth is not claimed; separation <= 0
        q = _parked(oracle.nb)
        q[h, :3] = [0.3, -0.2, 1.0]
        q[h, 3:] = _random_quat(rng)
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        q[s, :3] = q[h, :3] + d * 0.3 * np.linalg.norm(hulls[h], axis=1).min()
        st, rows, path = oracle.pair_query(q.reshape(-1), lo, hi, CONVEX_CLASS)
        assert st == 0 and len(rows) >= 1 and path == 2
        assert rows[0, 3] <= 0.0
    assert checked == 40


def _axis_separation(hulls, a, b, qa, qb, axis) -> float:
    wa, wb = _world_vertices(hulls, a, qa), _world_vertices(hulls, b, qb)
    return float(np.min(wb @ axis) - np.max(wa @ axis))


def test_overlapping_hulls_take_the_best_candidate_axis(scene):
    oracle, types, dims, hulls = scene
    rng = np.random.default_rng(6)
    a, b = list(hulls)[:2]
    seen = 0
    for _ in range(60):
        q = _parked(oracle.nb)
        q[a, :3] = [0.3, -0.2, 1.0]
        q[a, 3:] = _random_quat(rng)
        q[b, 3:] = _random_quat(rng)
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        q[b, :3] = q[a, :3] + d * 0.5 * (np.linalg.norm(hulls[a], axis=1).max() + np.linalg.norm(hulls[b], axis=1).max())
        st, rows, path = oracle.pair_query(q.reshape(-1), a, b, CONVEX_CLASS)
        assert st == 0
        if path != 2:
            continue  # GJK found them apart
        delta = q[b, :3] - q[a, :3]
        axes = [delta] + [(_rot(q[a, 3:]) @ e) for e in np.eye(3)] + [(_rot(q[b, 3:]) @ e) for e in np.eye(3)]
        best, best_axis = -np.inf, None
        for ax in axes:
            ax = ax / np.linalg.norm(ax)
            if ax @ delta < 0.0:
                ax = -ax
            sep = _axis_separation(hulls, a, b, q[a], q[b], ax)
            if sep > best:
                best, best_axis = sep, ax
        assert abs(rows[0, 3] - min(best, 0.0)) <= 1e-9
        np.testing.assert_allclose(rows[0, :3], best_axis, atol=1e-9)
        # Witness points `separation` apart along the normal.
        pa, pb = rows[0, 4:7], rows[0, 7:10]
        assert abs((pb - pa) @ rows[0, :3] - rows[0, 3]) <= 1e-9 or rows[0, 3] == 0.0
        seen += 1
    assert seen >= 10


def test_a_face_down_hull_resting_on_a_box_gets_a_patch(scene):
    """A hull lying on a large flat box face: the witness plus supports
    along the tilted normal give more than one contact point, every one at
    the query's separation along its normal."""

    oracle, types, dims, hulls = scene
    h = next(iter(hulls))
    bx = max((i for i, t in enumerate(types) if t == BOX), key=lambda i: dims[i].min())
    rng = np.random.default_rng(8)
    multi = 0
    for _ in range(30):
        q = _parked(oracle.nb)
        q[bx, :3] = [0.0, 0.0, 1.0]
        q[bx, 3:] = [0.0, 0.0, 0.0, 1.0]
        q[h, 3:] = _random_quat(rng)
        w = _world_vertices(hulls, h, np.concatenate([[0.0, 0.0, 0.0], q[h, 3:]]))
        q[h, :3] = [rng.uniform(-0.01, 0.01), rng.uniform(-0.01, 0.01), 1.0 + dims[bx][2] - w[:, 2].min() - 1e-3]
        lo, hi = min(h, bx), max(h, bx)
        st, rows, path = oracle.pair_query(q.reshape(-1), lo, hi, CONVEX_CLASS)
        assert st == 0 and len(rows) >= 1
        for r in rows:
            assert abs(r[3] - rows[0, 3]) <= 1e-12
            assert abs((r[7:10] - r[4:7]) @ r[:3] - r[3]) <= 1e-9
        multi += len(rows) > 1
    assert multi >= 1
