"""Comparison helpers for free-body pile collision: the oracle's raw
contacts and persistent manifolds against the reference's
(collideCpuReference, src/core/Collision.cpp:2959), live or from golden
fixtures.

The device path, like the reference's Metal collision, accepts a contact up
to the summed contact offsets plus a scale-aware query pad (about 1.5e-5 m
here); the reference's FP64 CPU collision accepts up to the offsets alone.
Contacts whose separation lies within ACCEPT_BAND of the summed offsets may
therefore be present on one side only; a pair that ever had such a contact
is left out of the manifold comparison for the rest of the run, because
its point lifetimes then legitimately differ; so is a pair whose box-box
support fallback picked the other end of a tied edge.
"""

from __future__ import annotations

import numpy as np

ACCEPT_BAND = 5e-5
GEOMETRY_TOL = 2e-6  # the reference publishes raw contacts in FP32


def contact_distance(records, a: int, b: int) -> float:
    return float(records.shapes[a].contact_rest_bound[0]) + float(records.shapes[b].contact_rest_bound[0])


def group_raw(raw: np.ndarray) -> dict[tuple[int, int], dict[tuple[int, int], np.ndarray]]:
    out: dict[tuple[int, int], dict[tuple[int, int], np.ndarray]] = {}
    for r in raw:
        out.setdefault((int(r[0]), int(r[1])), {})[(int(r[12]), int(r[13]))] = r
    return out


def compare_raw(records, raw_oracle: np.ndarray, raw_ref: np.ndarray, tainted: set, conditioning=None) -> dict:
    """Checks one collision pass; adds pairs with band-only contacts to `tainted`.

    `conditioning(pair, feat, row)`, when given, bounds how far a contact's
    geometry may move under rounding of its inputs (ill-conditioned
    features); a contact that differs by more than GEOMETRY_TOL but within
    that bound taints its pair.  An infinite bound marks a feature chosen
    by a decision within rounding of its threshold: it may be present on
    one side only."""

    go, gr = group_raw(raw_oracle), group_raw(raw_ref)
    worst = 0.0
    matched = 0
    for pair in set(go) | set(gr):
        co, cr = go.get(pair, {}), gr.get(pair, {})
        dist = contact_distance(records, *pair)
        for feat in set(co) ^ set(cr):
            row = co.get(feat, cr.get(feat))
            one_sided_band = conditioning is not None and np.isinf(conditioning(pair, feat, row))
            assert one_sided_band or abs(row[5] - dist) <= ACCEPT_BAND, (pair, feat, row[5], dist)
            tainted.add(pair)
        for feat in set(co) & set(cr):
            # The support-point fallback of box-box (features 256 + axis)
            # picks one end of a supporting edge that lies exactly across
            # the normal, by the sign of a rounding-level dot product; its
            # normal and separation are well defined, its points are not.
            fallback = (feat[0] & 0x0FFFFFFF) >= 256
            cols = slice(2, 6) if fallback else slice(2, 12)
            d = float(np.max(np.abs(co[feat][cols] - cr[feat][cols])))
            if fallback and float(np.max(np.abs(co[feat][6:12] - cr[feat][6:12]))) > GEOMETRY_TOL:
                tainted.add(pair)  # the other end of the edge: anchors differ from here on
            if d > GEOMETRY_TOL and conditioning is not None:
                bound = conditioning(pair, feat, co[feat])
                assert d <= GEOMETRY_TOL + bound, (pair, feat, d, bound)
                tainted.add(pair)
                continue
            assert d <= GEOMETRY_TOL, (pair, feat, d)
            worst = max(worst, d)
            matched += 1
    return {"worst": worst, "matched": matched}


def compare_manifolds(table, manifolds_ref: np.ndarray, tainted: set) -> int:
    """Oracle SceneTable vs reference manifold rows (58 doubles each)."""

    ref = {int(m[0]) * 65 + int(m[1]): m for m in manifolds_ref}
    ours = {int(table.slots[i].key): table.slots[i].m for i in range(table.count.value)}
    skip = {a * 65 + b for a, b in tainted}
    checked = 0
    for key in (set(ref) | set(ours)) - skip:
        assert key in ref and key in ours, key
        m, r = ours[key], ref[key]
        assert m.count == int(r[2]), key
        np.testing.assert_allclose(list(m.normal_local), r[3:6], atol=GEOMETRY_TOL)
        assert float(m.age) == float(r[6]), key
        tangent = np.array(list(m.tangent_local))
        if m.age == 0.0:
            # A fresh manifold takes the stable tangent of its normal on both
            # sides.  A persisting one carries its tangent along with body A
            # on the device path (the GPU manifold builder) where the
            # reference's CPU collision re-derives the stable tangent, so
            # there only the frame's orthonormality is checked.
            np.testing.assert_allclose(tangent, r[7:10], atol=GEOMETRY_TOL)
        assert abs(float(np.dot(tangent, np.array(list(m.normal_local))))) <= 1e-6
        assert abs(float(np.linalg.norm(tangent)) - 1.0) <= 1e-6
        for p in range(m.count):
            pt, pr = m.points[p], r[10 + 12 * p: 22 + 12 * p]
            assert (pt.feature_a, pt.feature_b, pt.life) == (int(pr[9]), int(pr[10]), int(pr[11])), key
            np.testing.assert_allclose(list(pt.anchor_a) + list(pt.anchor_b), pr[0:6], atol=GEOMETRY_TOL)
        checked += 1
    return checked
