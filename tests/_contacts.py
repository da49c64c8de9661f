"""Comparison helpers for articulated contacts: the oracle's collision,
persistent manifolds and ConstraintIR rows (oracle_articulated_contacts)
against the reference's CPU world-step front end (collideCpuReference,
assembleContactConstraints, evaluateConstraintIR; ref_articulated_contacts
in oracle/ref_harness.cpp), live or from golden fixtures.

Row layout (both sides): shape a, shape b, feature A, feature B, separation,
normal xyz, point xyz, target velocity n/t/u, regularisation n/t/u,
effective mu, relative velocity n/t/u, new impact, then on the oracle side
the speculative approach term and on the reference side the pre-solve
normal velocity.

Known differences, handled here:
* the GPU semantics (MetalWorldContact.metal) add the speculative approach
  term -separation / h to a separated contact's normal target, the CPU
  adapter does not (ConstraintIR.cpp:2605-2632): the oracle's term is
  removed before the targets are compared;
* a persisting manifold carries its tangent with body A on the device path
  and the CPU re-derives it, so tangential rows are compared by their
  rotation-invariant magnitude;
* contacts within the acceptance pad of the summed offsets, and friction
  picked within rounding of the stiction transition, may differ (bands).
"""

from __future__ import annotations

import numpy as np

import _pile

GEOMETRY_TOL = 2e-6      # the reference publishes contacts in FP32
VELOCITY_TOL = 1e-5      # relative to max(1, |v|)
STICTION = 1e-3


def key(row: np.ndarray) -> tuple[int, int, int, int]:
    return int(row[0]), int(row[1]), int(row[2]), int(row[3])


def compare_manifolds(records, manifolds, manifolds_ref: np.ndarray, tainted: set) -> int:
    """Oracle OracleManifold[pair] vs reference manifold rows (58 doubles)."""

    ref = {(int(m[0]), int(m[1])): m for m in manifolds_ref}
    checked = 0
    for p in range(records.world.pair_count):
        pair = (int(records.pairs[p].shape_a), int(records.pairs[p].shape_b))
        if pair in tainted:
            continue
        m = manifolds[p]
        if m.count == 0:
            assert pair not in ref, pair
            continue
        assert pair in ref, pair
        r = ref[pair]
        assert m.count == int(r[2]), pair
        np.testing.assert_allclose(list(m.normal_local), r[3:6], atol=GEOMETRY_TOL)
        assert float(m.age) == float(r[6]), pair
        if m.age == 0.0:
            np.testing.assert_allclose(list(m.tangent_local), r[7:10], atol=GEOMETRY_TOL)
        for i in range(m.count):
            pt, pr = m.points[i], r[10 + 12 * i: 22 + 12 * i]
            assert (pt.feature_a, pt.feature_b, pt.life) == (int(pr[9]), int(pr[10]), int(pr[11])), pair
            np.testing.assert_allclose(list(pt.anchor_a) + list(pt.anchor_b), pr[0:6], atol=GEOMETRY_TOL)
        checked += 1
    return checked


def compare_rows(rows: np.ndarray, rows_ref: np.ndarray, tainted: set, h: float) -> dict:
    """ConstraintIR rows of untainted pairs, matched by (pair, features)."""

    ours = {key(r): r for r in rows if (int(r[0]), int(r[1])) not in tainted}
    ref = {key(r): r for r in rows_ref if (int(r[0]), int(r[1])) not in tainted}
    assert set(ours) == set(ref), (sorted(set(ours) ^ set(ref)))
    worst = {"geometry": 0.0, "target": 0.0, "velocity": 0.0}
    bands = 0
    for k, o in ours.items():
        r = ref[k]
        geo = max(abs(o[4] - r[4]), float(np.max(np.abs(o[5:11] - r[5:11]))))
        assert geo <= GEOMETRY_TOL, (k, geo)
        worst["geometry"] = max(worst["geometry"], geo)
        vs = max(1.0, float(np.max(np.abs(r[18:21]))))
        dn = abs(o[18] - r[18]) / vs
        dt = abs(np.hypot(o[19], o[20]) - np.hypot(r[19], r[20])) / vs
        assert dn <= VELOCITY_TOL and dt <= VELOCITY_TOL, (k, dn, dt)
        assert abs(o[18] - r[22]) <= VELOCITY_TOL * vs, (k, o[18], r[22])  # pre-solve normal velocity
        worst["velocity"] = max(worst["velocity"], dn, dt)
        assert int(o[21]) == int(r[21]), k  # new impact
        target = o[11] - o[22]  # without the speculative approach term
        dtar = abs(target - r[11]) / max(1.0, abs(r[11]))
        assert dtar <= VELOCITY_TOL and o[12] == 0.0 and o[13] == 0.0 and r[12] == 0.0 and r[13] == 0.0, (k, target, r[11])
        worst["target"] = max(worst["target"], dtar)
        np.testing.assert_allclose(o[14:17], r[14:17], rtol=1e-7, atol=1e-12)  # regularisation
        slip = np.hypot(r[19], r[20])
        if abs(slip - STICTION) <= 1e-5:
            bands += 1  # static or dynamic friction picked within rounding of the transition
        else:
            assert abs(o[17] - r[17]) <= 1e-6 * max(1.0, abs(r[17])), (k, o[17], r[17])
    return {"matched": len(ours), "worst": worst, "bands": bands}


def compare_step(records, raw, manifolds, rows, raw_ref, man_ref, rows_ref, tainted: set, h: float) -> dict:
    r = _pile.compare_raw(records, raw, raw_ref, tainted)
    checked = compare_manifolds(records, manifolds, man_ref, tainted)
    c = compare_rows(rows, rows_ref, tainted, h)
    return {"raw": r["matched"], "manifolds": checked, "rows": c["matched"], "worst": c["worst"], "bands": c["bands"]}
