"""The oracle's articulated contact front end -- box-foot and sphere-proxy
collision against the plane, persistent manifolds and ConstraintIR rows --
and its island partitions, against the reference's own CPU code:
collideCpuReference (src/core/Collision.cpp:2959), assembleContactConstraints
(src/core/RigidBodyWorld.cpp:564), evaluateConstraintIR
(src/core/ConstraintIR.cpp:1414) and buildConstraintIslands
(src/core/ConstraintSolver.cpp:848), live where the reference core is built
and from the golden fixture tests/golden/contact_pins.npz
(tests/golden/make_contact_golden.py) everywhere.  CPU only."""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

import numi_lab_b200 as nb
from oracle import Oracle, SceneOracle, SceneTable

import _contacts

GOLDEN = Path(__file__).resolve().parent / "golden" / "contact_pins.npz"
H = 0.005
TREE_SEED = 2026      # the contact benchmark's world


def tree_trajectory(envs: int, steps: int, seed: int = TREE_SEED):
    """Seeded FP64 oracle trajectories of the tree29 contact world: per env,
    (q, v) after each control step, with PD targets ~ N(0, 0.3)."""

    rec = nb.compile_model("tree29", seed)
    oracle = Oracle(rec, H, 4, 8, 0)
    q0, v0, fr = nb.sample_reset("tree29", seed, seed, 0, envs)
    rng = np.random.default_rng(seed)
    out = []
    for e in range(envs):
        q, v = q0[e].astype(np.float64), v0[e].astype(np.float64)
        man = oracle.new_manifolds()
        states = []
        for _ in range(steps):
            st, _ = oracle.control_step(q, v, man, rng.normal(0.0, 0.3, 29), float(fr[e]))
            assert st == 0
            states.append((q.copy(), v.copy()))
        out.append(states)
    return rec, fr, out


@pytest.mark.reference
def test_tree_contacts_match_reference_live(reference_available):
    from oracle import Reference

    envs, steps = 6, 40
    rec, fr, traj = tree_trajectory(envs, steps)
    oracle = Oracle(rec, H, 4, 8, 0)
    totals = {"raw": 0, "manifolds": 0, "rows": 0, "bands": 0}
    tainted_pairs = 0
    for e in range(envs):
        ref = Reference(rec, H, float(fr[e]))
        cache = ref.contact_cache()
        man = oracle.new_manifolds()
        tainted: set = set()
        for q, v in traj[e]:
            s1, raw, rows = oracle.articulated_contacts(q, v, man, float(fr[e]))
            s2, raw_ref, man_ref, rows_ref = ref.articulated_contacts(cache, q, v)
            assert s1 == 0 and s2 == 0
            r = _contacts.compare_step(rec, raw, man, rows, raw_ref, man_ref, rows_ref, tainted, H)
            for k in totals:
                totals[k] += r[k]
        tainted_pairs += len(tainted)
    print(f"tree29 contact pin: {totals}, tainted pairs {tainted_pairs}")
    assert totals["rows"] > 300 and totals["manifolds"] > 200
    assert tainted_pairs <= 2
    assert totals["bands"] <= totals["rows"] // 20


def test_tree_contacts_match_reference_golden():
    if not GOLDEN.is_file():
        pytest.skip("golden fixture missing")
    g = np.load(GOLDEN)
    rec = nb.compile_model("tree29", TREE_SEED)
    fp = np.frombuffer(bytes(rec.bodies) + bytes(rec.shapes) + bytes(rec.pairs), np.uint8)
    assert np.array_equal(fp, g["tree_fingerprint"]), "tree29 model drifted from the fixture"
    oracle = Oracle(rec, H, 4, 8, 0)
    fr = g["tree_friction"]
    raw_at = np.concatenate([[0], np.cumsum(g["tree_raw_rows"])])
    man_at = np.concatenate([[0], np.cumsum(g["tree_manifold_rows"])])
    row_at = np.concatenate([[0], np.cumsum(g["tree_contact_rows"])])
    q_all, v_all = g["tree_q"], g["tree_v"]
    envs, steps = q_all.shape[:2]
    rows_total = 0
    for e in range(envs):
        man = oracle.new_manifolds()
        tainted: set = set()
        for k in range(steps):
            i = e * steps + k
            s1, raw, rows = oracle.articulated_contacts(q_all[e, k], v_all[e, k], man, float(fr[e]))
            assert s1 == 0
            r = _contacts.compare_step(rec, raw, man, rows, g["tree_raw"][raw_at[i]:raw_at[i + 1]],
                                       g["tree_manifolds"][man_at[i]:man_at[i + 1]],
                                       g["tree_contacts"][row_at[i]:row_at[i + 1]], tainted, H)
            rows_total += r["rows"]
        assert len(tainted) <= 1
    assert rows_total > 100


def pile_island_cases(seed: int, steps: int):
    """(island_of, contact pairs, nb) of the oracle's final substeps over a
    settling pile."""

    rec = nb.compile_model("pile", seed)
    oracle = SceneOracle(rec, H, 4, 8, 0)
    q, v, f = nb.sample_reset("pile", seed, 1, 0, 1)
    q, v = q[0].astype(np.float64), v[0].astype(np.float64)
    table = SceneTable()
    nbod = rec.world.body_count - 1
    cases = []
    for _ in range(steps):
        status, trace = oracle.step(q, v, table, float(f[0]))
        assert status == 0
        n = int(trace.island_contacts)
        pairs = np.array(trace.island_pairs[: 2 * n], np.int64).reshape(n, 2)
        cases.append((np.array(trace.island_of[:nbod], np.uint32), pairs, int(trace.islands)))
    return nbod, cases


def _reference_partition(nbod: int, pairs: np.ndarray):
    from oracle import reference_islands

    dyn = np.ones(nbod + 1, np.uint8)
    dyn[nbod] = 0  # the plane: a static body
    p = pairs.copy()
    p[p < 0] = nbod
    count, island = reference_islands(dyn, p)
    return count, island[:nbod]


@pytest.mark.reference
@pytest.mark.parametrize("seed", [1, 6, 13, 17])
def test_pile_islands_match_reference_live(reference_available, seed):
    nbod, cases = pile_island_cases(seed, 60)
    multi = 0
    for island_of, pairs, count in cases:
        if len(pairs) == 0:
            continue
        ref_count, ref_island = _reference_partition(nbod, pairs)
        assert ref_count == count
        assert np.array_equal(island_of, ref_island)
        multi += count > 1
    assert multi > 0  # partitions with several islands were compared


def test_pile_islands_match_reference_golden():
    if not GOLDEN.is_file():
        pytest.skip("golden fixture missing")
    g = np.load(GOLDEN)
    for seed in (6, 13):
        p = f"pile{seed}_"
        nbod, cases = pile_island_cases(seed, int(g[p + "steps"]))
        at = np.concatenate([[0], np.cumsum(g[p + "pair_rows"])])
        for k, (island_of, pairs, count) in enumerate(cases):
            assert np.array_equal(pairs, g[p + "pairs"][at[k]:at[k + 1]])
            assert count == int(g[p + "count"][k])
            assert np.array_equal(island_of, g[p + "island_of"][k])
