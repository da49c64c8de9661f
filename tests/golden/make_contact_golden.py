"""Generates tests/golden/contact_pins.npz from the reference's own FP64 CPU
core (oracle/_ref, built by oracle/Makefile from the reference's sources):

* tree29 (model seed 2026): for 3 environments x 30 control steps of a
  seeded FP64 oracle trajectory, the reference CPU world step's raw
  contacts, persistent manifolds and evaluated ConstraintIR contact rows
  (ref_articulated_contacts: collideCpuReference, assembleContactConstraints,
  evaluateConstraintIR) at each (q, v);
* piles (seeds 6, 13): the island partition buildConstraintIslands gives to
  the oracle's final-substep contact set over 40 control steps.

tests/test_contact_pin.py checks the oracle against it.

Run from the repository root:  python tests/golden/make_contact_golden.py
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

from oracle import Reference  # noqa: E402

import test_contact_pin as pin  # noqa: E402

OUT = Path(__file__).resolve().parent / "contact_pins.npz"


def main() -> None:
    data: dict[str, np.ndarray] = {}
    envs, steps = 3, 30
    rec, fr, traj = pin.tree_trajectory(envs, steps)
    data["tree_fingerprint"] = np.frombuffer(bytes(rec.bodies) + bytes(rec.shapes) + bytes(rec.pairs), np.uint8)
    data["tree_friction"] = fr[:envs]
    data["tree_q"] = np.array([[q for q, _ in traj[e]] for e in range(envs)])
    data["tree_v"] = np.array([[v for _, v in traj[e]] for e in range(envs)])
    raws, mans, rows, nr, nm, nc = [], [], [], [], [], []
    for e in range(envs):
        ref = Reference(rec, pin.H, float(fr[e]))
        cache = ref.contact_cache()
        for q, v in traj[e]:
            st, raw, man, row = ref.articulated_contacts(cache, q, v)
            assert st == 0
            raws.append(raw), mans.append(man), rows.append(row)
            nr.append(len(raw)), nm.append(len(man)), nc.append(len(row))
    data["tree_raw"] = np.concatenate(raws)
    data["tree_manifolds"] = np.concatenate(mans)
    data["tree_contacts"] = np.concatenate(rows)
    data["tree_raw_rows"] = np.array(nr)
    data["tree_manifold_rows"] = np.array(nm)
    data["tree_contact_rows"] = np.array(nc)
    for seed in (6, 13):
        nbod, cases = pin.pile_island_cases(seed, 40)
        p = f"pile{seed}_"
        pairs, counts, island_of, rows_ = [], [], [], []
        for _, pr, _ in cases:
            n, isl = pin._reference_partition(nbod, pr) if len(pr) else (0, np.full(nbod, 0xFFFFFFFF, np.uint32))
            pairs.append(pr), counts.append(n), island_of.append(isl), rows_.append(len(pr))
        data[p + "steps"] = np.array(40)
        data[p + "pairs"] = np.concatenate(pairs) if pairs else np.zeros((0, 2), np.int64)
        data[p + "pair_rows"] = np.array(rows_)
        data[p + "count"] = np.array(counts)
        data[p + "island_of"] = np.array(island_of, np.uint32)
    np.savez_compressed(OUT, **data)
    print(OUT, OUT.stat().st_size)


if __name__ == "__main__":
    main()
