"""Generates tests/golden/pile_collision.npz from the reference's own FP64
CPU collision (collideCpuReference, src/core/Collision.cpp:2959, compiled
from its sources into oracle/_ref by oracle/Makefile).

For three seeded synthetic piles (10, 17 and 61 bodies on a plane), and
two piles with cylinders (keys cylinder_seed*), the
fixture holds a run of consecutive body configurations -- taken from the
oracle's own simulation of the pile settling, so that boxes and spheres
rest on the plane and on each other -- and, for each configuration in
order, the reference's raw contacts and persistent manifolds (its cache
carried from one configuration to the next, starting empty).
tests/test_pile_oracle.py replays the configurations through the oracle.

Run from the repository root:  python tests/golden/make_pile_golden.py
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import numi_lab_b200 as nb  # noqa: E402
from oracle import ReferenceScene, SceneOracle, SceneTable  # noqa: E402

SEEDS = (3, 13, 14)
# Piles with cylinders ("cylinder_pile"): the reference's CPU collision
# handles cylinder on the plane and skips cylinder-finite pairs.
CYLINDER_SEEDS = (5, 11)
FIRST, COUNT = 30, 8
OUT = Path(__file__).resolve().parent / "pile_collision.npz"


def main() -> None:
    data: dict[str, np.ndarray] = {}
    for source, seed in [("pile", s) for s in SEEDS] + [("cylinder_pile", s) for s in CYLINDER_SEEDS]:
        rec = nb.compile_model(source, seed)
        oracle = SceneOracle(rec, 0.005, 4, 8, 0)
        q, v, f = nb.sample_reset(source, seed, 1, 0, 1)
        q = q[0].astype(np.float64)
        v = v[0].astype(np.float64)
        table = SceneTable()
        ref = ReferenceScene(rec)
        qs, raws, mans = [], [], []
        for k in range(FIRST + COUNT):
            status, _ = oracle.step(q, v, table, float(f[0]))
            assert status == 0
            if k >= FIRST:
                st, raw, man = ref.collide(q)
                assert st == 0
                qs.append(q.copy())
                raws.append(raw)
                mans.append(man)
        p = f"seed{seed}_" if source == "pile" else f"cylinder_seed{seed}_"
        data[p + "q"] = np.array(qs)
        data[p + "raw_rows"] = np.array([len(r) for r in raws])
        data[p + "raw"] = np.concatenate(raws)
        data[p + "manifold_rows"] = np.array([len(m) for m in mans])
        data[p + "manifolds"] = np.concatenate(mans)
        data[p + "fingerprint"] = np.frombuffer(bytes(rec.bodies) + bytes(rec.shapes), np.uint8)
    np.savez_compressed(OUT, **data)
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes)")


if __name__ == "__main__":
    main()
