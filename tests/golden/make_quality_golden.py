"""Generates tests/golden/quality_pins.npz from the reference's own FP64 CPU
core (oracle/_ref, built by oracle/Makefile from the reference's sources):
the converged contact solves of solveQualityContactProblem
(src/core/QualityContactSolver.cpp:1480, default configuration) on

* 16 contact patches of the 29-DoF tree (model seed 11, reset seed 5):
  the eight box-foot corners plus 0-12 sphere proxies, the joint-space
  inertia with the implicit-drive armature, seeded free velocities,
  targets, regularisation (1e-6 floor) and friction;
* 12 dense problems with random SPD inertia (nv 4-36, 1-19 contacts).

Problems are zero-padded to 35 DoFs x 20 contacts; `nv` and `nc` give the
used sizes.  tests/test_quality.py checks the oracle against the reference
outputs and tests/test_quality_gpu.py the library.

Run from the repository root:  python tests/golden/make_quality_golden.py
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

import numi_lab_b200 as nb  # noqa: E402
from oracle import Oracle, reference_quality_solve  # noqa: E402

import _quality  # noqa: E402

OUT = Path(__file__).resolve().parent / "quality_pins.npz"
H = 0.005
NV, NC = 36, 20


def problems():
    rng = np.random.default_rng(2026)
    rec = nb.compile_model("tree29", 11)
    oracle = Oracle(rec, H, 4, 8, 0)
    q, _, _ = nb.sample_reset("tree29", 11, 5, 0, 16)
    for e in range(16):
        yield "tree29", _quality.tree29_patch(oracle, rec, q[e].astype(np.float64), rng, H, spheres=int(rng.integers(0, 13)))
    for _ in range(12):
        yield "random", _quality.random_problem(rng, int(rng.integers(4, 37)), int(rng.integers(1, 20)))


def main() -> None:
    rows = []
    for kind, (M, G, vf, target, reg, mu) in problems():
        nv, nc = M.shape[0], len(mu)
        Minv = np.linalg.inv(M)
        st, lam, vel, cert = reference_quality_solve(0.5 * (Minv + Minv.T), vf, G, mu, target, reg)
        rows.append((kind, M, G, vf, target, reg, mu, st, lam, vel, cert))
    P = len(rows)
    data = {
        "kind": np.array([r[0] == "tree29" for r in rows]),
        "nv": np.array([r[1].shape[0] for r in rows], np.int32),
        "nc": np.array([len(r[6]) for r in rows], np.int32),
        "mass": np.zeros((P, NV, NV)),
        "jacobian": np.zeros((P, 3 * NC, NV)),
        "free_velocity": np.zeros((P, NV)),
        "target": np.zeros((P, 3 * NC)),
        "regularization": np.full((P, 3 * NC), _quality.FLOOR),
        "friction": np.zeros((P, NC)),
        "ref_status": np.array([r[7] for r in rows], np.int32),
        "ref_impulses": np.zeros((P, 3 * NC)),
        "ref_velocity": np.zeros((P, NV)),
        "ref_kkt": np.array([r[10]["kkt"] for r in rows]),
        "ref_iterations": np.array([r[10]["iterations"] for r in rows], np.int32),
    }
    for p, (_, M, G, vf, target, reg, mu, st, lam, vel, cert) in enumerate(rows):
        nv, nc = M.shape[0], len(mu)
        data["mass"][p, :nv, :nv] = M
        data["jacobian"][p, :3 * nc, :nv] = G
        data["free_velocity"][p, :nv] = vf
        data["target"][p, :3 * nc] = target
        data["regularization"][p, :3 * nc] = reg
        data["friction"][p, :nc] = mu
        data["ref_impulses"][p, :3 * nc] = lam
        data["ref_velocity"][p, :nv] = vel
    np.savez_compressed(OUT, **data)
    print(OUT, P, "problems;", int((data["ref_status"] == 0).sum()), "converged in the reference")


if __name__ == "__main__":
    main()
