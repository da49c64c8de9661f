"""Generates tests/golden/reference_core.npz from the reference's own FP64
CPU core (compiled from its sources into oracle/_ref by oracle/Makefile).

The fixture holds, for the seeded synthetic chain-7 and 29-DoF tree worlds:
forward dynamics (computeArticulatedForwardDynamics), mass matrices
(computeArticulatedMassMatrix), point Jacobians
(computeArticulatedPointJacobians), a free-motion step
(integrateArticulatedState) and a converged conic contact solve
(solveReferenceConicProblem) on a two-foot contact patch.
tests/test_golden.py checks the oracle against it.

Run from the repository root:  python tests/golden/make_golden.py
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

import numi_lab_b200 as nb  # noqa: E402
from oracle import Oracle, Reference  # noqa: E402

MODEL_SEED = 11
H = 0.005
OUT = Path(__file__).resolve().parent / "reference_core.npz"


def states(source: str, nv: int, n: int, seed: int):
    rng = np.random.default_rng(seed)
    q, _, _ = nb.sample_reset(source, MODEL_SEED, seed, 0, n)
    qs, vs, taus = [], [], []
    for e in range(n):
        qe = q[e].astype(np.float64)
        if source == "tree29":
            qe[7:] += rng.uniform(-0.6, 0.6, size=qe[7:].shape)
        v = rng.normal(0.0, 1.0, size=nv)
        tau = rng.normal(0.0, 5.0, size=nv)
        if source == "tree29":
            tau[:6] = 0.0
        qs.append(qe)
        vs.append(v)
        taus.append(tau)
    return np.array(qs), np.array(vs), np.array(taus)


def main() -> None:
    data: dict[str, np.ndarray] = {}
    for source in ("chain7", "tree29"):
        rec = nb.compile_model(source, MODEL_SEED)
        ref = Reference(rec, H)
        nv = rec.world.nv
        q, v, tau = states(source, nv, 6, 3)
        qdd = np.array([ref.forward_dynamics(q[i], v[i], tau[i])[1] for i in range(len(q))])
        mass = np.array([ref.mass_matrix(q[i]) for i in range(len(q))])
        rng = np.random.default_rng(4)
        nbody = sum(1 for b in range(rec.world.body_count) if rec.bodies[b].articulated)
        bodies = rng.integers(0, nbody, size=8)
        locals_ = rng.normal(0.0, 0.05, size=(8, 3))
        jac = np.array([ref.point_jacobian(q[0], int(b), locals_[i])[1] for i, b in enumerate(bodies)])
        prefix = f"{source}_"
        data[prefix + "fingerprint"] = np.frombuffer(bytes(rec.bodies) + bytes(rec.joints) + bytes(rec.dofs), np.uint8)
        data[prefix + "q"] = q
        data[prefix + "v"] = v
        data[prefix + "tau"] = tau
        data[prefix + "qdd"] = qdd
        data[prefix + "mass"] = mass
        data[prefix + "jac_bodies"] = bodies
        data[prefix + "jac_locals"] = locals_
        data[prefix + "jac"] = jac
        if source == "chain7":
            q1, v1 = q.copy(), v.copy()
            for i in range(len(q)):
                ref.integrate(q1[i], v1[i], tau[i])
            data[prefix + "step_q"] = q1
            data[prefix + "step_v"] = v1
        else:
            from test_oracle_pin import _foot_contact_problem

            oracle = Oracle(rec, H, 4, 8, 0)
            q0 = q[0].copy()
            q0[7:] = nb.sample_reset(source, MODEL_SEED, 0, 0, 1)[0][0][7:]
            G, _, Minv, mu = _foot_contact_problem(oracle, rec, q0, 0.8)
            Minv = 0.5 * (Minv + Minv.T)
            v_free = np.random.default_rng(7).normal(0.0, 0.1, size=nv)
            v_free[2] = -0.5
            reg = np.full(G.shape[0], 1.0e-6)
            st, lam, vel, viol = ref.conic_solve(Minv, v_free, G, mu, np.zeros(G.shape[0]), reg)
            assert st == 0
            data["conic_q"] = q0
            data["conic_v_free"] = v_free
            data["conic_mu"] = mu
            data["conic_lambda"] = lam
            data["conic_velocity"] = vel
    np.savez_compressed(OUT, **data)
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes)")


if __name__ == "__main__":
    main()
