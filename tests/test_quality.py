"""Converged (quality) contact solve on the CPU: the oracle's FP64
restatement (oracle_quality_solve, oracle/oracle.c) against the reference's
own solveQualityContactProblem (src/core/QualityContactSolver.cpp:1480),
through the committed golden outputs (tests/golden/quality_pins.npz, made
by tests/golden/make_quality_golden.py) and, where the reference core is
built, live on fresh problems.  The problem is strongly convex (every row
has a positive regularisation), so both solvers converge to the same unique
impulses; independent KKT certificates (tests/_quality.py) show which
answer is right where the reference stops short of convergence.  Also the
C ABI's argument checks of mr_quality_solve_batch (no device work).
"""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

import _quality as Q
import numi_lab_b200 as nb
from oracle import Oracle, quality_config, quality_dense

GOLDEN = Path(__file__).resolve().parent / "golden" / "quality_pins.npz"
# Oracle vs reference impulses and velocities, relative to max(1, |x|):
# the two converge (tolerances 1e-9 and 1e-11) to the same minimiser.
MATCH_TOL = 1.0e-7
# KKT certificates of a converged oracle answer (scaled, tests/_quality.py).
CERT_TOL = 1.0e-8


def _rel(a: np.ndarray, b: np.ndarray) -> float:
    return float(np.max(np.abs(a - b)) / max(1.0, float(np.max(np.abs(b))))) if a.size else 0.0


def golden_problems():
    d = np.load(GOLDEN)
    for p in range(len(d["nv"])):
        nv, nc = int(d["nv"][p]), int(d["nc"][p])
        yield p, d, (d["mass"][p, :nv, :nv], d["jacobian"][p, :3 * nc, :nv], d["free_velocity"][p, :nv],
                     d["target"][p, :3 * nc], d["regularization"][p, :3 * nc], d["friction"][p, :nc])


def test_oracle_quality_solve_matches_the_reference_solutions():
    matched = 0
    for p, d, prob in golden_problems():
        st, lam, vel, out = quality_dense(*prob)
        assert st == 0, (p, out.newton, out.residual)
        cert = Q.certificates(*prob, lam)
        assert max(cert.values()) <= CERT_TOL, (p, cert)
        assert out.cone <= 1e-12
        if d["ref_status"][p] != 0:
            continue
        nv, nc = prob[0].shape[0], len(prob[5])
        assert _rel(lam, d["ref_impulses"][p, :3 * nc]) <= MATCH_TOL, p
        assert _rel(vel, d["ref_velocity"][p, :nv]) <= MATCH_TOL, p
        matched += 1
    assert matched >= 24


def test_oracle_certifies_problems_the_reference_leaves_unconverged():
    """On degenerate problems (more contact rows than DoFs, nv 4-6) the
    reference stops at its 200-iteration budget (MR_STEP_DID_NOT_CONVERGE)
    with a natural residual of 1e-6..1e-5; the oracle converges, and its
    answer satisfies the KKT conditions to rounding."""

    unconverged = 0
    for p, d, prob in golden_problems():
        if d["ref_status"][p] == 0:
            continue
        unconverged += 1
        st, lam, _, _ = quality_dense(*prob)
        assert st == 0
        assert max(Q.certificates(*prob, lam).values()) <= CERT_TOL
        ref_cert = Q.certificates(*prob, d["ref_impulses"][p, :3 * len(prob[5])])
        assert ref_cert["natural_residual"] > 10 * CERT_TOL
    assert unconverged >= 1


def test_oracle_quality_solve_is_insensitive_to_the_warm_start():
    rng = np.random.default_rng(4)
    for p, _, prob in golden_problems():
        if p % 4:
            continue
        st0, lam0, _, _ = quality_dense(*prob)
        warm = lam0 + rng.normal(0.0, 0.1, size=lam0.shape) * max(1.0, float(np.max(np.abs(lam0))))
        st1, lam1, _, out = quality_dense(*prob, warm=warm)
        assert st0 == 0 and st1 == 0
        assert _rel(lam1, lam0) <= MATCH_TOL


@pytest.mark.reference
def test_oracle_quality_solve_matches_the_live_reference(reference_available):
    from oracle import reference_quality_solve

    rng = np.random.default_rng(99)
    rec = nb.compile_model("tree29", 11)
    oracle = Oracle(rec, 0.005, 4, 8, 0)
    q, _, _ = nb.sample_reset("tree29", 11, 17, 0, 6)
    probs = [Q.tree29_patch(oracle, rec, q[e].astype(np.float64), rng, 0.005, spheres=int(rng.integers(0, 13))) for e in range(6)]
    probs += [Q.random_problem(rng, int(rng.integers(8, 37)), int(rng.integers(1, 16))) for _ in range(6)]
    compared = 0
    for prob in probs:
        M, G, vf, target, reg, mu = prob
        Minv = np.linalg.inv(M)
        rst, rlam, rvel, _ = reference_quality_solve(0.5 * (Minv + Minv.T), vf, G, mu, target, reg)
        st, lam, vel, _ = quality_dense(*prob)
        assert st == 0
        assert max(Q.certificates(*prob, lam).values()) <= CERT_TOL
        if rst == 0:
            assert _rel(lam, rlam) <= MATCH_TOL
            assert _rel(vel, rvel) <= MATCH_TOL
            compared += 1
    assert compared >= 8


def test_oracle_world_steps_tree29_with_the_quality_solve():
    """The oracle's control step with converged contact solves: every step
    of a seeded 30-step rollout succeeds, with feasible impulses."""

    rec = nb.compile_model("tree29", 5)
    oracle_q = Oracle(rec, 0.005, 4, 8, 0)
    oracle_q.set_quality(quality_config())
    q0, v0, fr = nb.sample_reset("tree29", 5, 3, 0, 2)
    rng = np.random.default_rng(1)
    contacts = 0
    for e in range(2):
        q, v = q0[e].astype(np.float64), v0[e].astype(np.float64)
        man = oracle_q.new_manifolds()
        for _ in range(30):
            st, trace = oracle_q.control_step(q, v, man, rng.normal(0.0, 0.3, rec.world.action_count), float(fr[e]))
            assert st == 0
            assert trace.max_cone_violation <= 1e-9
            contacts += int(trace.contact_count)
    assert contacts > 0


def test_quality_solve_batch_rejects_malformed_problems():
    """Host-side argument checks of mr_quality_solve_batch (before any
    device work)."""

    rng = np.random.default_rng(0)
    M, G, vf, target, reg, mu = Q.random_problem(rng, 6, 3)
    args = (M[None], G[None], vf[None], target[None], reg[None], mu[None])
    bad_reg = reg.copy()
    bad_reg[4] = 1e-3  # contact 1: tangent 1e-3, bitangent 1e-6
    with pytest.raises(nb.MetalRoboError, match="tangent"):
        nb.quality_solve(M[None], G[None], vf[None], target[None], bad_reg[None], mu[None])
    with pytest.raises(nb.MetalRoboError, match="non-negative"):
        nb.quality_solve(*args[:5], -mu[None])
    with pytest.raises(nb.MetalRoboError, match="finite"):
        nb.quality_solve(M[None] * np.nan, *args[1:])
    with pytest.raises(nb.MetalRoboError, match="nv"):
        nb.quality_solve(np.eye(65)[None], np.zeros((1, 9, 65)), np.zeros((1, 65)), target[None], reg[None], mu[None])
    with pytest.raises(nb.MetalRoboError, match="contact_counts"):
        nb.quality_solve(*args, counts=np.array([4]))
