"""Pins the oracle (oracle/oracle.c, FP64 C restatement) against the
reference's own FP64 CPU core compiled from its sources (oracle/_ref)."""

from __future__ import annotations

import numpy as np
import pytest

import numi_lab_b200 as nb
from oracle import Oracle, Reference

pytestmark = pytest.mark.reference

H = 0.005


def _models():
    for source in ("chain7", "tree29"):
        rec = nb.compile_model(source, 11)
        yield source, rec, Oracle(rec, H, 4 if source == "tree29" else 1, 8, 0), Reference(rec, H)


def _armature_f32(rec) -> np.ndarray:
    # The reference stores the implicit-drive armature a + h kd + h^2 kp in FP32.
    implicit = rec.world.actuation_mode == 1
    out = []
    for k in range(rec.world.nv):
        d = rec.dofs[k]
        a = float(d.drive[2])
        if implicit and (d.flags & (1 << 5)):
            a += H * float(d.drive[1]) + H * H * float(d.drive[0])
        out.append(np.float32(a))
    return np.array(out, np.float64)


def _states(source: str, rec, n: int, seed: int):
    rng = np.random.default_rng(seed)
    q, _, _ = nb.sample_reset(source, 11, seed, 0, n)
    for e in range(n):
        qe = q[e].astype(np.float64)
        if source == "tree29":
            qe[7:] += rng.uniform(-0.6, 0.6, size=qe[7:].shape)
        v = rng.normal(0.0, 1.0, size=rec.world.nv)
        tau = rng.normal(0.0, 5.0, size=rec.world.nv)
        if source == "tree29":
            tau[:6] = 0.0
        yield qe, v, tau


def test_aba_matches_reference_forward_dynamics(reference_available):
    for source, rec, oracle, ref in _models():
        for q, v, tau in _states(source, rec, 6, 1):
            so, a_o = oracle.aba(q, v, tau)
            sr, a_r = ref.forward_dynamics(q, v, tau)
            assert so == 0 and sr == 0
            rel = np.max(np.abs(a_o - a_r)) / max(1.0, np.max(np.abs(a_r)))
            assert rel < 1e-6, (source, rel)


def test_mass_matrix_matches_reference(reference_available):
    for source, rec, oracle, ref in _models():
        arm = _armature_f32(rec)
        for q, _, _ in _states(source, rec, 4, 2):
            m_o = oracle.mass_matrix(q) + np.diag(arm)
            m_r = ref.mass_matrix(q)
            assert np.max(np.abs(m_o - m_r)) < 1e-9 * max(1.0, np.max(np.abs(m_r))), source


def test_point_jacobians_match_reference(reference_available):
    rng = np.random.default_rng(5)
    for source, rec, oracle, ref in _models():
        nbodies = sum(1 for b in range(rec.world.body_count) if rec.bodies[b].articulated)
        for q, _, _ in _states(source, rec, 3, 3):
            for body in range(nbodies):
                local = rng.normal(0.0, 0.05, size=3)
                p_o, j_o = oracle.point_jacobian(q, body, local)
                p_r, j_r = ref.point_jacobian(q, body, local)
                np.testing.assert_allclose(p_o, p_r, atol=1e-12)
                np.testing.assert_allclose(j_o, j_r, atol=1e-12)


def test_free_motion_step_matches_reference_integrator(reference_available):
    rec = nb.compile_model("chain7", 11)
    oracle = Oracle(rec, H, 1, 0, 0)
    ref = Reference(rec, H)
    for q, v, tau in _states("chain7", rec, 8, 4):
        q_o, v_o = q.copy(), v.copy()
        st, _ = oracle.control_step(q_o, v_o, None, tau, 1.0)
        q_r, v_r = q.copy(), v.copy()
        sr = ref.integrate(q_r, v_r, tau)
        assert st == 0 and sr == 0
        np.testing.assert_allclose(v_o, v_r, rtol=0, atol=1e-10)
        np.testing.assert_allclose(q_o, q_r, rtol=0, atol=1e-12)


def test_cone_projection_known_answers():
    rec = nb.compile_model("tree29", 0)
    oracle = Oracle(rec, H, 4, 8, 0)
    np.testing.assert_allclose(oracle.project_cone([1.0, 0.2, -0.1], 0.5, 0.5), [1.0, 0.2, -0.1])
    np.testing.assert_allclose(oracle.project_cone([-1.0, 0.2, 0.3], 0.5, 0.5), [0.0, 0.0, 0.0])
    out = oracle.project_cone([2.0, 3.0, 4.0], 0.5, 0.5)  # |t| = 5 > mu n = 1
    np.testing.assert_allclose(out, [2.0, 0.6, 0.8])
    out = oracle.project_cone([1.0, 1.0, 1.0], 0.5, 0.25)  # elliptic, anisotropic
    assert abs((out[1] / 0.5) ** 2 + (out[2] / 0.25) ** 2 - 1.0) < 1e-12
    ok, inv = oracle.invert3x3(np.eye(3) * 4.0)
    assert ok
    np.testing.assert_allclose(inv, np.eye(3) / (4.0 * 1.01))
    ok, _ = oracle.invert3x3(np.zeros((3, 3)))
    assert not ok


def _foot_contact_problem(oracle: Oracle, rec, q, mu: float):
    """Four corner contacts under each foot of the 29-DoF tree."""

    rows = []
    foot_shapes = [s for s in range(rec.world.shape_count) if rec.shapes[s].shape_type == 2]
    n = np.array([0.0, 0.0, -1.0])  # robot (A) -> ground (B)
    t = np.array([1.0, 0.0, 0.0])
    b = np.cross(n, t)
    for s in foot_shapes:
        sh = rec.shapes[s]
        hx, hy, hz = sh.dimensions[0], sh.dimensions[1], sh.dimensions[2]
        for sx in (-1, 1):
            for sy in (-1, 1):
                local = np.array(sh.local_position[:3]) + np.array([sx * hx, sy * hy, -hz])
                _, J = oracle.point_jacobian(q, sh.body, local)
                for d in (n, t, b):
                    rows.append(-(d @ J))
    G = np.array(rows)
    M = oracle.mass_matrix(q) + np.diag(_armature_f32(rec))
    Minv = np.linalg.inv(M)
    return G, M, Minv, np.full(len(rows) // 3, mu)


def test_temporal_cone_iteration_approaches_converged_conic_solution(reference_available):
    rec = nb.compile_model("tree29", 11)
    oracle = Oracle(rec, H, 4, 8, 0)
    ref = Reference(rec, H)
    q, _, _ = nb.sample_reset("tree29", 11, 0, 0, 1)
    q = q[0].astype(np.float64)
    G, M, Minv, mu = _foot_contact_problem(oracle, rec, q, 0.8)
    rng = np.random.default_rng(7)
    v_free = rng.normal(0.0, 0.1, size=rec.world.nv)
    v_free[2] = -0.5  # falling into the ground
    # The reference's composed path requires a positive regularization floor
    # for redundant contact patches (ArticulatedWorld.hpp, 1e-6).
    reg = np.full(G.shape[0], 1.0e-6)
    Minv = 0.5 * (Minv + Minv.T)
    W = G @ Minv @ G.T + np.diag(reg)
    u0 = G @ v_free
    lam_tc = oracle.temporal_cone_dense(W, u0, mu, 4000)
    st, lam_ref, vel_ref, viol = ref.conic_solve(Minv, v_free, G, mu, np.zeros(G.shape[0]), reg)
    assert st == 0 and viol < 1e-8
    # exact cone feasibility of the temporal-cone iterate
    for i in range(len(mu)):
        ln, lt = lam_tc[3 * i], np.hypot(lam_tc[3 * i + 1], lam_tc[3 * i + 2])
        assert ln >= 0.0 and lt <= mu[i] * ln * (1 + 1e-12) + 1e-15
    obj = lambda lam: 0.5 * lam @ W @ lam + u0 @ lam  # noqa: E731
    # The block-Jacobi fixed point with the Euclidean cone projection reaches
    # the converged conic optimum to within 1e-4 in objective and 1e-3 in the
    # total normal impulse on this two-foot patch.
    assert obj(lam_tc) <= obj(lam_ref) + 1e-4 * abs(obj(lam_ref))
    assert abs(lam_tc[0::3].sum() - lam_ref[0::3].sum()) <= 1e-3 * lam_ref[0::3].sum()
    # post-impulse velocity: the reference applies M^-1 G^T lambda
    np.testing.assert_allclose(v_free + Minv @ G.T @ lam_ref, vel_ref, atol=1e-9)


def test_reference_contact_world_steps_the_tree(reference_available):
    rec = nb.compile_model("tree29", 11)
    ref = Reference(rec, H, friction=0.7)
    q, v, _ = nb.sample_reset("tree29", 11, 0, 0, 2)
    q = q.astype(np.float64)
    v = v.astype(np.float64)
    actions = np.random.default_rng(0).normal(0, 0.3, size=(3, 2, 29)).astype(np.float32)
    secs, failed = ref.run(q, v, actions, 4, 2)
    assert failed == 0 and secs > 0.0
    assert np.all(np.isfinite(q))
