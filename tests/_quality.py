"""Contact problems and certificates for the converged (quality) solve tests.

A problem is the input of mr_quality_solve_batch for one problem:
mass H [nv, nv], Jacobian G [3 n, nv] (rows normal, tangent, bitangent per
contact, A -> B convention), free velocity, target velocity [3 n],
regularisation [3 n] (the 1e-6 floor already applied, so every solver sees
the same numbers) and friction [n].  The reference's solver takes H^-1
(DenseConicProblem.inverseMass, ReferenceConicSolver.hpp:35-41).
"""

from __future__ import annotations

import numpy as np

FLOOR = 1.0e-6  # ArticulatedWorld.hpp:58 minimumRegularization


def armature_f32(rec, h: float) -> np.ndarray:
    """Effective armature a + h kd + h^2 kp of implicit drives, in FP32 like the reference."""

    implicit = rec.world.actuation_mode == 1
    out = []
    for k in range(rec.world.nv):
        d = rec.dofs[k]
        a = float(d.drive[2])
        if implicit and (d.flags & (1 << 5)):
            a += h * float(d.drive[1]) + h * h * float(d.drive[0])
        out.append(np.float32(a))
    return np.array(out, np.float64)


def tree29_patch(oracle, rec, q: np.ndarray, rng: np.random.Generator, h: float, spheres: int):
    """Box-foot corner contacts (4 per foot) plus `spheres` sphere-proxy
    contacts of the 29-DoF tree at configuration q, each with its own
    tangent frame about the ground normal."""

    points = []
    for s in range(rec.world.shape_count):
        sh = rec.shapes[s]
        if sh.shape_type == 2:  # box foot: its four bottom corners
            hx, hy, hz = sh.dimensions[0], sh.dimensions[1], sh.dimensions[2]
            for sx in (-1, 1):
                for sy in (-1, 1):
                    points.append((sh.body, np.array(sh.local_position[:3]) + np.array([sx * hx, sy * hy, -hz])))
    sphere_shapes = [s for s in range(rec.world.shape_count) if rec.shapes[s].shape_type == 0]
    for s in rng.choice(sphere_shapes, size=min(spheres, len(sphere_shapes)), replace=False):
        sh = rec.shapes[int(s)]
        points.append((sh.body, np.array(sh.local_position[:3], np.float64)))
    n = np.array([0.0, 0.0, -1.0])
    rows = []
    for body, local in points:
        _, J = oracle.point_jacobian(q, body, local)
        a = rng.uniform(0.0, 2.0 * np.pi)
        t = np.array([np.cos(a), np.sin(a), 0.0])
        b = np.cross(n, t)
        for d in (n, t, b):
            rows.append(-(d @ J))
    G = np.array(rows)
    M = oracle.mass_matrix(q) + np.diag(armature_f32(rec, h))
    M = 0.5 * (M + M.T)
    nc = len(points)
    nv = M.shape[0]
    vf = rng.normal(0.0, 0.2, size=nv)
    vf[2] = -rng.uniform(0.1, 0.6)  # falling into the ground
    target = np.zeros(3 * nc)
    target[0::3] = rng.uniform(0.0, 0.05, nc)  # stabilisation / restitution terms
    reg = np.zeros(3 * nc)
    reg[0::3] = rng.choice([0.0, 1.0e-4, 1.0e-3], size=nc)
    reg = np.maximum(reg, FLOOR)
    mu = rng.uniform(0.3, 1.1, nc)
    return M, G, vf, target, reg, mu


def random_problem(rng: np.random.Generator, nv: int, nc: int):
    """A dense problem with a random SPD mass matrix and Jacobian; contact 0
    is frictionless."""

    A = rng.normal(size=(nv, nv))
    M = A @ A.T + nv * np.eye(nv)
    G = rng.normal(size=(3 * nc, nv))
    vf = rng.normal(size=nv)
    target = np.zeros(3 * nc)
    target[0::3] = rng.uniform(0.0, 0.3, nc)
    reg = np.full(3 * nc, FLOOR)
    reg[0::3] = rng.uniform(FLOOR, 1.0e-3, nc)
    mu = rng.uniform(0.2, 1.0, nc)
    mu[0] = 0.0
    return M, G, vf, target, reg, mu


def project_cone(x: np.ndarray, mu: float) -> np.ndarray:
    """Euclidean projection onto {||l_t|| <= mu l_n} (mu = 0: l_t = 0, l_n >= 0)."""

    if mu <= 0.0:
        return np.array([max(x[0], 0.0), 0.0, 0.0])
    s = np.hypot(x[1], x[2])
    if s <= mu * x[0]:
        return x.copy()
    if mu * s <= -x[0]:
        return np.zeros(3)
    a = (x[0] + mu * s) / (1.0 + mu * mu)
    return np.array([a, mu * a * x[1] / s, mu * a * x[2] / s])


def certificates(M, G, vf, target, reg, mu, lam) -> dict[str, float]:
    """KKT certificates of impulses `lam` for the dual problem
    min 0.5 l'(W + R) l + c'l over the cones, W = G M^-1 G', c = G vf - target:
    primal cone violation, dual cone violation of w = (W + R) l + c,
    conic complementarity |l_c' w_c|, and the natural residual
    ||l - P_K(l - w)||_inf, each scaled by 1 + the magnitudes involved."""

    W = G @ np.linalg.solve(M, G.T)
    c = G @ vf - target
    w = (W + np.diag(reg)) @ lam + c
    nc = len(mu)
    scale = 1.0 + np.max(np.abs(lam)) + np.max(np.abs(w))
    primal = dual = comp = nat = 0.0
    for i in range(nc):
        li, wi = lam[3 * i:3 * i + 3], w[3 * i:3 * i + 3]
        lt = np.hypot(li[1], li[2])
        primal = max(primal, -li[0], lt - mu[i] * li[0] if mu[i] > 0 else lt)
        dual = max(dual, mu[i] * np.hypot(wi[1], wi[2]) - wi[0] if mu[i] > 0 else -wi[0])
        comp = max(comp, abs(li @ wi) if mu[i] > 0 else abs(li[0] * wi[0]))
        nat = max(nat, np.max(np.abs(li - project_cone(li - wi, mu[i]))))
    return {"primal_cone": primal / scale, "dual_cone": dual / scale, "complementarity": comp / scale ** 2,
            "natural_residual": nat / scale}
