"""The per-environment FP64 energy and momentum audit on the device
(mr_task_rollout_set_audit): its records must equal the same quantities
computed on the host in FP64 from the device's committed FP32 state --
trees through the FP64 oracle's mass matrix and point Jacobians, piles
body by body -- and its reference / drift accumulators must follow resets."""

from __future__ import annotations

import numpy as np
import pytest

import numi_lab_b200 as nb
from oracle import Oracle

pytestmark = pytest.mark.gpu

REL = 1e-5  # relative to max(1, |x|): the device's FP32 forward kinematics against FP64


def _close(a: float, b: float, scale: float) -> None:
    assert abs(a - b) <= REL * max(1.0, abs(scale)), (a, b)


def test_tree_audit_matches_host_fp64(cuda_device):
    import torch

    envs = 16
    with nb.World("tree29", envs, seed=5) as world:
        world.set_audit(True)
        rec = world.model()
        oracle = Oracle(rec, 0.005, 4, 8, 0)
        gen = torch.Generator(device="cuda").manual_seed(3)
        world.step(0.3 * torch.randn((6, envs, world.action_count), device="cuda", generator=gen), wait=True)
        q, v, _ = world.state()
        audit = world.audit()
        g = np.array(rec.world.gravity[:3], np.float64)
        for e in range(envs):
            qe, ve = q[e].astype(np.float64), v[e].astype(np.float64)
            kinetic = 0.5 * ve @ oracle.mass_matrix(qe) @ ve
            potential, momentum = 0.0, np.zeros(3)
            for b in range(rec.world.body_count):
                if not rec.bodies[b].articulated:
                    continue
                m = float(rec.bodies[b].mass_inverse_mass[0])
                c, J = oracle.point_jacobian(qe, b, np.zeros(3))
                potential -= m * float(g @ c)
                momentum += m * (J @ ve)
            a = audit[e]
            _close(a[0], kinetic, kinetic + abs(potential))
            _close(a[1], potential, kinetic + abs(potential))
            _close(a[2], kinetic + potential, kinetic + abs(potential))
            np.testing.assert_allclose(a[5:8], momentum, atol=REL * max(1.0, float(np.abs(momentum).max())))
            assert a[11] == 6  # six audited control steps since the reference
            assert a[4] >= abs(a[2] - a[3]) - 1e-12


def _pile_reference(rec, q, v):
    n = rec.world.body_count - 1
    g = np.array(rec.world.gravity[:3], np.float64)
    kinetic = potential = 0.0
    p, L = np.zeros(3), np.zeros(3)
    for b in range(n):
        m = float(rec.bodies[b].mass_inverse_mass[0])
        inertia = np.diag([float(rec.bodies[b].inertia[i][i]) for i in range(3)])
        c = q[7 * b: 7 * b + 3]
        x, y, z, w = q[7 * b + 3: 7 * b + 7]
        R = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                      [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                      [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])
        lin, ang = v[6 * b: 6 * b + 3], v[6 * b + 3: 6 * b + 6]
        Iw = R @ inertia @ R.T
        kinetic += 0.5 * m * lin @ lin + 0.5 * ang @ Iw @ ang
        potential -= m * g @ c
        p += m * lin
        L += np.cross(c, m * lin) + Iw @ ang
    return kinetic, potential, p, L


def test_pile_audit_matches_host_fp64_and_follows_resets(cuda_device):
    import torch

    envs = 8
    with nb.World("pile", envs, seed=13) as world:
        world.set_audit(True)
        rec = world.model()
        acts = torch.zeros((10, envs, 0), device="cuda")
        world.step(acts, wait=True)
        q, v, _ = world.state()
        audit = world.audit()
        for e in range(envs):
            kinetic, potential, p, L = _pile_reference(rec, q[e].astype(np.float64), v[e].astype(np.float64))
            scale = kinetic + abs(potential)
            a = audit[e]
            _close(a[0], kinetic, scale)
            _close(a[1], potential, scale)
            np.testing.assert_allclose(a[5:8], p, atol=REL * max(1.0, float(np.abs(p).max())))
            np.testing.assert_allclose(a[8:11], L, atol=REL * max(1.0, float(np.abs(L).max())))
            assert a[11] == 10
            # Falling bodies trade potential for kinetic energy; damping and
            # contacts dissipate: the drift accumulator records the change.
            assert a[4] >= abs(a[2] - a[3]) - 1e-9
        # A reset of environment 2 takes a new reference there only.
        mask = torch.zeros((1, envs), dtype=torch.int32, device="cuda")
        mask[0, 2] = 1
        world.step(torch.zeros((1, envs, 0), device="cuda"), reset_mask=mask, wait=True)
        after = world.audit()
        assert after[2, 11] == 1 and after[2, 4] == 0.0
        assert after[0, 11] == 11
