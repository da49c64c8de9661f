"""Converged (quality) contact solve on the device.

* mr_quality_solve_batch on the golden problems (tests/golden/
  quality_pins.npz: contact patches of the 29-DoF tree and random dense
  problems): every solve converges, its KKT certificates (tests/_quality.py,
  computed here from the returned impulses) are at most 1e-8, its impulses
  and velocities match the reference's solveQualityContactProblem within
  1e-6 wherever the reference converged, and the oracle's restatement of
  the same iteration within 1e-8;
* the tree29 world with MR_SOLVER_QUALITY_NEWTON: per control step from
  identical FP32 state against the oracle world with the converged solve,
  each env-step held to max(base, K x its FP32 sensitivity)
  (tests/_sensitivity.py), and the device's own certificates;
* the solver's argument checks on worlds it does not run.
"""

from __future__ import annotations

import numpy as np
import pytest

import _quality as Q
import numi_lab_b200 as nb
from oracle import quality_dense

from test_quality import golden_problems

pytestmark = pytest.mark.gpu

REF_TOL = 1.0e-6     # device vs reference, relative to max(1, |x|)
ORACLE_TOL = 1.0e-8  # device vs the oracle's restatement of the same iteration
CERT_TOL = 1.0e-8


def _rel(a: np.ndarray, b: np.ndarray) -> float:
    return float(np.max(np.abs(a - b)) / max(1.0, float(np.max(np.abs(b))))) if a.size else 0.0


def test_device_quality_solve_matches_the_reference(cuda_device):
    matched = 0
    worst = {"ref": 0.0, "oracle": 0.0, "cert": 0.0}
    for p, d, prob in golden_problems():
        M, G, vf, target, reg, mu = prob
        imp, vel, res = nb.quality_solve(M[None], G[None], vf[None], target[None], reg[None], mu[None])
        lam, v = imp[0], vel[0]
        assert res[0]["code"] == 0, (p, res[0])
        assert res[0]["cone_violation"] <= 1e-12
        cert = Q.certificates(*prob, lam)
        worst["cert"] = max(worst["cert"], max(cert.values()))
        assert max(cert.values()) <= CERT_TOL, (p, cert)
        _, olam, ovel, _ = quality_dense(*prob)
        worst["oracle"] = max(worst["oracle"], _rel(lam, olam), _rel(v, ovel))
        assert _rel(lam, olam) <= ORACLE_TOL and _rel(v, ovel) <= ORACLE_TOL, p
        if d["ref_status"][p] == 0:
            nv, nc = M.shape[0], len(mu)
            err = max(_rel(lam, d["ref_impulses"][p, :3 * nc]), _rel(v, d["ref_velocity"][p, :nv]))
            worst["ref"] = max(worst["ref"], err)
            assert err <= REF_TOL, (p, err)
            matched += 1
    print("worst relative errors:", worst)
    assert matched >= 24


def test_device_quality_solve_batches_ragged_contact_sets(cuda_device):
    """The 16 tree29 patches (8-20 contacts) in one call, padded to 20
    contacts with per-problem counts, warm-started from perturbed
    impulses: every problem's answer equals its own solve."""

    d = np.load(str(__import__("test_quality").GOLDEN))
    tree = [p for p in range(len(d["nv"])) if d["kind"][p]]
    nv = int(d["nv"][tree[0]])
    cap = 20
    M = d["mass"][tree, :nv, :nv]
    G = d["jacobian"][tree, :3 * cap, :nv]
    counts = d["nc"][tree].astype(np.uint32)
    rng = np.random.default_rng(5)
    warm = d["ref_impulses"][tree] * (1.0 + 0.05 * rng.normal(size=(len(tree), 3 * cap)))
    imp, vel, res = nb.quality_solve(M, G, d["free_velocity"][tree, :nv], d["target"][tree], d["regularization"][tree],
                                     d["friction"][tree], counts=counts, warm=warm)
    for i, p in enumerate(tree):
        nc = int(counts[i])
        assert res[i]["code"] == 0
        assert np.all(imp[i, 3 * nc:] == 0.0)
        _, olam, ovel, _ = quality_dense(M[i], G[i, :3 * nc], d["free_velocity"][p, :nv], d["target"][p, :3 * nc],
                                         d["regularization"][p, :3 * nc], d["friction"][p, :nc])
        assert _rel(imp[i, :3 * nc], olam) <= 1e-7 and _rel(vel[i], ovel) <= 1e-7


def _tree_world(envs: int, seed: int):
    return nb.World("tree29", envs, substeps=4, velocity_iterations=8, control_dt=0.02, seed=seed)


def test_tree29_quality_world_per_step(cuda_device):
    """Per control step from identical FP32 state, the device's quality
    world against the oracle world with the converged solve; q and qd held
    to max(1e-5, K x sensitivity), impulses to max(1e-4, K x sensitivity).
    The device's own certificates of every solve stay at or below 1e-6."""

    import torch

    import _sensitivity as S

    envs, warm, steps, seed = 32, 10, 8, 5
    with _tree_world(envs, seed) as world, S.pool() as ex:
        world.set_solver("quality_newton")
        friction = world.friction_scales()
        pairs = world.pair_count
        gen = torch.Generator(device="cuda").manual_seed(21)
        _, status, _ = world.step(0.3 * torch.randn((warm, envs, world.action_count), device="cuda", generator=gen), wait=True)
        assert int(status.abs().sum()) == 0
        failures, band_cases, contacts_seen = [], 0, 0
        newton = 0
        for k in range(steps):
            q0, v0, m0 = world.state()
            actions = 0.3 * torch.randn((1, envs, world.action_count), device="cuda", generator=gen)
            _, status, _ = world.step(actions, wait=True)
            assert int(status.abs().sum()) == 0
            diag = world.quality_diagnostics()
            assert diag["scaled_optimality"] <= 1e-6 and diag["cone_violation"] <= 1e-6, diag
            newton = max(newton, diag["newton_iterations"])
            q1, v1, m1 = world.state()
            acts = actions.cpu().numpy()[0].astype(np.float64)
            jobs = [{"source": "tree29", "seed": seed, "h": 0.005, "substeps": 4, "iters": 8, "q": q0[e], "v": v0[e],
                     "manifolds": S.manifold_bytes(m0, e, pairs), "actions": acts[e], "friction": float(friction[e]),
                     "rng": 1000 * k + e, "quality": True} for e in range(envs)]
            for e, res in enumerate(ex.map(S.tree_env_step, jobs, chunksize=4)):
                assert res["status"] == 0
                imps, feats = [], []
                for p in range(pairs):
                    gm = m1[e * pairs + p]
                    feats.append((int(gm.count), tuple((int(gm.points[i].feature_a), int(gm.points[i].feature_b),
                                                        int(gm.points[i].life)) for i in range(gm.count))))
                    imps += [list(gm.points[i].impulses) for i in range(gm.count)]
                imp = np.array(imps, np.float64).reshape(-1, 3)
                same = tuple(feats) == res["features"]
                dq, dv = S.rel_err(q1[e], res["q"]), S.rel_err(v1[e], res["v"])
                di = (float(np.max(np.abs(imp - res["imp"]))) / max(1.0, float(np.max(np.abs(res["imp"]))))
                      if same and imp.size else 0.0)
                verdict, misses = S.judge(res, same, {"q": dq, "v": dv, "imp": di})
                if verdict == "band":
                    band_cases += 1
                elif verdict == "fail":
                    failures.append((k, e, misses))
                else:
                    contacts_seen += res["contacts"]
        print(f"tree29 quality: {band_cases} band cases, most Newton steps of one solve {newton}")
        assert not failures, failures[:10]
        assert contacts_seen > 0
        assert band_cases <= envs * steps // 20


def test_quality_solver_is_refused_where_it_does_not_run(cuda_device):
    with nb.World("pile", 2, seed=3) as pile:
        with pytest.raises(nb.MetalRoboError, match="articulated contact"):
            pile.set_solver("quality_newton")
    with nb.World("chain7", 2, seed=3) as chain:
        with pytest.raises(nb.MetalRoboError, match="contact world"):
            chain.set_solver("quality_newton")
    with _tree_world(4, 3) as tree:
        tree.set_solver("quality_newton")
        with pytest.raises(nb.MetalRoboError, match="temporalCone"):
            nb.Batch([tree])
        tree.set_solver("temporal_cone")
        with nb.Batch([tree]):
            pass
