"""Per-env-step parity bounds from the oracle's own conditioning.

For one environment-step the oracle (FP64) is run from the device's FP32
input state and, twice more, from that state with every q and v component
moved by one FP32 rounding (relative 2^-23, random signs).  The spread of
those runs is the step's sensitivity to FP32 inputs: the change in the
result that rounding the inputs alone causes.  A device result is held to
max(base tolerance, K x sensitivity): on a well-conditioned step (tiny
sensitivity) that is the base tolerance itself (q and qd 1e-5, impulses
1e-4, relative to max(1, |x|)); where contact targets divide positions by
the substep (-sep / h) and amplify rounding, the bound follows the
problem's own amplification instead of a blanket loosening.

The oracle work runs in a process pool started with the 'spawn' method, so
it is safe after CUDA has been initialised in the parent.  Workers rebuild
the oracle from (source, model seed) and keep it per process.
"""

from __future__ import annotations

import ctypes as ct
import functools
import multiprocessing as mp
import os
from concurrent.futures import ProcessPoolExecutor

import numpy as np

K_SENS = 8.0           # device error allowed per unit of oracle input sensitivity
PERTURBATIONS = 2
ULP = 2.0 ** -23


def rel_err(a: np.ndarray, b: np.ndarray) -> float:
    return float(np.max(np.abs(a - b)) / max(1.0, float(np.max(np.abs(b))))) if a.size else 0.0


@functools.lru_cache(maxsize=8)
def _tree_oracle(source: str, seed: int, h: float, substeps: int, iters: int):
    import numi_lab_b200 as nb
    from oracle import Oracle

    rec = nb.compile_model(source, seed)
    return rec, Oracle(rec, h, substeps, iters, 0)


@functools.lru_cache(maxsize=8)
def _scene_oracle(source: str, seed: int, h: float, substeps: int, iters: int):
    import numi_lab_b200 as nb
    from oracle import SceneOracle

    rec = nb.compile_model(source, seed)
    return rec, SceneOracle(rec, h, substeps, iters, 0)


def _impulses_tree(man, pairs: int) -> tuple[np.ndarray, tuple]:
    imps, feats = [], []
    for p in range(pairs):
        m = man[p]
        feats.append((int(m.count), tuple((int(m.points[i].feature_a), int(m.points[i].feature_b), int(m.points[i].life))
                                          for i in range(m.count))))
        for i in range(m.count):
            imps.append(list(m.points[i].impulses))
    return np.array(imps, np.float64).reshape(-1, 3), tuple(feats)


def tree_env_step(job: dict) -> dict:
    """One articulated control step of one environment in the oracle, plus
    its input sensitivity.  job: source, seed, h, substeps, iters, q, v
    (float32), manifolds (bytes of the env's MRManifoldC slots), actions,
    friction, rng."""

    from numi_lab_b200 import native

    rec, oracle = _tree_oracle(job["source"], job["seed"], job["h"], job["substeps"], job["iters"])
    pairs = int(rec.world.pair_count)

    def run(q, v):
        dev = (native.ManifoldC * max(pairs, 1)).from_buffer_copy(job["manifolds"])
        man = oracle.env_manifolds(dev, 0)
        q, v = q.astype(np.float64), v.astype(np.float64)
        st, trace = oracle.control_step(q, v, man, job["actions"], job["friction"])
        imp, feats = _impulses_tree(man, pairs)
        return st, trace, q, v, imp, feats

    st, trace, q, v, imp, feats = run(job["q"], job["v"])
    rng = np.random.default_rng(job["rng"])
    sens = {"q": 0.0, "v": 0.0, "imp": 0.0}
    for _ in range(PERTURBATIONS):
        qp = job["q"].astype(np.float64) * (1.0 + ULP * rng.choice([-1.0, 1.0], size=job["q"].shape))
        vp = job["v"].astype(np.float64) * (1.0 + ULP * rng.choice([-1.0, 1.0], size=job["v"].shape))
        stp, _, q2, v2, imp2, feats2 = run(qp, vp)
        if stp != st or feats2 != feats:
            sens = {"q": np.inf, "v": np.inf, "imp": np.inf}  # a decision flips under input rounding: a band step
            break
        sens["q"] = max(sens["q"], rel_err(q2, q))
        sens["v"] = max(sens["v"], rel_err(v2, v))
        if imp.size:
            sens["imp"] = max(sens["imp"], float(np.max(np.abs(imp2 - imp))) / max(1.0, float(np.max(np.abs(imp)))))
    return {"status": st, "band": int(trace.band_decisions), "q": q, "v": v, "imp": imp, "features": feats, "sens": sens,
            "contacts": int(trace.contact_count)}


def scene_env_step(job: dict) -> dict:
    """One free-body control step of one environment in the oracle, plus its
    input sensitivity.  job: source, seed, h, substeps, iters, q, v
    (float32), table (the env's [slot][57] words), count, friction, rng."""

    rec, oracle = _scene_oracle(job["source"], job["seed"], job["h"], job["substeps"], job["iters"])

    def run(q, v):
        table = oracle.table_from_device(job["table"], job["count"])
        q, v = q.astype(np.float64), v.astype(np.float64)
        st, trace = oracle.step(q, v, table, job["friction"])
        imps, feats = [], []
        for i in range(table.count.value):
            m = table.slots[i].m
            feats.append((int(table.slots[i].key), tuple((int(m.points[p].feature_a), int(m.points[p].feature_b),
                                                          int(m.points[p].life)) for p in range(m.count))))
            for p in range(m.count):
                imps.append(list(m.points[p].impulses))
        return st, trace, q, v, np.array(imps, np.float64).reshape(-1, 3), tuple(feats)

    st, trace, q, v, imp, feats = run(job["q"], job["v"])
    rng = np.random.default_rng(job["rng"])
    sens = {"q": 0.0, "v": 0.0, "imp": 0.0}
    for _ in range(PERTURBATIONS):
        qp = job["q"].astype(np.float64) * (1.0 + ULP * rng.choice([-1.0, 1.0], size=job["q"].shape))
        vp = job["v"].astype(np.float64) * (1.0 + ULP * rng.choice([-1.0, 1.0], size=job["v"].shape))
        stp, _, q2, v2, imp2, feats2 = run(qp, vp)
        if stp != st or feats2 != feats:
            sens = {"q": np.inf, "v": np.inf, "imp": np.inf}
            break
        sens["q"] = max(sens["q"], rel_err(q2, q))
        sens["v"] = max(sens["v"], rel_err(v2, v))
        if imp.size:
            sens["imp"] = max(sens["imp"], float(np.max(np.abs(imp2 - imp))) / max(1.0, float(np.max(np.abs(imp)))))
    return {"status": st, "band": int(trace.band_decisions), "q": q, "v": v, "imp": imp, "features": feats, "sens": sens,
            "contacts": int(trace.contact_count), "island_of": np.array(trace.island_of, np.uint32)}


def pool(workers: int | None = None) -> ProcessPoolExecutor:
    n = workers or max(1, min(16, (os.cpu_count() or 2)))
    return ProcessPoolExecutor(max_workers=n, mp_context=mp.get_context("spawn"))


def bounded(err: float, sens: float, base: float) -> tuple[bool, float]:
    """(within the per-step bound, the bound)."""

    bound = max(base, K_SENS * sens)
    return err <= bound, bound


def manifold_bytes(manifolds, env: int, pairs: int) -> bytes:
    size = ct.sizeof(manifolds._type_)
    return ct.string_at(ct.addressof(manifolds) + env * pairs * size, pairs * size)
