"""Per-env-step parity bounds from the oracle's own FP32 conditioning.

For one environment-step the oracle (FP64) is run from the device's FP32
input state and, NOISE_RUNS more times, in its Monte Carlo rounding mode
(oracle_set_rounding_noise: every intermediate an FP32 implementation
rounds -- poses, twists, joint accelerations, Jacobian and response terms,
impulse and velocity updates, integration -- and every input, including
the warm-start impulses and manifold anchors, is multiplied by 1 + d with d
uniform in [-2^-24, 2^-24], one rounding to nearest; Parker 1997).  The
largest deviation of those runs from the exact one is the step's
sensitivity: how far FP32 rounding alone moves this step's result.  A
device result is held to max(base tolerance, K x sensitivity) (K below): on a
well-conditioned step that is the base tolerance itself (q and qd 1e-5,
impulses 1e-4, relative to max(1, |x|)); where a step amplifies rounding
(contact targets divide positions by the substep, an impulse sits at the
cone's apex) the bound follows that step's own amplification instead of a
blanket loosening.  Runs in which rounding flips a discrete decision do
not count towards the sensitivity; a step where every run flips one is a
band step.

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

# Device error allowed per unit of measured rounding sensitivity.  Over
# 5,748 clean env-steps of the 4096-env tree29 benchmark the ratio of the
# device's deviation to the sensitivity had median 0.6, 99th percentile 3.3
# and maximum 10.7; over 1,961 clean pile env-steps (8-50 bodies, with and
# without cylinders) median 1.3, 99th percentile 14, maximum 36: the pile
# kernel's narrowphase and body-list sums take more FP32 roundings than the
# oracle's noise points model.
K_TREE = 16.0
K_SCENE = 64.0
NOISE_RUNS = 3
ULP = 2.0 ** -24       # one rounding to nearest, relative


def rel_err(a: np.ndarray, b: np.ndarray) -> float:
    return float(np.max(np.abs(a - b)) / max(1.0, float(np.max(np.abs(b))))) if a.size else 0.0


@functools.lru_cache(maxsize=8)
def _tree_oracle(source: str, seed: int, h: float, substeps: int, iters: int, quality: bool = False):
    import numi_lab_b200 as nb
    from oracle import Oracle, quality_config

    rec = nb.compile_model(source, seed)
    oracle = Oracle(rec, h, substeps, iters, 0)
    if quality:
        oracle.set_quality(quality_config())
    return rec, oracle


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
    friction, rng; optional quality (the converged contact solve)."""

    from numi_lab_b200 import native

    rec, oracle = _tree_oracle(job["source"], job["seed"], job["h"], job["substeps"], job["iters"], bool(job.get("quality")))
    pairs = int(rec.world.pair_count)

    def run(q, v, rng=None):
        dev = (native.ManifoldC * max(pairs, 1)).from_buffer_copy(job["manifolds"])
        man = oracle.env_manifolds(dev, 0)
        if rng is not None:
            # The warm-start impulses and anchors are FP32 inputs too.
            for p in range(pairs):
                for i in range(man[p].count):
                    pt = man[p].points[i]
                    for a in range(3):
                        pt.impulses[a] *= 1.0 + ULP * rng.uniform(-1.0, 1.0)
                        pt.anchor_a[a] *= 1.0 + ULP * rng.uniform(-1.0, 1.0)
                        pt.anchor_b[a] *= 1.0 + ULP * rng.uniform(-1.0, 1.0)
        q, v = q.astype(np.float64), v.astype(np.float64)
        st, trace = oracle.control_step(q, v, man, job["actions"], job["friction"])
        imp, feats = _impulses_tree(man, pairs)
        return st, trace, q, v, imp, feats

    from oracle import set_rounding_noise

    st, trace, q, v, imp, feats = run(job["q"], job["v"])
    rng = np.random.default_rng(job["rng"])
    sens = {"q": 0.0, "v": 0.0, "imp": 0.0}
    flips = 0
    for r in range(NOISE_RUNS):
        qp = job["q"].astype(np.float64) * (1.0 + ULP * rng.uniform(-1.0, 1.0, size=job["q"].shape))
        vp = job["v"].astype(np.float64) * (1.0 + ULP * rng.uniform(-1.0, 1.0, size=job["v"].shape))
        set_rounding_noise(int(rng.integers(1, 2**62)))
        try:
            stp, _, q2, v2, imp2, feats2 = run(qp, vp, rng)
        finally:
            set_rounding_noise(0)
        if stp != st or feats2 != feats:
            flips += 1
            continue
        sens["q"] = max(sens["q"], rel_err(q2, q))
        sens["v"] = max(sens["v"], rel_err(v2, v))
        if imp.size:
            sens["imp"] = max(sens["imp"], float(np.max(np.abs(imp2 - imp))) / max(1.0, float(np.max(np.abs(imp)))))
    if flips == NOISE_RUNS:
        sens = {"q": np.inf, "v": np.inf, "imp": np.inf}  # rounding flips a decision in every run: a band step
    return {"status": st, "band": int(trace.band_decisions), "q": q, "v": v, "imp": imp, "features": feats, "sens": sens,
            "contacts": int(trace.contact_count), "flips": flips, "k": K_TREE}


def scene_env_step(job: dict) -> dict:
    """One free-body control step of one environment in the oracle, plus its
    input sensitivity.  job: source, seed, h, substeps, iters, q, v
    (float32), table (the env's [slot][57] words), count, friction, rng."""

    rec, oracle = _scene_oracle(job["source"], job["seed"], job["h"], job["substeps"], job["iters"])

    def run(q, v, rng=None):
        table = oracle.table_from_device(job["table"], job["count"])
        if rng is not None:
            for i in range(table.count.value):
                m = table.slots[i].m
                for p in range(m.count):
                    pt = m.points[p]
                    for a in range(3):
                        pt.impulses[a] *= 1.0 + ULP * rng.uniform(-1.0, 1.0)
                        pt.anchor_a[a] *= 1.0 + ULP * rng.uniform(-1.0, 1.0)
                        pt.anchor_b[a] *= 1.0 + ULP * rng.uniform(-1.0, 1.0)
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

    from oracle import set_rounding_noise

    st, trace, q, v, imp, feats = run(job["q"], job["v"])
    rng = np.random.default_rng(job["rng"])
    sens = {"q": 0.0, "v": 0.0, "imp": 0.0}
    flips = 0
    for r in range(NOISE_RUNS):
        qp = job["q"].astype(np.float64) * (1.0 + ULP * rng.uniform(-1.0, 1.0, size=job["q"].shape))
        vp = job["v"].astype(np.float64) * (1.0 + ULP * rng.uniform(-1.0, 1.0, size=job["v"].shape))
        set_rounding_noise(int(rng.integers(1, 2**62)))
        try:
            stp, _, q2, v2, imp2, feats2 = run(qp, vp, rng)
        finally:
            set_rounding_noise(0)
        if stp != st or feats2 != feats:
            flips += 1
            continue
        sens["q"] = max(sens["q"], rel_err(q2, q))
        sens["v"] = max(sens["v"], rel_err(v2, v))
        if imp.size:
            sens["imp"] = max(sens["imp"], float(np.max(np.abs(imp2 - imp))) / max(1.0, float(np.max(np.abs(imp)))))
    if flips == NOISE_RUNS:
        sens = {"q": np.inf, "v": np.inf, "imp": np.inf}
    return {"status": st, "band": int(trace.band_decisions), "q": q, "v": v, "imp": imp, "features": feats, "sens": sens,
            "contacts": int(trace.contact_count), "island_of": np.array(trace.island_of, np.uint32), "flips": flips,
            "k": K_SCENE}


def pool(workers: int | None = None) -> ProcessPoolExecutor:
    n = workers or max(1, min(16, (os.cpu_count() or 2)))
    return ProcessPoolExecutor(max_workers=n, mp_context=mp.get_context("spawn"))


BASES = {"q": 1e-5, "v": 1e-5, "imp": 1e-4}


def judge(res: dict, features_equal: bool, errors: dict) -> tuple[str, list]:
    """Classifies one env-step: "ok" (identical decisions, every error
    within its bound), "band" (it is not, on a step where the oracle took a
    decision within its band of a threshold or where rounding flipped one
    in a noisy run: FP32 may legitimately differ there) or "fail"."""

    near = res["band"] > 0 or res["flips"] > 0
    misses = []
    if features_equal:
        for name, err in errors.items():
            ok, bound = bounded(err, res["sens"][name], BASES[name], res["k"])
            if not ok:
                misses.append((name, err, bound, res["sens"][name]))
    if features_equal and not misses:
        return "ok", []
    return ("band" if near else "fail"), misses or ["decisions differ"]


def bounded(err: float, sens: float, base: float, k: float) -> tuple[bool, float]:
    """(within the per-step bound, the bound)."""

    bound = max(base, k * sens)
    return err <= bound, bound


def manifold_bytes(manifolds, env: int, pairs: int) -> bytes:
    size = ct.sizeof(manifolds._type_)
    return ct.string_at(ct.addressof(manifolds) + env * pairs * size, pairs * size)
