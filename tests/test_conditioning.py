"""FP32 conditioning of the 29-DoF contact workload, measured on the oracle.

The per-step parity bound for contact worlds cannot be tighter than the
change the FP64 oracle itself makes when its FP32-representable inputs move
by one part in 1e7: contact targets divide positions by the substep
(speculative target -sep / h, stabilisation ~ -err / h), so a 1e-7 m change
in a foot corner moves a target velocity by ~2e-5 m/s.  This test measures
that sensitivity on the same workload the GPU parity test uses and checks
that the GPU tolerance sits above it.
"""

from __future__ import annotations

import ctypes as ct

import numpy as np

import numi_lab_b200 as nb
from oracle import Oracle, OracleManifold

H = 0.005
TREE_V_WORST = 2e-4  # tests/test_gpu_parity.py


def test_oracle_sensitivity_to_fp32_input_rounding_is_below_gpu_tolerance():
    envs, warm, steps = 12, 16, 3
    rec = nb.compile_model("tree29", 5)
    q0, v0, friction = nb.sample_reset("tree29", 5, 5, 0, envs)
    oracle = Oracle(rec, H, 4, 8, 0)
    rng = np.random.default_rng(7)
    na = oracle.nv - 6
    man = [(OracleManifold * oracle.np)() for _ in range(envs)]
    qs = [q0[e].astype(np.float64) for e in range(envs)]
    vs = [v0[e].astype(np.float64) for e in range(envs)]
    for _ in range(warm):
        for e in range(envs):
            st, _ = oracle.control_step(qs[e], vs[e], man[e], 0.3 * rng.standard_normal(na), float(friction[e]))
            assert st == 0
    sens = []
    contacts = 0
    for _ in range(steps):
        for e in range(envs):
            acts = 0.3 * rng.standard_normal(na)
            # FP32-representable start state, as the device holds it.
            q = qs[e].astype(np.float32).astype(np.float64)
            v = vs[e].astype(np.float32).astype(np.float64)
            qa, va = q.copy(), v.copy()
            ma = (OracleManifold * oracle.np)()
            ct.memmove(ma, man[e], ct.sizeof(ma))
            qb = q * (1.0 + 1e-7 * rng.standard_normal(q.size))
            vb = v * (1.0 + 1e-7 * rng.standard_normal(v.size))
            mb = (OracleManifold * oracle.np)()
            ct.memmove(mb, man[e], ct.sizeof(mb))
            st_a, tr = oracle.control_step(qa, va, ma, acts, float(friction[e]))
            st_b, _ = oracle.control_step(qb, vb, mb, acts, float(friction[e]))
            assert st_a == 0 and st_b == 0
            contacts += tr.contact_count
            sens.append(float(np.max(np.abs(va - vb)) / max(1.0, float(np.max(np.abs(va))))))
            qs[e], vs[e], man[e] = qa, va, ma
    worst = max(sens)
    print(f"oracle qd response to 1e-7 input perturbation: median {np.median(sens):.2e} worst {worst:.2e}")
    assert contacts > 0
    # The FP64 reference response alone exceeds the 1e-5 per-step bar ...
    assert worst > 1e-6
    # ... and stays below the tolerance the GPU parity test applies.
    assert worst < TREE_V_WORST


PILE_V_WORST = 1e-3  # tests/test_scene_parity.py
PERTURBATION = 8 * 2.0 ** -24  # eight FP32 roundings


def test_pile_oracle_sensitivity_to_fp32_input_rounding_is_below_gpu_tolerance():
    # Piles stack contacts body on body.  The device forms every world
    # contact point from body-frame anchors by a quaternion rotation and a
    # translation in FP32 -- a chain of about eight rounded operations per
    # component -- so its positions carry relative errors of several parts
    # in 1e7 before the -sep / h targets amplify them.  The FP64 oracle's
    # response to an input perturbation of that size bounds what the
    # per-step comparison can resolve.
    from oracle import SceneOracle, SceneTable

    rng = np.random.default_rng(9)
    sens = []
    contacts = 0
    for seed in (1, 13):
        rec = nb.compile_model("pile", seed)
        oracle = SceneOracle(rec, H, 4, 8, 0)
        q0, v0, f = nb.sample_reset("pile", seed, 1, 0, 1)
        q = q0[0].astype(np.float64)
        v = v0[0].astype(np.float64)
        table = SceneTable()
        for k in range(60):
            assert oracle.step(q, v, table, float(f[0]))[0] == 0
            if k < 30 or k % 3:
                continue
            qa = q.astype(np.float32).astype(np.float64)
            va = v.astype(np.float32).astype(np.float64)
            qb = qa * (1.0 + PERTURBATION * rng.standard_normal(qa.size))
            vb = va * (1.0 + PERTURBATION * rng.standard_normal(va.size))
            ta, tb = SceneTable(), SceneTable()
            ct.memmove(ta.slots, table.slots, ct.sizeof(ta.slots))
            ct.memmove(tb.slots, table.slots, ct.sizeof(tb.slots))
            ta.count.value = tb.count.value = table.count.value
            sa, tr = oracle.step(qa, va, ta, float(f[0]))
            sb, trb = oracle.step(qb, vb, tb, float(f[0]))
            assert sa == 0 and sb == 0
            if tr.band_decisions or trb.band_decisions or ta.keys() != tb.keys():
                continue
            contacts += tr.contact_count
            sens.append(float(np.max(np.abs(va - vb)) / max(1.0, float(np.max(np.abs(va))))))
    worst = max(sens)
    print(f"pile oracle velocity response to {PERTURBATION:.0e} input perturbation: median {np.median(sens):.2e} worst {worst:.2e}")
    assert contacts > 0
    assert worst > 1e-6
    assert worst < PILE_V_WORST
