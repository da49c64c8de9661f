"""C-ABI surface checks that need no GPU: the library loads, exports every
entry point include/numi_b200.h declares, follows the reference's error
conventions, and compiles the synthetic worlds deterministically."""

from __future__ import annotations

import ctypes as ct
import re
from pathlib import Path

import numpy as np

import numi_lab_b200 as nb
from numi_lab_b200 import native

HEADER = Path(__file__).resolve().parents[1] / "include" / "numi_b200.h"


def declared_entry_points() -> list[str]:
    text = HEADER.read_text()
    return sorted(set(re.findall(r"MR_API[^;]*?\b(mr_[a-z0-9_]+)\s*\(", text, re.S)))


def test_library_exports_every_declared_symbol():
    lib = native.bindings()
    names = declared_entry_points()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib.lib, name), f"{name} declared in numi_b200.h but not exported"
    for name in native.EXPORTED_SYMBOLS:
        assert name in names, f"binding configures {name} which the header does not declare"


def test_version_and_fingerprint():
    lib = native.bindings()
    assert b"sm_100a" in lib.lib.mr_version()
    assert lib.lib.mr_runtime_abi_fingerprint() == lib.lib.mr_runtime_abi_fingerprint() != 0


def test_struct_sizes_match_header_layout(tmp_path):
    # The ctypes mirror must agree with the C compiler's layout of every record.
    import subprocess

    records = {
        "MRTaskRolloutConfigC": native.TaskRolloutConfigC,
        "MRRunManifestC": native.RunManifestC,
        "MRTaskRolloutLayoutC": native.TaskRolloutLayoutC,
        "MRTaskRolloutStageHighWaterC": native.StageHighWaterC,
        "MRTaskRolloutAdvanceC": native.TaskRolloutAdvanceC,
        "MRModelWorldC": native.ModelWorldC,
        "MRModelJointC": native.ModelJointC,
        "MRModelBodyC": native.ModelBodyC,
        "MRModelDofC": native.ModelDofC,
        "MRModelShapeC": native.ModelShapeC,
        "MRModelMaterialC": native.ModelMaterialC,
        "MRModelPairC": native.ModelPairC,
        "MRModelViewC": native.ModelViewC,
        "MRManifoldC": native.ManifoldC,
        "MRServerConfigC": native.ServerConfigC,
        "MRServerRequestC": native.ServerRequestC,
        "MRServerCompletionC": native.ServerCompletionC,
        "MRServerStatsC": native.ServerStatsC,
        "MRPolicyDenseLayerC": native.PolicyDenseLayerC,
        "MRPolicyPackC": native.PolicyPackC,
        "MRPolicyPackInfoC": native.PolicyPackInfoC,
        "MRQualitySolverConfigC": native.QualitySolverConfigC,
        "MRQualityDiagnosticsC": native.QualityDiagnosticsC,
        "MRQualityResultC": native.QualityResultC,
        "MRBatchLaunchShapeC": native.BatchLaunchShapeC,
        "MRTaskActionBindingC": native.TaskActionBindingC,
        "MRTaskObservationOperatorC": native.TaskObservationOperatorC,
        "MRTaskRewardOperatorC": native.TaskRewardOperatorC,
        "MRTaskTerminationOperatorC": native.TaskTerminationOperatorC,
        "MRTaskRandomizationOperatorC": native.TaskRandomizationOperatorC,
        "MRTaskIndexGroupC": native.TaskIndexGroupC,
        "MRTaskProgramC": native.TaskProgramC,
        "MRTaskContactGroupC": native.TaskContactGroupC,
        "MRTaskTransitionC": native.TaskTransitionC,
        "MRPolicyRolloutBatchC": native.PolicyRolloutBatchC,
        "MRPolicyRolloutPackC": native.PolicyRolloutPackC,
        "MRPolicyRolloutPackInfoC": native.PolicyRolloutPackInfoC,
        "MRTaskPackInfoC": native.TaskPackInfoC,
    }
    src = tmp_path / "sizes.c"
    body = "".join(f'printf("%zu\\n", sizeof({name}));' for name in records)
    src.write_text(f'#include <stdio.h>\n#include "numi_b200.h"\nint main(void){{{body}return 0;}}\n')
    exe = tmp_path / "sizes"
    subprocess.run(["gcc", "-I", str(HEADER.parent), str(src), "-o", str(exe)], check=True)
    sizes = [int(x) for x in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    for (name, cls), size in zip(records.items(), sizes):
        assert ct.sizeof(cls) == size, (name, ct.sizeof(cls), size)


def test_null_manifest_sets_last_error():
    lib = native.bindings()
    assert lib.lib.mr_create_task_rollout(None) is None
    assert "manifest is null" in lib.last_error()


def test_unsupported_source_is_rejected_with_message():
    lib = native.bindings()
    manifest = native.default_manifest(native.MR_RUN_SOURCE_SYNTHETIC_TREE29, 4)
    manifest.source = 0  # Unitree G1 asset source: not compiled by this library
    assert lib.lib.mr_create_task_rollout(ct.byref(manifest)) is None
    assert "unsupported run source" in lib.last_error()


def test_invalid_profile_is_rejected_before_device_work():
    lib = native.bindings()
    manifest = native.default_manifest(native.MR_RUN_SOURCE_SYNTHETIC_TREE29, 0)
    assert lib.lib.mr_create_task_rollout(ct.byref(manifest)) is None
    assert "environment_count" in lib.last_error()
    manifest = native.default_manifest(native.MR_RUN_SOURCE_SYNTHETIC_TREE29, 4, physics_substeps=65)
    assert lib.lib.mr_create_task_rollout(ct.byref(manifest)) is None
    assert "physics_substeps" in lib.last_error()


def test_null_handle_calls_fail_cleanly():
    lib = native.bindings()
    out = native.TaskRolloutAdvanceC()
    assert lib.lib.mr_task_rollout_reset(None, 1) == -1
    assert "handle is null" in lib.last_error()
    assert lib.lib.mr_task_rollout_advance(None, None, 0, None, 0, 1, 0, 0, ct.byref(out)) == -1
    assert lib.lib.mr_task_rollout_status_codes(None) is None or not lib.lib.mr_task_rollout_status_codes(None)


def test_synthetic_worlds_compile_deterministically():
    a = nb.compile_model("tree29", 42)
    b = nb.compile_model("tree29", 42)
    c = nb.compile_model("tree29", 43)
    w = a.world
    assert (w.body_count, w.nq, w.nv, w.action_count) == (31, 36, 35, 29)
    assert (w.shape_count, w.pair_count, w.contact_capacity) == (15, 14, 20)
    assert bytes(a.bodies) == bytes(b.bodies) and bytes(a.bodies) != bytes(c.bodies)
    chain = nb.compile_model("chain7", 0).world
    assert (chain.body_count, chain.nq, chain.nv, chain.pair_count) == (8, 7, 7, 0)
    # 7-revolute chain: link masses U(0.5, 4) kg, axes alternate z / y.
    m = nb.compile_model("chain7", 0)
    masses = [m.bodies[i].mass_inverse_mass[0] for i in range(1, 8)]
    assert all(0.5 <= x <= 4.0 for x in masses)
    axes = [tuple(m.joints[j].axis[:3]) for j in range(7)]
    assert axes[0] == (0.0, 0.0, 1.0) and axes[1] == (0.0, 1.0, 0.0)


def test_reset_sampling_is_reproducible_and_valid():
    q1, v1, f1 = nb.sample_reset("tree29", 3, 9, 0, 16)
    q2, v2, f2 = nb.sample_reset("tree29", 3, 9, 8, 8)
    np.testing.assert_array_equal(q1[8:], q2)
    np.testing.assert_array_equal(f1[8:], f2)
    norms = np.linalg.norm(q1[:, 3:7], axis=1)
    np.testing.assert_allclose(norms, 1.0, atol=1e-6)
    assert np.all((f1 >= 0.4) & (f1 <= 1.0))
    qc, vc, _ = nb.sample_reset("chain7", 0, 0, 0, 256)
    assert np.all(np.abs(qc) <= np.pi / 2 + 1e-6)
    assert 0.8 < np.std(vc) < 1.2
