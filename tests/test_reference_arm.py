"""The reference CPU arm of the benchmark: it reads the workload from the
committed fixture (oracle/workloads/) and steps it with the reference's own
compiled CPU core, without loading this project's CUDA library."""

from __future__ import annotations

import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]

pytestmark = pytest.mark.reference


def test_fixture_matches_the_compiled_world_and_reset_states():
    import numi_lab_b200 as nb
    from oracle import workloads

    records, arrays = workloads.load(workloads.path("tree29_seed2026"))
    fresh = nb.compile_model("tree29", 2026)
    assert bytes(records.world) == bytes(fresh.world)
    for f in ("joints", "bodies", "dofs", "shapes", "materials", "pairs"):
        assert bytes(getattr(records, f)) == bytes(getattr(fresh, f)), f
    q, v, fr = nb.sample_reset("tree29", 2026, 2026, 0, 512)
    assert np.array_equal(arrays["q"], q) and np.array_equal(arrays["v"], v) and np.array_equal(arrays["friction"], fr)


def test_reference_sample_loads_only_the_reference_core(reference_available):
    code = (
        "import sys; sys.path.insert(0, %r)\n"
        "import bench\n"
        "res = bench._reference_sample(2, bench._reference_actions(0)[:1, :])\n" % str(ROOT)
    )
    # One control step of the 512-environment sample, then the process's
    # mapped files: the reference core, never libnumi_b200.so.
    code = code.replace("bench._reference_actions(0)[:1, :]", "bench._reference_actions(0)[:1]")
    code += "print(res['value'] > 0)\nprint(open('/proc/self/maps').read())\n"
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr
    assert out.stdout.startswith("True")
    assert "libnumiref.so" in out.stdout
    assert "libnumi_b200.so" not in out.stdout
