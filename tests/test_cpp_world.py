"""The C++ world API (include/numi_world.hpp, the shape of the reference's
MetalWorldContext): compiles as C++17; on a GPU, a C++ caller's run() and
resident submissions reproduce the Python World bit for bit."""

from __future__ import annotations

import subprocess
from pathlib import Path

import numpy as np
import pytest

import numi_lab_b200 as nb

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "cpp" / "world_api_check.cpp"


def test_world_api_header_compiles_as_cpp17(tmp_path):
    out = tmp_path / "check.o"
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Wextra", "-Werror", f"-I{ROOT / 'include'}", "-c", str(SRC), "-o", str(out)],
                   check=True)


@pytest.mark.gpu
def test_cpp_world_api_matches_python_world(cuda_device, tmp_path):
    import torch

    lib = nb.native.bindings()
    libdir = Path(lib.path).resolve().parent
    exe = tmp_path / "world_api_check"
    subprocess.run(["g++", "-std=c++17", f"-I{ROOT / 'include'}", str(SRC), "-o", str(exe), f"-L{libdir}", "-lnumi_b200",
                    f"-Wl,-rpath,{libdir}"], check=True)
    tree_out, pile_out, acts_out = tmp_path / "tree.bin", tmp_path / "pile.bin", tmp_path / "actions.bin"
    run = subprocess.run([str(exe), str(tree_out), str(pile_out), str(acts_out)], capture_output=True, text=True)
    assert run.returncode == 0, run.stderr
    envs, steps, na = 4, 6, 29
    acts = np.fromfile(acts_out, np.float32).reshape(steps, envs, na)
    with nb.World("tree29", envs, substeps=4, velocity_iterations=8, control_dt=0.02, seed=11) as world:
        world.step(torch.from_numpy(acts).cuda(), wait=True)
        q, _, _ = world.state()
    np.testing.assert_array_equal(np.fromfile(tree_out, np.float32).reshape(envs, -1), q)
    with nb.World("pile", 3, substeps=4, velocity_iterations=8, control_dt=0.02, seed=10) as world:
        world.step(torch.zeros((10, 3, 0), device="cuda"), wait=True)
        q, _, _ = world.state()
    np.testing.assert_array_equal(np.fromfile(pile_out, np.float32).reshape(3, -1), q)
