"""Builds the in-tree native library ``numi_lab_b200/libnumi_b200.so``.

The library holds every CUDA kernel of the microstep (compiled for sm_100a
only) and the C-ABI entry points declared in ``include/numi_b200.h``.  It is
compiled with nvcc directly; no torch extension machinery is involved, so the
same ``.so`` serves ctypes, cgo-style or C/C++ callers.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PACKAGE_DIR = Path(__file__).resolve().parent
REPO_ROOT = PACKAGE_DIR.parent
CSRC = PACKAGE_DIR / "csrc"
INCLUDE = REPO_ROOT / "include"
LIBRARY = PACKAGE_DIR / "libnumi_b200.so"
BUILD_DIR = PACKAGE_DIR / "_build"

SOURCES = ["model.cpp", "world_step.cu", "scene_step.cu", "mix_step.cu", "policy.cu", "rollout.cu", "serve.cu", "no_alloc.cu",
           "peaks.cu", "quality.cu", "packs.cpp", "task.cu"]
HEADERS = ["model.h", "device_model.h", "layout.h", "dmath.cuh", "runtime.h", "contact.cuh", "scene.h", "policy.h",
           "world_step.cuh", "scene_step.cuh", "mix.h", "audit.cuh", "quality.cuh", "packs.h"]

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    cuda_home = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    candidate = Path(cuda_home) / "bin" / "nvcc"
    if candidate.is_file():
        return str(candidate)
    found = shutil.which("nvcc")
    if found:
        return found
    raise RuntimeError("nvcc not found; set CUDA_HOME")


def _stale(target: Path, inputs: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(p.stat().st_mtime > t for p in inputs)


def build(force: bool = False, verbose: bool = False, ptxas_verbose: bool = False) -> Path:
    """Compiles the library if any source or header is newer than it."""

    inputs = [CSRC / s for s in SOURCES] + [CSRC / h for h in HEADERS] + [INCLUDE / "numi_b200.h", Path(__file__)]
    if not force and not ptxas_verbose and not _stale(LIBRARY, inputs):
        return LIBRARY
    BUILD_DIR.mkdir(exist_ok=True)
    nvcc = nvcc_path()
    common = [
        "-O3",
        "-std=c++17",
        "-lineinfo",
        "-Xcompiler",
        "-fPIC,-fvisibility=hidden",
        f"-I{INCLUDE}",
        f"-I{CSRC}",
        *ARCH_FLAGS,
    ]
    objects = []
    for src in SOURCES:
        obj = BUILD_DIR / (Path(src).stem + ".o")
        cmd = [nvcc, *common, "-c", str(CSRC / src), "-o", str(obj)]
        if ptxas_verbose and src.endswith(".cu"):
            cmd.insert(1, "-Xptxas=-v")
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
        objects.append(str(obj))
    tmp = LIBRARY.with_suffix(".so.tmp")
    link = [nvcc, "-shared", *ARCH_FLAGS, "-o", str(tmp), *objects, "-cudart", "static"]
    if verbose:
        print(" ".join(link), file=sys.stderr)
    subprocess.run(link, check=True)
    os.replace(tmp, LIBRARY)
    return LIBRARY


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_verbose="--ptxas" in sys.argv)
    print(LIBRARY)
