"""ORACLE — test infrastructure only.

Workload fixtures for the reference CPU arm: the compiled records of a
synthetic world and the reset states of a sample of its environments, saved
by ``make_workloads.py`` so that timing the reference's CPU core needs
neither this project's CUDA library nor a GPU.  The records are stored as
the raw bytes of the C-ABI structs (``MRModel*C`` in include/numi_b200.h).
"""

from __future__ import annotations

import ctypes as ct
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent

_FIELDS = ("joints", "bodies", "dofs", "shapes", "materials", "pairs")


def path(name: str) -> Path:
    return HERE / f"{name}.npz"


def save(path_: Path, records, **arrays: np.ndarray) -> None:
    blobs = {"world": np.frombuffer(bytes(records.world), np.uint8)}
    for f in _FIELDS:
        blobs[f] = np.frombuffer(bytes(getattr(records, f)), np.uint8)
    np.savez_compressed(path_, **blobs, **arrays)


def load(path_: Path):
    """(records, arrays): ctypes records rebuilt from the struct bytes, and
    the saved arrays.  Only the Python struct definitions of the C ABI are
    used; no native library is loaded."""

    from numi_lab_b200 import native
    from numi_lab_b200.world import ModelRecords

    data = np.load(path_)
    world = native.ModelWorldC.from_buffer_copy(data["world"].tobytes())
    types = {"joints": native.ModelJointC, "bodies": native.ModelBodyC, "dofs": native.ModelDofC,
             "shapes": native.ModelShapeC, "materials": native.ModelMaterialC, "pairs": native.ModelPairC}
    parts = {}
    for f in _FIELDS:
        raw = data[f].tobytes()
        n = len(raw) // ct.sizeof(types[f])
        parts[f] = (types[f] * n).from_buffer_copy(raw)
    records = ModelRecords(world=world, **parts)
    arrays = {k: data[k] for k in data.files if k != "world" and k not in _FIELDS}
    return records, arrays
