"""Writes the reference arm's workload fixtures (run where the CUDA library
is built; no GPU needed):

  tree29_seed2026.npz  the 29-DoF floating-tree contact world (model seed
                       2026) and the reset states (q, v, friction scale) of
                       its first 512 environments for reset seed 2026: the
                       first 512 environments of the 4096-environment
                       contact benchmark.

    python -m oracle.workloads.make_workloads
"""

from __future__ import annotations

import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

from oracle import workloads  # noqa: E402

SEED = 2026
SAMPLE_ENVS = 512


def main() -> None:
    import numi_lab_b200 as nb

    records = nb.compile_model("tree29", SEED)
    q, v, f = nb.sample_reset("tree29", SEED, SEED, 0, SAMPLE_ENVS)
    workloads.save(workloads.path("tree29_seed2026"), records, q=q, v=v, friction=f)
    print(workloads.path("tree29_seed2026"))


if __name__ == "__main__":
    main()
