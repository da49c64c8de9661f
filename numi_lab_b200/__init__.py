"""numi_lab_b200: numi-lab's batched physics microstep on NVIDIA B200 (sm_100a).

The CUDA library ``libnumi_b200.so`` (built in-tree by ``numi_lab_b200.build``)
implements the task-rollout C ABI of ``include/numi_b200.h``; this package is
the thin Python layer over it: ``native`` (ctypes binding), ``world``
(world / reset / step with zero-copy torch tensors; ``Batch``, several
worlds in one launch per control step), ``task`` (task programs for the
task layer) and ``serve`` (continuous-batching request server).
"""

from .native import MetalRoboError, bindings
from .serve import Server
from .world import (Batch, World, compile_model, inspect_policy_pack, inspect_policy_rollout_pack, quality_solve, sample_reset,
                    write_policy_pack, write_policy_rollout_pack)

__all__ = ["Batch", "MetalRoboError", "Server", "World", "bindings", "compile_model", "inspect_policy_pack",
           "inspect_policy_rollout_pack", "quality_solve", "sample_reset", "write_policy_pack", "write_policy_rollout_pack"]
