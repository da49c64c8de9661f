"""mr_pile_step_no_alloc: pile steps for callers that cannot allocate device
memory (hosts whose own allocator or fixed budget owns the GPU's memory).

The entry point runs the rollout's pile kernel on caller-owned buffers with
its workspace in fixed library arrays.  Two consecutive calls, each several
control steps, must reproduce the rollout handle's trajectory (same kernel,
same inputs) within the per-step parity tolerance of the pile tests, and a
batch above the fixed maximum must be refused with a message.  This file is
collected last so that a stop at its first failure has run every other test.
"""

from __future__ import annotations

import ctypes as ct

import numpy as np
import pytest

import numi_lab_b200 as nb

pytestmark = pytest.mark.gpu

Q_TOL = 1e-5          # tests/test_scene_parity.py, relative to max(1, |x|)
MAX_ENVS = 64         # MR_B200_NO_ALLOC_MAX_ENVS
SCENE_MANIFOLDS, SLOT_WORDS = 128, 57


def _ptr(t) -> ct.c_void_p:
    return ct.c_void_p(t.data_ptr())


def _table_keys(table: np.ndarray) -> list[list[int]]:
    out = []
    for e in range(table.shape[0]):
        keys, c = [], 0
        while c < table.shape[1] and int(table[e, c, 7].view(np.uint32)) != 0:
            keys.append(int(table[e, c, 56].view(np.uint32)))
            c += 1
        out.append(keys)
    return out


def _close(a: np.ndarray, b: np.ndarray) -> None:
    scale = max(1.0, float(np.max(np.abs(b))))
    assert float(np.max(np.abs(a - b))) <= Q_TOL * scale


def test_no_alloc_pile_steps_match_the_rollout_on_two_calls(cuda_device):
    import torch

    lib = nb.native.bindings()
    seed, envs, steps, substeps, iters, dt = 13, 8, 15, 4, 8, 0.02
    with nb.World("pile", envs, substeps=substeps, velocity_iterations=iters, control_dt=dt, seed=seed) as world:
        q0, v0, _ = world.state()
        q = torch.from_numpy(q0).to(cuda_device)
        v = torch.from_numpy(v0).to(cuda_device)
        friction = torch.from_numpy(world.friction_scales()).to(cuda_device)
        manifolds = torch.zeros((envs, SCENE_MANIFOLDS, SLOT_WORDS), device=cuda_device)
        counts = torch.zeros((envs,), dtype=torch.int32, device=cuda_device)
        status = torch.full((steps, envs), 99, dtype=torch.int32, device=cuda_device)
        stream = torch.cuda.current_stream(cuda_device).cuda_stream
        contacts_seen = 0
        for _ in range(2):
            rc = lib.lib.mr_pile_step_no_alloc(
                nb.native.MR_RUN_SOURCE_SYNTHETIC_PILE, seed, envs, _ptr(q), _ptr(v), _ptr(manifolds), _ptr(counts),
                _ptr(friction), _ptr(status), steps, dt, substeps, iters, 0, stream)
            assert rc == 0, lib.last_error()
            world.step(torch.zeros((steps, envs, 0), device=cuda_device), wait=True)
            torch.cuda.synchronize(cuda_device)
            qw, vw, tw = world.state()
            assert int(status.abs().sum()) == 0
            _close(q.cpu().numpy(), qw)
            _close(v.cpu().numpy(), vw)
            table = manifolds.cpu().numpy()
            assert _table_keys(table) == _table_keys(tw)
            assert counts.cpu().numpy().tolist() == [len(k) for k in _table_keys(tw)]
            contacts_seen += int(counts.sum())
        assert contacts_seen > 0  # the piles reached the plane: the contact path ran


def _counters(lib, stream) -> list[int]:
    out = (ct.c_uint32 * 16)()
    rc = lib.lib.mr_pile_step_no_alloc_counters(out, 16, stream)
    assert rc == 0, lib.last_error()
    return list(out)


def _run_against_rollout(lib, cuda_device, source: int, name: str, seed: int, envs: int, steps: int, substeps: int):
    """One no-allocation call of `steps` control steps on fresh buffers,
    compared with a rollout handle of the same world advanced as far."""

    import torch

    iters, dt = 8, 0.02
    with nb.World(name, envs, substeps=substeps, velocity_iterations=iters, control_dt=dt, seed=seed) as world:
        q0, v0, _ = world.state()
        q = torch.from_numpy(q0).to(cuda_device)
        v = torch.from_numpy(v0).to(cuda_device)
        friction = torch.from_numpy(world.friction_scales()).to(cuda_device)
        manifolds = torch.zeros((envs, SCENE_MANIFOLDS, SLOT_WORDS), device=cuda_device)
        counts = torch.zeros((envs,), dtype=torch.int32, device=cuda_device)
        status = torch.full((steps, envs), 99, dtype=torch.int32, device=cuda_device)
        stream = torch.cuda.current_stream(cuda_device).cuda_stream
        rc = lib.lib.mr_pile_step_no_alloc(source, seed, envs, _ptr(q), _ptr(v), _ptr(manifolds), _ptr(counts),
                                           _ptr(friction), _ptr(status), steps, dt, substeps, iters, 0, stream)
        assert rc == 0, lib.last_error()
        world.step(torch.zeros((steps, envs, 0), device=cuda_device), wait=True)
        torch.cuda.synchronize(cuda_device)
        qw, vw, tw = world.state()
        assert int(status.abs().sum()) == 0
        _close(q.cpu().numpy(), qw)
        _close(v.cpu().numpy(), vw)
        assert _table_keys(manifolds.cpu().numpy()) == _table_keys(tw)
        counters = _counters(lib, stream)
        assert counters[0] == 0 and counters[9] == 0  # no failed or skipped environment-steps
        assert counters[6] == 0xFFFFFFFF             # no failing environment
        return counters


def test_no_alloc_follows_world_changes_between_calls(cuda_device):
    """Stack, pile, pile with another substep length, stack again: every
    change of (source, seed, substep length) replaces the resident world
    record, and each call still reproduces its own rollout."""

    lib = nb.native.bindings()
    pile, stack = nb.native.MR_RUN_SOURCE_SYNTHETIC_PILE, nb.native.MR_RUN_SOURCE_SYNTHETIC_STACK
    seen = []
    for source, name, seed, substeps in ((stack, "stack32", 5, 4), (pile, "pile", 13, 4), (pile, "pile", 13, 2),
                                         (stack, "stack32", 5, 4)):
        seen.append(_run_against_rollout(lib, cuda_device, source, name, seed, 6, 12, substeps))
    assert max(c[1] for c in seen) > 0  # contacts were active: the contact path ran


def test_no_alloc_work_run_after_a_world_change_steps_nothing(cuda_device):
    """Work recorded for one world and replayed after another world's record
    was uploaded must not step the caller's buffers with the wrong world: it
    reports MR_STEP_UNSUPPORTED and leaves the state untouched.  Buffers are
    sized for 64-body environments, so every access stays in bounds even for
    a world of another body count."""

    import torch

    lib = nb.native.bindings()
    pile, stack = nb.native.MR_RUN_SOURCE_SYNTHETIC_PILE, nb.native.MR_RUN_SOURCE_SYNTHETIC_STACK
    seed, envs, steps, substeps, iters, dt = 13, 4, 3, 4, 8, 0.02
    with nb.World("pile", envs, substeps=substeps, velocity_iterations=iters, control_dt=dt, seed=seed) as world:
        q0, v0, _ = world.state()
        friction = torch.from_numpy(world.friction_scales()).to(cuda_device)
    nq, nvel = q0.shape[1], v0.shape[1]
    q = torch.zeros((envs, 64 * 7), device=cuda_device)
    v = torch.zeros((envs, 64 * 6), device=cuda_device)
    q.view(-1)[: envs * nq].copy_(torch.from_numpy(q0.reshape(-1)))
    v.view(-1)[: envs * nvel].copy_(torch.from_numpy(v0.reshape(-1)))
    manifolds = torch.zeros((envs, SCENE_MANIFOLDS, SLOT_WORDS), device=cuda_device)
    counts = torch.zeros((envs,), dtype=torch.int32, device=cuda_device)
    status = torch.full((steps, envs), 99, dtype=torch.int32, device=cuda_device)
    side = torch.cuda.Stream(cuda_device)
    args = (seed, envs, _ptr(q), _ptr(v), _ptr(manifolds), _ptr(counts), _ptr(friction), _ptr(status), steps, dt,
            substeps, iters, 0, side.cuda_stream)
    assert lib.lib.mr_pile_step_no_alloc(pile, *args) == 0, lib.last_error()  # uploads the pile's record
    torch.cuda.synchronize(cuda_device)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=side):
        assert lib.lib.mr_pile_step_no_alloc(pile, *args) == 0, lib.last_error()
    torch.cuda.synchronize(cuda_device)
    # Another world replaces the resident record.
    _run_against_rollout(lib, cuda_device, stack, "stack32", 5, 2, 2, 4)
    before_q, before_v = q.clone(), v.clone()
    status.fill_(99)
    graph.replay()
    torch.cuda.synchronize(cuda_device)
    assert torch.equal(q, before_q) and torch.equal(v, before_v)
    assert (status == 12).all()  # MR_STEP_UNSUPPORTED
    counters = _counters(lib, side.cuda_stream)
    assert counters[9] == envs * steps and counters[0] == envs * steps
    del graph


def test_no_alloc_rejects_batches_beyond_its_fixed_workspace(cuda_device):
    import torch

    lib = nb.native.bindings()
    envs = MAX_ENVS + 1
    buf = torch.zeros((envs * 64 * 13 + envs * SCENE_MANIFOLDS * SLOT_WORDS,), device=cuda_device)
    rc = lib.lib.mr_pile_step_no_alloc(nb.native.MR_RUN_SOURCE_SYNTHETIC_PILE, 3, envs, _ptr(buf), _ptr(buf), _ptr(buf),
                                       _ptr(buf), _ptr(buf), None, 1, 0.02, 4, 8, 0,
                                       torch.cuda.current_stream(cuda_device).cuda_stream)
    assert rc == -1
    assert "64" in lib.last_error()
