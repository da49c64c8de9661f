"""The heterogeneous batch (mr_create_batch): chains, trees and piles of
several body counts advanced by one persistent launch per control step
must reproduce each world advanced on its own (the same device code per
environment, so bit for bit), with resets, status codes and after the
autotuner has changed the launch shape and claim order."""

from __future__ import annotations

import numpy as np
import pytest

import numi_lab_b200 as nb

pytestmark = pytest.mark.gpu

PILE_BODIES = (9, 30, 64)


def _worlds(gjk: bool = False):
    seeds = nb.world.pile_seeds_by_body_count(PILE_BODIES)
    worlds = [nb.World("chain7", 40, substeps=1, control_dt=0.005, seed=3),
              nb.World("tree29", 24, substeps=4, velocity_iterations=8, control_dt=0.02, seed=5)]
    worlds += [nb.World("pile", 12, substeps=4, velocity_iterations=8, control_dt=0.02, seed=seeds[n]) for n in PILE_BODIES]
    if gjk:
        # Capsule-box pairs through GJK / EPA: the batch runs per family with
        # the support-mapped free-body kernel.
        worlds.append(nb.World("pile_gjk", 12, substeps=4, velocity_iterations=8, control_dt=0.02, seed=seeds[30]))
    return worlds


def _actions(worlds, steps, seed):
    import torch

    gen = torch.Generator(device="cuda").manual_seed(seed)
    return [0.3 * torch.randn((steps, w.envs, w.action_count), device="cuda", generator=gen) if w.action_count else
            torch.zeros((steps, w.envs, 0), device="cuda") for w in worlds]


def _state(w):
    q, v, m = w.state()
    if w.scene:
        return q, v, m
    return q, v, np.frombuffer(bytes(m), np.uint8)


def _assert_same(a, b):
    for name, x, y in zip(("q", "v", "manifolds"), _state(a), _state(b)):
        np.testing.assert_array_equal(x, y, err_msg=f"{a.source} ({a.envs} envs, seed {a.seed}): {name}")


@pytest.mark.parametrize("gjk", [False, True])
def test_batch_matches_each_world_alone(cuda_device, gjk):
    import torch

    alone, batched = _worlds(gjk), _worlds(gjk)
    try:
        with nb.Batch(batched) as batch:
            shape = batch.launch_shape()
            assert shape["worlds"] == len(batched) and shape["items"] == sum(w.envs for w in batched)
            for rnd in range(3):
                acts = _actions(alone, 5, 100 + rnd)
                masks = [torch.zeros((5, w.envs), dtype=torch.int32, device="cuda") for w in alone]
                if rnd == 1:
                    for m in masks:
                        m[2, ::3] = 1  # some environments reset on the third step
                status = [torch.full((5, w.envs), 77, dtype=torch.int32, device="cuda") for w in alone]
                for w, a, m in zip(alone, acts, masks):
                    w.step(a, reset_mask=m, wait=True)
                batch.step(acts, masks, status)
                torch.cuda.synchronize()
                assert all(int(s.abs().sum()) == 0 for s in status)
                for a, b in zip(alone, batched):
                    _assert_same(a, b)
    finally:
        for w in alone + batched:
            w.close()


def test_tuned_batch_still_matches(cuda_device):
    import torch

    alone, batched = _worlds(), _worlds()
    try:
        with nb.Batch(batched) as batch:
            before = [w.state()[0].copy() for w in batched]
            batch.tune(_actions(batched, 4, 7))
            shape = batch.launch_shape()
            assert shape["tuned"] == 1 and shape["warps_per_block"] in (1, 2, 4) and shape["tuned_step_milliseconds"] > 0
            costs = batch.world_costs()
            assert np.all(costs > 0)
            for w, q in zip(batched, before):
                np.testing.assert_array_equal(w.state()[0], q)  # the tuner put the state back
            acts = _actions(alone, 6, 9)
            for w, a in zip(alone, acts):
                w.step(a, wait=True)
            batch.step(acts)
            torch.cuda.synchronize()
            for a, b in zip(alone, batched):
                _assert_same(a, b)
    finally:
        for w in alone + batched:
            w.close()


def test_batch_rejects_what_it_cannot_run(cuda_device):
    with nb.World("tree29", 4, precision="fp64-inertia") as w64, nb.World("chain7", 4, substeps=1, control_dt=0.005) as c:
        with pytest.raises(nb.MetalRoboError, match="FP32"):
            nb.Batch([c, w64])
        with pytest.raises(nb.MetalRoboError, match="twice"):
            nb.Batch([c, c])
        with nb.Batch([c]) as b:
            import torch

            with pytest.raises(nb.MetalRoboError, match="actions"):
                b.step([torch.zeros((1, 4, 0), device="cuda")])
