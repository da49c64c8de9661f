"""Continuous-batching server: a request's result is the same alone, in a
mix admitted at different ticks, and through the plain rollout handle."""

from __future__ import annotations

import numpy as np
import pytest

import numi_lab_b200 as nb
from numi_lab_b200.serve import poisson_requests, request_actions


def test_poisson_stream_is_seeded_and_bounded():
    a = poisson_requests(200.0, 1.0, seed=3)
    b = poisson_requests(200.0, 1.0, seed=3)
    assert a == b and len(a) > 100
    assert all(1 <= r["env_count"] <= 512 and 10 <= r["horizon"] <= 500 for r in a)
    assert all(r["source"] in ("chain7", "tree29", "pile") for r in a)
    assert {r["source"] for r in a} == {"chain7", "tree29", "pile"}
    arrivals = [r["arrival"] for r in a]
    assert arrivals == sorted(arrivals) and arrivals[-1] < 1.0


def _run_until_done(server, ids):
    done = {}
    for _ in range(1000):
        server.tick()
        for c in server.poll():
            done[c.request_id] = c
        if all(i in done for i in ids):
            return done
    raise AssertionError("requests did not complete")


@pytest.mark.gpu
@pytest.mark.parametrize("steps_per_tick", [1, 4])
def test_request_result_is_the_same_alone_in_a_mix_and_through_a_rollout(cuda_device, steps_per_tick):
    """With one or several control steps per tick (horizons that are not
    multiples of it end mid-tick)."""
    import torch

    seed, envs, horizon = 11, 3, 6
    with nb.Server(model_seed=seed, max_envs_per_source=256, steps_per_tick=steps_per_tick) as server:
        na = server.action_count("tree29")
        acts = (0.3 * np.random.default_rng(1).standard_normal((horizon, envs, na))).astype(np.float32)
        rid = server.submit("tree29", envs, horizon, seed, acts)
        _run_until_done(server, [rid])
        q_alone, v_alone = server.result(rid)

    with nb.Server(model_seed=seed, max_envs_per_source=256, steps_per_tick=steps_per_tick) as server:
        other = []
        for k, (src, n, hz) in enumerate([("chain7", 17, 9), ("tree29", 5, 4), ("tree29", 9, 12), ("chain7", 2, 3)]):
            a = (0.3 * np.random.default_rng(100 + k).standard_normal((hz, n, server.action_count(src)))).astype(np.float32)
            other.append(server.submit(src, n, hz, 1000 + k, a))
        server.tick()
        server.tick()
        rid = server.submit("tree29", envs, horizon, seed, acts)  # joins a running batch
        done = _run_until_done(server, other + [rid])
        q_mix, v_mix = server.result(rid)
        assert done[rid].failed_env_steps == 0
        assert done[rid].latency_seconds >= done[rid].queue_seconds >= 0.0

    np.testing.assert_array_equal(q_mix, q_alone)
    np.testing.assert_array_equal(v_mix, v_alone)

    with nb.World("tree29", envs, substeps=4, velocity_iterations=8, control_dt=0.02, seed=seed) as world:
        world.step(torch.from_numpy(acts).cuda(), wait=True)
        q_w, v_w, _ = world.state()
    np.testing.assert_array_equal(q_w, q_alone)
    np.testing.assert_array_equal(v_w, v_alone)


@pytest.mark.gpu
def test_admission_waits_for_free_slots(cuda_device):
    with nb.Server(model_seed=2, max_envs_per_source=8) as server:
        na = server.action_count("chain7")
        first = server.submit("chain7", 6, 5, 1, np.zeros((5, 6, na), np.float32))
        second = server.submit("chain7", 4, 2, 2, np.zeros((2, 4, na), np.float32))
        reqs, envs = server.tick()
        assert (reqs, envs) == (1, 6)  # 8 slots: the second request waits
        done = _run_until_done(server, [first, second])
        assert done[second].queue_seconds > done[first].queue_seconds
        for rid in (first, second):
            server.result(rid)
        assert server.stats().free_slots == (8 + server.shapes[nb.native.MR_RUN_SOURCE_SYNTHETIC_TREE29][0]
                                             + server.shapes[nb.native.MR_RUN_SOURCE_SYNTHETIC_PILE][0])


@pytest.mark.gpu
def test_pile_request_matches_a_rollout_alone_and_in_a_mix(cuda_device):
    import torch

    seed, envs, horizon = 10, 3, 30  # an 8-body pile, dropped onto the plane
    with nb.Server(model_seed=seed, max_envs_per_source=64) as server:
        assert server.action_count("pile") == 0
        rid = server.submit("pile", envs, horizon, seed, np.zeros((horizon, envs, 0), np.float32))
        _run_until_done(server, [rid])
        q_alone, v_alone = server.result(rid)
    with nb.Server(model_seed=seed, max_envs_per_source=64) as server:
        other = [server.submit("pile", 5, 7, 77, np.zeros((7, 5, 0), np.float32)),
                 server.submit("chain7", 4, 9, 78, np.zeros((9, 4, server.action_count("chain7")), np.float32))]
        server.tick()
        rid = server.submit("pile", envs, horizon, seed, np.zeros((horizon, envs, 0), np.float32))
        done = _run_until_done(server, other + [rid])
        assert done[rid].failed_env_steps == 0
        q_mix, v_mix = server.result(rid)
    np.testing.assert_array_equal(q_mix, q_alone)
    np.testing.assert_array_equal(v_mix, v_alone)
    with nb.World("pile", envs, substeps=4, velocity_iterations=8, control_dt=0.02, seed=seed) as world:
        world.step(torch.zeros((horizon, envs, 0), device="cuda"), wait=True)
        q_w, v_w, _ = world.state()
    np.testing.assert_array_equal(q_w, q_alone)
    np.testing.assert_array_equal(v_w, v_alone)
