"""World-size-2 gloo test of the multi-GPU host logic on CPU: environment
shards are disjoint and complete, a sharded run of the oracle equals the
unsharded run bit for bit (environments are independent), and the statistics
reduction sums env-steps and takes the max time over ranks."""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from numi_lab_b200.sharding import HorizonStats, reduce_stats, shard_range


def test_shard_ranges_partition_the_envs():
    for total in (1, 7, 4096, 4099):
        for world in (1, 2, 3, 8):
            if world > total:
                continue
            ranges = [shard_range(total, r, world) for r in range(world)]
            assert ranges[0][0] == 0 and ranges[-1][1] == total
            for (a, b), (c, d) in zip(ranges, ranges[1:]):
                assert b == c and b > a
    with pytest.raises(ValueError):
        shard_range(10, 2, 2)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rollout(envs: slice, steps: int) -> np.ndarray:
    import numi_lab_b200 as nb
    from oracle import Oracle

    rec = nb.compile_model("chain7", 5)
    oracle = Oracle(rec, 0.005, 1, 0, 0)
    q, v, _ = nb.sample_reset("chain7", 5, 5, envs.start, envs.stop - envs.start)
    rng = np.random.default_rng(99)
    actions = rng.normal(0.0, 5.0, size=(steps, 16, 7))[:, envs]
    out = []
    for e in range(q.shape[0]):
        qe, ve = q[e].astype(np.float64), v[e].astype(np.float64)
        for k in range(steps):
            oracle.control_step(qe, ve, None, actions[k, e], 1.0)
        out.append(np.concatenate([qe, ve]))
    return np.array(out)


def _worker(rank: int, world: int, port: int, queue) -> None:
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        begin, end = shard_range(16, rank, world)
        result = _rollout(slice(begin, end), 3)
        stats = reduce_stats(HorizonStats((end - begin) * 3, rank, 10.0 + rank), dist)
        queue.put((rank, begin, result, stats))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_rank_sharded_rollout_equals_single_process():
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, queue)) for r in range(2)]
    for p in procs:
        p.start()
    results = [queue.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    results.sort(key=lambda x: x[0])
    sharded = np.concatenate([r[2] for r in results])
    single = _rollout(slice(0, 16), 3)
    np.testing.assert_array_equal(sharded, single)
    for _, _, _, stats in results:
        assert stats.env_steps == 16 * 3
        assert stats.failed_env_steps == 1
        assert stats.device_ms == 11.0
