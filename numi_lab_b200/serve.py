"""Continuous-batching rollout server (Python face of mr_create_server ...).

A ``Server`` holds resident environment slots for the 7-DoF chain and the
29-DoF tree on one GPU.  ``submit`` queues a request (world, env count,
horizon, seed, actions); every ``tick`` admits waiting requests into free
slots within the HBM budget (request actions in a preallocated per-world
arena), advances all admitted requests by ``steps_per_tick`` control steps
(one launch per world and step), and retires finished requests; one
synchronisation per tick.  ``poll``
returns completions with queueing delay and latency; ``result`` returns a
finished request's final state.

``poisson_requests`` and ``serve_arrivals`` replay a seeded Poisson request
stream in real time and report latency percentiles and throughput.
"""

from __future__ import annotations

import ctypes as ct
import time
from dataclasses import dataclass

import numpy as np

from . import native
from .native import MetalRoboError

SOURCES = {"chain7": native.MR_RUN_SOURCE_SYNTHETIC_CHAIN7, "tree29": native.MR_RUN_SOURCE_SYNTHETIC_TREE29,
           "pile": native.MR_RUN_SOURCE_SYNTHETIC_PILE}


@dataclass
class Completion:
    request_id: int
    source: int
    env_count: int
    horizon: int
    failed_env_steps: int
    queue_seconds: float
    latency_seconds: float


class Server:
    def __init__(
        self,
        *,
        hbm_budget_bytes: int = 120 * 10**9,
        model_seed: int = 0,
        substeps: int = 4,
        velocity_iterations: int = 8,
        final_velocity_iterations: int = 0,
        control_dt: float = 0.02,
        max_envs_per_source: int = 8192,
        steps_per_tick: int = 1,
        library: native.Bindings | None = None,
    ) -> None:
        self._lib = library or native.bindings()
        cfg = native.ServerConfigC()
        cfg.hbm_budget_bytes = hbm_budget_bytes
        cfg.model_seed = model_seed
        cfg.physics_substeps = substeps
        cfg.velocity_iterations = velocity_iterations
        cfg.final_velocity_iterations = final_velocity_iterations
        cfg.control_steps_per_tick = steps_per_tick
        cfg.control_timestep_seconds = control_dt
        cfg.max_envs_per_source = max_envs_per_source
        handle = self._lib.lib.mr_create_server(ct.byref(cfg))
        if not handle:
            raise MetalRoboError(f"mr_create_server: {self._lib.last_error()}")
        self._handle = ct.c_void_p(handle)
        from .world import compile_model

        self.shapes = {}
        self.state_dims = {}
        for name, sid in SOURCES.items():
            slots, na = ct.c_uint32(), ct.c_uint32()
            self._lib.check(self._lib.lib.mr_server_capacity(self._handle, sid, ct.byref(slots), ct.byref(na)), "capacity")
            self.shapes[sid] = (int(slots.value), int(na.value))
            w = compile_model(sid, model_seed, library=self._lib).world
            self.state_dims[sid] = (int(w.nq), int(w.nv))
        self._dims = {}

    def close(self) -> None:
        if getattr(self, "_handle", None) and self._handle.value:
            self._lib.lib.mr_server_destroy(self._handle)
            self._handle = ct.c_void_p(None)

    def __enter__(self) -> "Server":
        return self

    def __exit__(self, *exc: object) -> None:
        self.close()

    def action_count(self, source: str | int) -> int:
        return self.shapes[SOURCES.get(source, source)][1]

    def submit(self, source: str | int, env_count: int, horizon: int, seed: int, actions: np.ndarray) -> int:
        sid = SOURCES.get(source, source)
        acts = np.ascontiguousarray(actions, np.float32)
        req = native.ServerRequestC()
        req.source = sid
        req.env_count = env_count
        req.horizon = horizon
        req.seed = seed
        req.actions = acts.ctypes.data_as(ct.POINTER(ct.c_float))
        rid = ct.c_uint64()
        self._lib.check(self._lib.lib.mr_server_submit(self._handle, ct.byref(req), ct.byref(rid)), "mr_server_submit")
        self._dims[int(rid.value)] = (sid, env_count)
        return int(rid.value)

    def tick(self) -> tuple[int, int]:
        reqs, envs = ct.c_uint32(), ct.c_uint32()
        self._lib.check(self._lib.lib.mr_server_tick(self._handle, ct.byref(reqs), ct.byref(envs)), "mr_server_tick")
        return int(reqs.value), int(envs.value)

    def poll(self) -> list[Completion]:
        out = (native.ServerCompletionC * 256)()
        done: list[Completion] = []
        while True:
            n = ct.c_uint32()
            self._lib.check(self._lib.lib.mr_server_poll(self._handle, out, 256, ct.byref(n)), "mr_server_poll")
            for i in range(n.value):
                c = out[i]
                done.append(Completion(int(c.request_id), int(c.source), int(c.env_count), int(c.horizon),
                                       int(c.failed_env_steps), float(c.queue_seconds), float(c.latency_seconds)))
            if n.value < 256:
                return done

    def result(self, request_id: int, *, release: bool = True) -> tuple[np.ndarray, np.ndarray]:
        sid, envs = self._dims[request_id]
        nq, nv = self.state_dims[sid]
        q = np.zeros((envs, nq), np.float32)
        v = np.zeros((envs, nv), np.float32)
        self._lib.check(self._lib.lib.mr_server_copy_result(
            self._handle, request_id, q.ctypes.data_as(ct.POINTER(ct.c_float)), q.size,
            v.ctypes.data_as(ct.POINTER(ct.c_float)), v.size), "mr_server_copy_result")
        if release:
            self._lib.check(self._lib.lib.mr_server_release(self._handle, request_id), "mr_server_release")
            del self._dims[request_id]
        return q, v

    def stats(self) -> native.ServerStatsC:
        s = native.ServerStatsC()
        self._lib.check(self._lib.lib.mr_server_stats(self._handle, ct.byref(s)), "mr_server_stats")
        return s


def poisson_requests(rate_hz: float, window_s: float, seed: int, *, max_envs: int = 512, horizon: tuple[int, int] = (10, 500),
                     sources: tuple[str, ...] = ("chain7", "tree29", "pile")) -> list[dict]:
    """Seeded Poisson request stream: arrival time, world, env count
    (log-uniform 1..max_envs), horizon U(lo, hi), seed; actions are drawn
    N(0, 0.3) at submission (``request_actions``)."""

    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate_hz)
        if t >= window_s:
            return out
        envs = int(np.clip(np.round(np.exp(rng.uniform(0.0, np.log(max_envs)))), 1, max_envs))
        out.append({
            "arrival": t,
            "source": sources[int(rng.integers(len(sources)))],
            "env_count": envs,
            "horizon": int(rng.integers(horizon[0], horizon[1] + 1)),
            "seed": int(rng.integers(1 << 62)),
        })


def request_actions(req: dict, action_count: int) -> np.ndarray:
    rng = np.random.default_rng(req["seed"] ^ 0x5EED)
    return (0.3 * rng.standard_normal((req["horizon"], req["env_count"], action_count))).astype(np.float32)


def serve_arrivals(server: Server, requests: list[dict], *, drain: bool = True, time_limit_s: float = 120.0) -> dict:
    """Replays the arrivals in real time against ``server``; returns latency
    percentiles of completed requests, queueing delay and env-steps/s."""

    pending = sorted(requests, key=lambda r: r["arrival"])
    actions = [request_actions(r, server.action_count(r["source"])) for r in pending]
    t0 = time.perf_counter()
    i, submitted, completions = 0, 0, []
    env_steps_done = 0
    while True:
        now = time.perf_counter() - t0
        while i < len(pending) and pending[i]["arrival"] <= now:
            r = pending[i]
            server.submit(r["source"], r["env_count"], r["horizon"], r["seed"], actions[i])
            i += 1
            submitted += 1
        reqs, envs = server.tick()
        env_steps_done += envs
        for c in server.poll():
            completions.append(c)
            server.result(c.request_id, release=True)
        if i >= len(pending) and (not drain or len(completions) == submitted):
            break
        if now > time_limit_s:
            break
        if reqs == 0 and i < len(pending):
            time.sleep(max(0.0, min(0.001, pending[i]["arrival"] - now)))
    elapsed = time.perf_counter() - t0
    lat = np.array([c.latency_seconds for c in completions]) if completions else np.zeros(1)
    queue = np.array([c.queue_seconds for c in completions]) if completions else np.zeros(1)
    return {
        "submitted": submitted,
        "completed": len(completions),
        "elapsed_s": elapsed,
        "env_steps": env_steps_done,
        "env_steps_per_s": env_steps_done / elapsed,
        "latency_p50_s": float(np.percentile(lat, 50)),
        "latency_p99_s": float(np.percentile(lat, 99)),
        "queue_p50_s": float(np.percentile(queue, 50)),
        "queue_p99_s": float(np.percentile(queue, 99)),
        "failed_env_steps": int(sum(c.failed_env_steps for c in completions)),
    }
