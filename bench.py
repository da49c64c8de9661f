"""Benchmark: contact env-steps/s of the 29-DoF floating-tree contact
microstep on B200.

Workload (one GPU): 4096 environments of the floating 29-DoF humanoid tree
(box feet + 12 sphere proxies on a ground plane, friction U(0.4, 1.0)),
PD drive targets ~ N(0, 0.3) rad, 20 ms control step = 4 microsteps of 5 ms,
8 temporalCone iterations per microstep, FP32.  One bench step = one advance
of 25 control steps (one CUDA graph); the default 20 timed steps cover the
500-control-step horizon.  Synthetic seeded inputs stand in for a dataset.

Lines printed (rank 0, one JSON line):
  * value: device-resident throughput (actions already in HBM, zero-copy
    torch path), CUDA events on the launching stream around each timed
    advance, L2 flushed (256 MiB write) between timed advances;
  * e2e: the same metric through the reference-shaped C ABI call
    mr_task_rollout_advance with host buffers (actions H2D, status /
    contacts / observations / final q D2H inside the timed region);
  * roofline of the control-step kernel against measured HBM bandwidth;
  * cpu_baseline: the reference's own FP64 CPU contact step
    (stepControlledArticulatedWorldCpu, compiled from its sources) timed on
    this host's cores over a bounded sample of the same workload;
  * plain_aba_chain7: the plain-ABA chain configuration;
  * heterogeneous_mix: 16,384 chains, trees and piles of 8-64 bodies as a
    batch (one persistent launch per horizon) against plain per-config
    kernels (mix_vs_plain) and per-world launches on concurrent streams;
  * serving: Poisson request streams against the continuous-batching
    server (p50 / p99 latency);
  * quality_newton: the same world with the converged FP64 contact solve,
    the solver class of the reference's CPU world step (cpu_baseline), and
    its ratio to cpu_baseline;
  * task_closed_loop: the same world driven by a native policy through the
    locomotion task layer (observe, policy, apply, physics, complete per
    control step).

``--impl reference`` times only that CPU reference (rank 0; other ranks exit).
Multi-GPU (torchrun): one process per GPU; the job is world_size x 4096
environments of one world, each rank stepping its contiguous range; no
collective on the data path; value = total env-steps / max time.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

ENVS = 4096
HORIZON = 25          # control steps per advance (one bench step)
SUBSTEPS = 4
ITERATIONS = 8
CONTROL_DT = 0.02
SEED = 2026
METRIC = "contact env-steps/s"
UNIT = "env-steps/s"
WORKLOAD = "tree29 floating 29-DoF humanoid contact: 4096 envs, 20 ms control = 4 x 5 ms microsteps, 8 temporalCone iterations"
CPU_SAMPLE_ENVS = 512
CPU_SAMPLE_STEPS = 10


def _config(n_gpus: int) -> dict:
    return {
        "workload": WORKLOAD,
        "envs_per_gpu": ENVS,
        "control_steps_per_bench_step": HORIZON,
        "microsteps": SUBSTEPS,
        "velocity_iterations": ITERATIONS,
        "dt_ms": 1000.0 * CONTROL_DT / SUBSTEPS,
        "l2": "flushed (256 MiB write) between timed steps",
        "parallelism": f"replicas x{n_gpus}",
    }


def _algorithmic_bytes_per_env_step(nq: int, nv: int, n_act: int, points: float, manifolds: float) -> float:
    # State in+out, actions in, manifold points / headers in+out, status
    # (no free scene bodies in this world).
    return 8.0 * (nq + nv) + 4.0 * n_act + 2.0 * (48.0 * points + 24.0 * manifolds) + 4.0


def _measured_peaks() -> dict:
    path = ROOT / "MEASURED_PEAKS.json"
    if path.is_file():
        data = json.loads(path.read_text())
        return {"hbm_gbs": float(data["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def _profile_value(key: str, name: str = "control_step_contact_tree29.md") -> float | None:
    """A `key: value` figure of a committed ncu summary under profiles/."""

    path = ROOT / "profiles" / name
    if not path.is_file():
        return None
    for line in path.read_text().splitlines():
        if line.strip().startswith(key + ":"):
            try:
                return float(line.split(":", 1)[1].strip())
            except ValueError:
                return None
    return None


def _issue_peak() -> dict:
    """FP32 FMA peak and warp-instruction issue rate of this device
    (mr_measure_issue_peak, CUDA events)."""

    import ctypes as ct

    import numi_lab_b200 as nb

    lib = nb.bindings()
    tf, ips = ct.c_double(), ct.c_double()
    lib.check(lib.lib.mr_measure_issue_peak(ct.byref(tf), ct.byref(ips)), "mr_measure_issue_peak")
    return {"fma_tflops": tf.value, "warp_instructions_per_s": ips.value}


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    QUERY = (
        "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
        "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
        "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"
    )

    def __init__(self, device_index: int) -> None:
        self.device_index = device_index
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def _smi_id(self) -> str:
        """nvidia-smi's name for the CUDA device: its PCI bus id (CUDA's
        device index need not match nvidia-smi's order, e.g. under
        CUDA_VISIBLE_DEVICES)."""

        try:
            import torch

            props = torch.cuda.get_device_properties(self.device_index)
            bus = f"{props.pci_domain_id:08X}:{props.pci_bus_id:02X}:{props.pci_device_id:02X}.0"
            probe = subprocess.run(["nvidia-smi", f"--id={bus}", "--query-gpu=index", "--format=csv,noheader"],
                                   capture_output=True, text=True, timeout=30)
            if probe.returncode == 0 and probe.stdout.strip():
                return bus
        except (AttributeError, RuntimeError, AssertionError, OSError, subprocess.TimeoutExpired):
            pass
        return str(self.device_index)

    def __enter__(self) -> "ClockSampler":
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self._smi_id()}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.file,
                stderr=subprocess.DEVNULL,
            )
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def __exit__(self, *exc: object) -> None:
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        self.file.flush()
        self.file.seek(0)
        rows = [r.split(",") for r in self.file.read().strip().splitlines() if r.strip()]
        os.unlink(self.file.name)
        sm, smax, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                smax = max(smax, float(r[2]))
                for name, flag in zip(names, r[5:9]):
                    if flag.strip().lower() == "active":
                        reasons.add(name)
            except (ValueError, IndexError):
                continue
        return {
            "sm_mhz": statistics.median(sm) if sm else None,
            "sm_max_mhz": smax or None,
            "reasons": sorted(reasons),
            "samples": len(sm),
        }


REFERENCE_WORKLOAD = "tree29_seed2026"  # oracle/workloads/: records + reset states of the first 512 envs


def _reference_sample(threads: int, actions: np.ndarray) -> dict:
    """Times the reference's own CPU contact step on a bounded sample of the
    workload: the first CPU_SAMPLE_ENVS environments of the benchmark (the
    same compiled world, reset states and per-environment friction, read
    from a committed fixture, so no CUDA library is loaded), stepped for
    actions.shape[0] control steps from their reset states."""

    from oracle import ReferenceBatch, workloads

    records, arrays = workloads.load(workloads.path(REFERENCE_WORKLOAD))
    q = arrays["q"][:CPU_SAMPLE_ENVS].astype(np.float64)
    v = arrays["v"][:CPU_SAMPLE_ENVS].astype(np.float64)
    batch = ReferenceBatch(records, CONTROL_DT / SUBSTEPS, arrays["friction"][:CPU_SAMPLE_ENVS])
    secs, failed = batch.run(q, v, np.ascontiguousarray(actions, np.float32), SUBSTEPS, threads, 1)
    env_steps = CPU_SAMPLE_ENVS * actions.shape[0]
    return {
        "value": env_steps / secs,
        "unit": UNIT,
        "cores": threads,
        "kind": "reference",
        "sample": f"{CPU_SAMPLE_ENVS} envs x {actions.shape[0]} control steps of the same workload from its reset states "
        f"(stepControlledArticulatedWorldCpu with the reference's default quality-Newton contact solve, FP64, per-env friction), "
        f"{failed} substeps failed in the reference (quality-Newton MR_STEP_DID_NOT_CONVERGE)",
        "seconds": secs,
        "failed_substeps": failed,
    }


def _reference_actions(i: int) -> np.ndarray:
    return np.random.default_rng(SEED + i).normal(0.0, 0.3, size=(CPU_SAMPLE_STEPS, CPU_SAMPLE_ENVS, 29)).astype(np.float32)


def run_reference_arm(args, rank: int) -> None:
    if rank != 0:
        return
    from oracle import REF_LIB

    if not REF_LIB.is_file():
        print(json.dumps({"impl": "reference", "unavailable": "reference CPU core library oracle/_ref/libnumiref.so was not built"}))
        return
    threads = os.cpu_count() or 1
    samples = []
    for i in range(args.warmup + args.steps):
        res = _reference_sample(threads, _reference_actions(i))
        if i >= args.warmup:
            samples.append(res)
    value = float(np.mean([s["value"] for s in samples]))
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": float(np.mean([s["seconds"] for s in samples]) * 1e3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded)",
        "config": _config(args.gpus),
        "bench_step": f"{CPU_SAMPLE_ENVS} envs x {CPU_SAMPLE_STEPS} control steps on the host CPU",
        "cpu_baseline": {k: samples[0][k] for k in ("kind", "cores", "sample")} | {"value": value, "unit": UNIT},
        "failed_substeps": int(sum(s["failed_substeps"] for s in samples)),
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


C1_EPISODE = 20  # control steps per episode of the plain-ABA chain


def plain_aba_chain7(device) -> dict:
    """The plain-ABA configuration: 1024 envs of the 7-revolute chain,
    tau ~ N(0, 5), dt = 5 ms, 1000 steps in one advance (one CUDA graph),
    device-resident.  Under that torque scale the chain (no armature, no
    damping) gains energy until its velocities overflow -- after 39 steps at
    the earliest over 1024 environments, 132 at the median -- on the device
    and in the FP64 oracle alike, so the 1000 steps run as 50 episodes of 20
    steps (every environment resets on the first step of an episode) and
    every timed env-step is a successful one."""

    import torch

    import numi_lab_b200 as nb

    envs, steps = 1024, 1000
    with nb.World("chain7", envs, substeps=1, control_dt=0.005, seed=SEED) as world:
        gen = torch.Generator(device=device).manual_seed(SEED)
        acts = 5.0 * torch.randn((steps, envs, world.action_count), device=device, generator=gen)
        masks = torch.zeros((steps, envs), device=device, dtype=torch.int32)
        masks[::C1_EPISODE] = 1
        status = torch.empty((steps, envs), device=device, dtype=torch.int32)
        obs = torch.empty((steps, envs, world.observation_count), device=device)
        for _ in range(3):
            world.step(acts, reset_mask=masks, observations=obs, status=status, wait=True)
        torch.cuda.synchronize(device)
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        world.step(acts, reset_mask=masks, observations=obs, status=status)
        stop.record()
        torch.cuda.synchronize(device)
        ms = start.elapsed_time(stop)
        failed = int((status != 0).sum().item())
    ok = envs * steps - failed
    bytes_per_env_step = 8.0 * (7 + 7) + 4.0 * 7
    peaks = _measured_peaks()
    return {
        "value": ok / (ms / 1e3),
        "unit": UNIT,
        "config": f"chain7: 1024 envs, 1000 steps of 5 ms, tau ~ N(0, 5), FP32, one CUDA-graph advance, "
                  f"episodes of {C1_EPISODE} steps (reset on each episode's first step)",
        "ms": ms,
        "successful_env_steps": ok,
        "failed_env_steps": failed,
        "roofline": {"bound": "hbm", "algorithmic_bytes_per_env_step": bytes_per_env_step,
                     "achieved": bytes_per_env_step * ok / (ms / 1e3) / 1e9, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": bytes_per_env_step * ok / (ms / 1e3) / 1e9 / peaks["hbm_gbs"]},
        "gpu_launches": steps,
    }


def measure_quality(device, steps: int = 5) -> dict:
    """The benchmark world (4096 tree29 environments, seed 2026, 4 x 5 ms
    substeps) with the converged contact solve (MR_SOLVER_QUALITY_NEWTON):
    every substep's contact problem solved in FP64 to scaled optimality
    1e-9 -- the solver class the reference's CPU world step (the
    cpu_baseline / reference arm) runs.  Device-resident, one CUDA-graph
    advance of `steps` control steps after one warm-up advance."""

    import torch

    import numi_lab_b200 as nb

    envs = ENVS
    with nb.World("tree29", envs, substeps=SUBSTEPS, velocity_iterations=ITERATIONS, control_dt=CONTROL_DT, seed=SEED) as world:
        world.set_solver("quality_newton")
        gen = torch.Generator(device=device).manual_seed(SEED)
        acts = 0.3 * torch.randn((steps, envs, world.action_count), device=device, generator=gen)
        status = torch.empty((steps, envs), device=device, dtype=torch.int32)
        world.step(acts, status=status, wait=True)
        torch.cuda.synchronize(device)
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        world.step(acts, status=status)
        stop.record()
        torch.cuda.synchronize(device)
        ms = start.elapsed_time(stop)
        failed = int((status != 0).sum().item())
        diag = world.quality_diagnostics()
    ok = envs * steps - failed
    return {
        "value": ok / (ms / 1e3),
        "unit": UNIT,
        "config": f"tree29: {envs} envs, {steps} control steps of 4 x 5 ms, PD targets ~ N(0, 0.3), converged FP64 contact "
                  "solve (tolerance 1e-9, regularisation floor 1e-6), FP32 state, one CUDA-graph advance",
        "ms_per_control_step": ms / steps,
        "successful_env_steps": ok,
        "failed_env_steps": failed,
        "certificates": diag,
        "gpu_launches": 2 * steps,
    }


def run_quality(args) -> None:
    """One JSON line: the tree29 world with the converged contact solve
    (measure_quality), `--envs` environments (default 4096) and `--steps`
    control steps per timed advance."""

    import torch

    global ENVS
    torch.cuda.set_device(0)
    if args.envs:
        ENVS = args.envs
    line = {"metric": "quality contact env-steps/s", "workload": "quality", **measure_quality(torch.device("cuda", 0),
                                                                                           steps=max(1, args.steps))}
    print(json.dumps(line))


SERVE_RATES = ((2000.0, 1.0), (400.0, 2.0), (100.0, 2.0), (25.0, 2.0))


SERVE_STEPS_PER_TICK = 2  # control steps per server tick (1-8 measured within 3 % of each other)


def measure_serving(rates=SERVE_RATES) -> dict:
    """Poisson request streams (the serving configuration: chain, tree and
    pile worlds, envs log-uniform 1-512, horizons U(10, 500)) against the
    continuous-batching server: served env-steps/s and request latency
    percentiles per arrival rate (each window drained)."""

    import torch

    import numi_lab_b200 as nb
    from numi_lab_b200.serve import poisson_requests, serve_arrivals

    torch.cuda.set_device(0)
    results = {}
    for rate, window in rates:
        with nb.Server(hbm_budget_bytes=120 * 10**9, model_seed=SEED, max_envs_per_source=16384,
                       steps_per_tick=SERVE_STEPS_PER_TICK) as server:
            reqs = poisson_requests(rate, window, seed=SEED + int(rate))
            results[str(int(rate))] = serve_arrivals(server, reqs, drain=True, time_limit_s=300.0)
    head = results[str(int(rates[0][0]))]
    return {
        "value": head["env_steps_per_s"],
        "unit": UNIT,
        "latency_p50_s": head["latency_p50_s"],
        "latency_p99_s": head["latency_p99_s"],
        "queue_p50_s": head["queue_p50_s"],
        "queue_p99_s": head["queue_p99_s"],
        "config": {"workload": f"Poisson arrivals {rates[0][0]:.0f} req/s for {rates[0][1]:.0f} s, worlds chain7 | tree29 | pile, "
                               "envs log-uniform 1-512, horizon U(10, 500), actions N(0, 0.3), 120 GB HBM budget, drained, "
                               f"{SERVE_STEPS_PER_TICK} control steps per tick",
                   "rate_sweep_req_per_s": {k: {kk: v[kk] for kk in ("env_steps_per_s", "latency_p50_s", "latency_p99_s",
                                                                       "queue_p99_s", "completed")}
                                            for k, v in results.items()}},
    }


def run_serving(args) -> None:
    r = measure_serving()
    line = {"metric": "served env-steps/s and request latency (Poisson arrivals)", **r, "higher_is_better": True,
            "data": "synthetic (seeded)", "dtype": "f32"}
    print(json.dumps(line))


PILE_SEED = 60            # a 36-body pile (the mean pile of the heterogeneous mix)
PILE_BODIES = 36


def _pile_cpu_port_sample(records, q0: np.ndarray, v0: np.ndarray, friction: float, steps: int) -> dict:
    """The oracle (FP64 C restatement, one core) on a bounded sample of one
    pile environment: `steps` control steps from a settled state."""

    from oracle import SceneOracle, SceneTable

    oracle = SceneOracle(records, CONTROL_DT / SUBSTEPS, SUBSTEPS, ITERATIONS, 0)
    q = q0.astype(np.float64)
    v = v0.astype(np.float64)
    table = SceneTable()
    for _ in range(60):  # settle (untimed)
        oracle.step(q, v, table, friction)
    t0 = time.perf_counter()
    for _ in range(steps):
        oracle.step(q, v, table, friction)
    secs = time.perf_counter() - t0
    return {"value": steps / secs, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"1 env x {steps} control steps of the {records.world.body_count - 1}-body pile after a 60-step settle, "
                      "oracle/oracle.c (FP64, scalar)"}


def _timed_advances(worlds, args, horizon: int, device, streams=None, episodic=()):
    """Warm-up then `args.steps` timed advances of every world (each on its
    own stream when given); CUDA events on the default stream bracket each
    step after a join of all streams; L2 flushed before each step.  Worlds
    listed in `episodic` reset every environment on the first control step
    of each advance (episodes of `horizon` control steps)."""

    import torch

    flush = torch.empty(256 * 1024 * 1024 // 4, device=device, dtype=torch.float32)
    acts = [torch.zeros((horizon, w.envs, w.action_count), device=device) if w.action_count == 0 else
            0.3 * torch.randn((horizon, w.envs, w.action_count), device=device, generator=torch.Generator(device=device).manual_seed(SEED))
            for w in worlds]
    status = [torch.empty((horizon, w.envs), device=device, dtype=torch.int32) for w in worlds]
    obs = [torch.empty((horizon, w.envs, w.observation_count), device=device) for w in worlds]
    masks = []
    for i, w in enumerate(worlds):
        if i in episodic:
            m = torch.zeros((horizon, w.envs), device=device, dtype=torch.int32)
            m[0] = 1
            masks.append(m)
        else:
            masks.append(None)
    main = torch.cuda.current_stream(device)
    streams = streams or [main] * len(worlds)

    def one_step():
        for w, a, st, ob, sm, mk in zip(worlds, acts, status, obs, streams, masks):
            sm.wait_stream(main)
            with torch.cuda.stream(sm):
                w.step(a, reset_mask=mk, observations=ob, status=st)
        for sm in streams:
            main.wait_stream(sm)

    for _ in range(args.warmup):
        one_step()
    torch.cuda.synchronize(device)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    stops = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    with ClockSampler(device.index if device.index is not None else 0) as clocks:
        for i in range(args.steps):
            flush.fill_(float(i))
            starts[i].record(main)
            one_step()
            stops[i].record(main)
        torch.cuda.synchronize(device)
    failures = [int((st != 0).sum().item()) for st in status]
    ms = float(sum(a.elapsed_time(b) for a, b in zip(starts, stops)))
    return ms, failures, clocks.summary()


def run_pile(args, source: str = "pile") -> None:
    """Free-body piles: 16,384 environments of a 36-body pile of boxes,
    spheres and capsules (source "pile") or of boxes, spheres, capsules and
    cylinders ("cylinder_pile": cylinder pairs take the support-mapped GJK /
    EPA narrowphase) on a plane (settled), 4 x 5 ms substeps, 8 iterations."""

    import torch

    import numi_lab_b200 as nb

    torch.cuda.set_device(0)
    device = torch.device("cuda", 0)
    envs, horizon = args.envs or 16384, 25
    with nb.World(source, envs, substeps=SUBSTEPS, velocity_iterations=ITERATIONS, control_dt=CONTROL_DT, seed=PILE_SEED) as world:
        assert world.scene_bodies == PILE_BODIES
        settle = torch.zeros((100, envs, 0), device=device)
        world.step(settle, wait=True)  # drop and settle (2 s), untimed
        ms, failures, clock_summary = _timed_advances([world], args, horizon, device)
        q_, v_, tab = world.state()
        counts = tab[:, :, 7].view(np.uint32)
        live = counts.astype(np.int64)
        mean_points = float(live.sum(axis=1).mean())
        mean_manifolds = float((live > 0).sum(axis=1).mean())
        cpu = None
        if not args.no_cpu_baseline:
            rq, rv, rf = nb.sample_reset(source, PILE_SEED, PILE_SEED, 0, 1)
            cpu = _pile_cpu_port_sample(world.model(), rq[0], rv[0], float(rf[0]), 40)
    value = envs * horizon * args.steps / (ms / 1e3)
    line = {
        "metric": f"{source.replace('_', ' ')} env-steps/s",
        "value": value,
        "unit": UNIT,
        "n_gpus": 1,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded)",
        "config": {"workload": f"free-body piles: {envs} envs x {PILE_BODIES} "
                               f"{ {'pile': 'boxes/spheres/capsules', 'hull_pile': 'boxes/spheres/capsules/12-vertex convex hulls'}.get(source, 'boxes/spheres/capsules/cylinders')} "
                               "(size U(0.05, 0.3) m, density 500-2000) "
                               "settled on a plane, 20 ms control = 4 x 5 ms substeps, 8 temporalCone iterations, "
                               f"{horizon} control steps per bench step", "l2": "flushed (256 MiB write) between steps"},
        "cpu_baseline": cpu,
        "gpu_launches": horizon * args.steps,
        "clocks": {k: clock_summary[k] for k in ("sm_mhz", "sm_max_mhz", "reasons")},
        "failed_env_steps": sum(failures),
        "mean_active_contacts": mean_points,
        "mean_manifolds": mean_manifolds,
    }
    print(json.dumps(line))


def run_policy(args, task: bool = False) -> None:
    print(json.dumps(measure_closed_loop(args, task)))


def measure_closed_loop(args, task: bool = False) -> dict:
    """Closed loop: 4096 tree29 environments driven by a native policy on
    the device (mr_task_rollout_set_policy) -- a seeded random actor
    obs-256-128-29 (elu, silu, tanh) with observation normalisation and
    Gaussian sampling, plus an obs-64-1 critic -- 25 policy-driven control
    steps per bench step.  The policy reads [q, v] (71 values), or with
    `task` the actor frames of a velocity-tracking locomotion task
    (numi_lab_b200.task.locomotion_task: 99 values) whose observe, apply and
    complete kernels run around every control step."""

    import torch

    import numi_lab_b200 as nb
    from numi_lab_b200 import task as T

    torch.cuda.set_device(0)
    device = torch.device("cuda", 0)
    envs, horizon = args.envs or ENVS, HORIZON
    rng = np.random.default_rng(SEED)

    def dense(sizes, acts):
        return [(rng.normal(0.0, 1.0 / np.sqrt(a), (b, a)).astype(np.float32), rng.normal(0.0, 0.1, b).astype(np.float32), f)
                for (a, b), f in zip(zip(sizes[:-1], sizes[1:]), acts)]

    with nb.World("tree29", envs, substeps=SUBSTEPS, velocity_iterations=ITERATIONS, control_dt=CONTROL_DT, seed=SEED) as world:
        if task:
            q0, _, _ = nb.sample_reset("tree29", SEED, SEED, 0, 1)
            default_q = np.zeros(world.nq, np.float32)
            default_q[2], default_q[6] = q0[0, 2], 1.0
            world.set_task(T.locomotion_task(world.model(), default_q, maximum_episode_steps=500, noise=0.01))
        nobs, na = world.observation_count, world.action_count
        world.set_policy(layers=dense([nobs, 256, 128, na], ["elu", "silu", "tanh"]), critic_layers=dense([nobs, 64, 1], ["relu", "identity"]),
                         revision=1, action_clip=2.5, observation_mean=np.zeros(nobs, np.float32),
                         observation_inverse_std=np.ones(nobs, np.float32), observation_clip=10.0,
                         action_scale=np.full(na, 0.5, np.float32), action_log_std=np.full(na, -1.5, np.float32))
        flush = torch.empty(256 * 1024 * 1024 // 4, device=device, dtype=torch.float32)
        status = None
        for _ in range(args.warmup):  # the same allocation pattern as the timed loop (graphs keyed on buffers)
            _, status = world.step_policy(horizon, wait=False)
        torch.cuda.synchronize(device)
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        stops = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        stream = torch.cuda.current_stream(device)
        failures = 0
        with ClockSampler(0) as clocks:
            for i in range(args.steps):
                flush.fill_(float(i))
                starts[i].record(stream)
                _, status = world.step_policy(horizon, wait=False)
                stops[i].record(stream)
                failures += int((status != 0).sum().item()) if i + 1 == args.steps else 0
            torch.cuda.synchronize(device)
        clock_summary = clocks.summary()
        ms = float(sum(a.elapsed_time(b) for a, b in zip(starts, stops)))
        chains = world.environment_chains
        episodes = None
        if task:
            tr = world.transitions(horizon)
            episodes = {"mean_reward": float(tr["reward"].mean()), "episodes_ended": int(tr["done"].sum()),
                        "timeouts": int(tr["timeout"].sum()), "height_or_tilt": int(np.isin(tr["termination_reason"], (1, 2)).sum())}
    workload = (f"tree29 x {envs} envs driven by a native policy (actor {nobs}-256-128-29, critic {nobs}-64-1, stochastic)"
                + (" through a locomotion task layer (observe, apply, complete kernels per control step)" if task else "")
                + f", {horizon} control steps per bench step")
    line = {
        "metric": "closed-loop env-steps/s",
        "value": envs * horizon * args.steps / (ms / 1e3),
        "unit": UNIT,
        "n_gpus": 1,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded random policy weights)",
        "config": {"workload": workload, "l2": "flushed (256 MiB write) between steps"},
        # policy + control step (+ observe, apply, complete) per chain and control step, one counter per bench step
        "gpu_launches": (5 if task else 2) * chains * horizon * args.steps + args.steps,
        "environment_chains": chains,
        "clocks": {k: clock_summary[k] for k in ("sm_mhz", "sm_max_mhz", "reasons")},
        "failed_env_steps_last_step": failures,
    }
    if task:
        line["last_step_transitions"] = episodes
    return line


def run_task(args) -> None:
    run_policy(args, task=True)


MIX_TOTAL = 16384
MIX_HORIZON = 25


def _mix_worlds(total: int):
    """The heterogeneous mix: 40 % 7-link chains (one 5 ms step per control
    step), 30 % 29-DoF trees and 30 % piles whose body count is drawn per
    environment from U{8..64} (boxes, spheres and capsules of size
    U(0.05, 0.3) m, density 500-2000 kg/m^3, dropped as a heap; capsule-box
    pairs through GJK / EPA); one world per distinct configuration, as the
    reference compiles one topology per context."""

    import numi_lab_b200 as nb

    n_chain = int(0.4 * total)
    n_tree = int(0.3 * total)
    n_pile = total - n_chain - n_tree
    counts = np.random.default_rng(SEED).integers(8, 65, size=n_pile)
    per = {int(n): int((counts == n).sum()) for n in np.unique(counts)}
    seeds = nb.world.pile_seeds_by_body_count(per)
    worlds = [nb.World("chain7", n_chain, substeps=1, control_dt=0.005, seed=SEED),
              nb.World("tree29", n_tree, substeps=SUBSTEPS, velocity_iterations=ITERATIONS, control_dt=CONTROL_DT, seed=SEED)]
    for n in sorted(per):
        worlds.append(nb.World("pile_gjk", per[n], substeps=SUBSTEPS, velocity_iterations=ITERATIONS, control_dt=CONTROL_DT,
                               seed=seeds[n]))
    return worlds, {"chain7": n_chain, "tree29": n_tree, "pile": n_pile, "pile_configs": len(per),
                    "mean_pile_bodies": float(counts.mean())}


def measure_mix(args, device) -> dict:
    """Three arms over the same settled start state: the batch (one
    persistent launch per control step over all worlds, autotuned, one
    CUDA graph per horizon), plain per-config kernels (each world's own
    launches, one world after another, as one context per topology would
    run them) and per-world launches on concurrent streams."""

    import torch

    import numi_lab_b200 as nb

    total = getattr(args, "envs", 0) or MIX_TOTAL
    worlds, mix = _mix_worlds(total)
    horizon = MIX_HORIZON
    try:
        gen = torch.Generator(device=device).manual_seed(SEED)
        acts = [0.3 * torch.randn((horizon, w.envs, w.action_count), device=device, generator=gen) if w.action_count else
                torch.zeros((horizon, w.envs, 0), device=device) for w in worlds]
        # Chains run episodes of one horizon: every chain resets on the
        # first control step of an advance.
        masks = [None] * len(worlds)
        masks[0] = torch.zeros((horizon, worlds[0].envs), dtype=torch.int32, device=device)
        masks[0][0] = 1
        status = [torch.empty((horizon, w.envs), dtype=torch.int32, device=device) for w in worlds]
        for w in worlds[2:]:
            w.step(torch.zeros((100, w.envs, 0), device=device), wait=True)  # drop and settle the piles (2 s), untimed
        start = [w.state() for w in worlds]
        flush = torch.empty(256 * 1024 * 1024 // 4, device=device, dtype=torch.float32)
        main = torch.cuda.current_stream(device)

        def restore():
            torch.cuda.synchronize(device)
            for w, st in zip(worlds, start):
                w.set_state(*st)

        def timed(one_step) -> tuple[float, int]:
            for _ in range(args.warmup):
                one_step()
            torch.cuda.synchronize(device)
            ms = 0.0
            failures = 0
            for i in range(args.steps):
                flush.fill_(float(i))
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(main)
                one_step()
                b.record(main)
                torch.cuda.synchronize(device)
                ms += a.elapsed_time(b)
                failures += sum(int((st != 0).sum().item()) for st in status)
            return ms / args.steps, failures

        env_steps = total * horizon
        # Batched: one launch per control step over every environment.
        restore()
        batch = nb.Batch(worlds)
        try:
            batch.tune([a[:5] for a in acts])
            restore()
            batch_ms, batch_fail = timed(lambda: batch.step(acts, masks, status))
            shape = batch.launch_shape()
        finally:
            batch.close()
        # Plain per-config kernels: each world's own advance, one after another.
        restore()

        def plain_step():
            for w, a, m, st in zip(worlds, acts, masks, status):
                w.step(a, reset_mask=m, status=st)

        plain_ms, plain_fail = timed(plain_step)
        # Per-world launches on concurrent streams.
        restore()
        streams = [torch.cuda.Stream(device) for _ in worlds]

        def concurrent_step():
            for w, a, m, st, sm in zip(worlds, acts, masks, status, streams):
                sm.wait_stream(main)
                with torch.cuda.stream(sm):
                    w.step(a, reset_mask=m, status=st)
            for sm in streams:
                main.wait_stream(sm)

        conc_ms, conc_fail = timed(concurrent_step)
    finally:
        for w in worlds:
            w.close()
    return {
        "value": env_steps / (batch_ms / 1e3),
        "unit": UNIT,
        "plain_per_config_value": env_steps / (plain_ms / 1e3),
        "concurrent_streams_value": env_steps / (conc_ms / 1e3),
        "mix_vs_plain": plain_ms / batch_ms,
        "ms_per_step": {"batched": batch_ms, "plain_per_config": plain_ms, "concurrent_streams": conc_ms},
        "config": {"workload": f"{total} envs: {mix['chain7']} chain7 (5 ms steps, actions N(0, 0.3), one-horizon episodes), "
                               f"{mix['tree29']} tree29 (PD targets N(0, 0.3)), {mix['pile']} settled piles with body counts "
                               f"drawn per env from U{{8..64}} (mean {mix['mean_pile_bodies']:.1f}; {mix['pile_configs']} configurations; "
                               "dropped as heaps; capsule-box pairs through GJK / EPA), "
                               f"{horizon} control steps per bench step", "worlds": len(worlds),
                   "l2": "flushed (256 MiB write) between steps"},
        "batch_launch": shape,
        # Batched: the queue reset plus one persistent launch per horizon (fused)
        # or one per device-code family; plain: one launch per world and step.
        "gpu_launches_per_step": {"batched": 1 if shape["mode"] == 0 else 2, "plain_per_config": horizon * len(worlds)},
        "failed_env_steps": {"batched": batch_fail, "plain_per_config": plain_fail, "concurrent_streams": conc_fail},
    }


def run_mix(args) -> None:
    import torch

    torch.cuda.set_device(0)
    device = torch.device("cuda", 0)
    with ClockSampler(0) as clocks:
        r = measure_mix(args, device)
    clock_summary = clocks.summary()
    line = {
        "metric": "heterogeneous env-steps/s",
        "value": r["value"],
        "unit": UNIT,
        "n_gpus": 1,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": r["ms_per_step"]["batched"],
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded)",
        "config": r["config"],
        "gpu_launches": r["gpu_launches_per_step"]["batched"] * args.steps,
        "clocks": {k: clock_summary[k] for k in ("sm_mhz", "sm_max_mhz", "reasons")},
        **{k: v for k, v in r.items() if k not in ("value", "unit", "config", "ms_per_step")},
        "ms_per_step_by_arm": r["ms_per_step"],
    }
    print(json.dumps(line))


def _stack_energy(records, q: np.ndarray, v: np.ndarray) -> float:
    """Kinetic + potential energy of one scene environment (J)."""

    n = records.world.body_count - 1
    g = -float(records.world.gravity[2])
    e = 0.0
    for b in range(n):
        m = float(records.bodies[b].mass_inverse_mass[0])
        inertia = np.array([float(records.bodies[b].inertia[i][i]) for i in range(3)])
        x, y, z, w = (float(c) for c in q[7 * b + 3: 7 * b + 7])
        rot = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])
        lin = v[6 * b: 6 * b + 3]
        ang = rot.T @ v[6 * b + 3: 6 * b + 6]
        e += 0.5 * m * float(lin @ lin) + 0.5 * float(ang @ (inertia * ang)) + m * g * float(q[7 * b + 2])
    return e


def _tree_energy(oracle, records, q: np.ndarray, v: np.ndarray) -> float:
    """0.5 v^T M(q) v + sum of m g z over the articulated bodies (J)."""

    mass = oracle.mass_matrix(q)
    g = -float(records.world.gravity[2])
    e = 0.5 * float(v @ mass @ v)
    for b in range(records.world.body_count):
        if not records.bodies[b].articulated:
            continue
        wp, _ = oracle.point_jacobian(q, b, np.zeros(3))
        e += float(records.bodies[b].mass_inverse_mass[0]) * g * float(wp[2])
    return e


def _cone_violation_rows(impulses: np.ndarray, mu: np.ndarray) -> float:
    """Largest elliptic-cone violation of impulse rows [.., 3] (normal,
    tangent, bitangent), relative to max(1, normal)."""

    n, t, b = impulses[..., 0], impulses[..., 1], impulses[..., 2]
    scale = np.maximum(1.0, np.abs(n))
    viol = np.maximum(np.maximum(-n, 0.0), np.hypot(t, b) - mu * np.maximum(n, 0.0)) / scale
    return float(viol.max()) if viol.size else 0.0


def run_precision(args) -> None:
    """Precision configuration: 1024 envs of 32-box stacks plus 512 29-DoF
    trees for 10,000 microsteps (2,500 control steps of 4 x 5 ms) in FP32,
    in the compensated-sum mode and, for the trees, in the FP64
    articulated-inertia mode; a seeded subset of
    environments is replayed by the FP64 oracle (the checker) and the line
    reports position drift, energy drift and cone violation against it at
    checkpoints, beside the device throughput."""

    import torch

    import numi_lab_b200 as nb
    from oracle import Oracle, SceneOracle, SceneTable

    torch.cuda.set_device(0)
    device = torch.device("cuda", 0)
    n_stack, n_tree, subset = 1024, 512, 4
    checkpoints = (1, 10, 100, 1000, 2500)
    h = CONTROL_DT / SUBSTEPS
    report: dict = {}
    timing: dict = {}
    # --- stacks (free bodies): FP32 and compensated sums ---
    oracle_rows = None
    for precision in ("fp32", "compensated"):
        with nb.World("stack32", n_stack, substeps=SUBSTEPS, velocity_iterations=ITERATIONS, control_dt=CONTROL_DT, seed=SEED,
                      precision=precision) as world:
            rec = world.model()
            q0, v0, _ = world.state()
            acts = torch.zeros((checkpoints[-1], n_stack, 0), device=device)
            gpu = {}
            done, ms = 0, 0.0
            for cp in checkpoints:
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                world.step(acts[: cp - done], wait=False)
                e1.record()
                torch.cuda.synchronize(device)
                ms += e0.elapsed_time(e1)
                done = cp
                gpu[cp] = world.state()
        timing[f"stack32_{precision}"] = n_stack * checkpoints[-1] / (ms / 1e3)
        if oracle_rows is None:
            # The FP64 replay of the subset, shared by both device modes.
            oracle = SceneOracle(rec, h, SUBSTEPS, ITERATIONS, 0)
            oracle_rows = {}
            for e in range(subset):
                q = q0[e].astype(np.float64)
                v = v0[e].astype(np.float64)
                table = SceneTable()
                oracle_rows[(e, 0)] = (q.copy(), v.copy())
                k = 0
                for cp in checkpoints:
                    while k < cp:
                        oracle.step(q, v, table, 1.0)
                        k += 1
                    oracle_rows[(e, cp)] = (q.copy(), v.copy())
        rows = {cp: {"position_drift_m": 0.0, "energy_drift_gpu_J": 0.0, "energy_drift_oracle_J": 0.0, "cone_violation": 0.0}
                for cp in checkpoints}
        for e in range(subset):
            energy0 = _stack_energy(rec, *oracle_rows[(e, 0)])
            for cp in checkpoints:
                q, v = oracle_rows[(e, cp)]
                gq, gv, gt = gpu[cp]
                r = rows[cp]
                pos_g = gq[e].reshape(-1, 7)[:, :3]
                pos_o = q.reshape(-1, 7)[:, :3]
                r["position_drift_m"] = max(r["position_drift_m"], float(np.abs(pos_g - pos_o).max()))
                r["energy_drift_gpu_J"] = max(r["energy_drift_gpu_J"], abs(_stack_energy(rec, gq[e].astype(np.float64), gv[e].astype(np.float64)) - energy0))
                r["energy_drift_oracle_J"] = max(r["energy_drift_oracle_J"], abs(_stack_energy(rec, q, v) - energy0))
        for cp in checkpoints:
            tab = gpu[cp][2]
            pts = tab[:, :, 8:56].reshape(n_stack, -1, 4, 12)[..., 9:12]
            counts = tab[:, :, 7].view(np.uint32)
            live = np.arange(4)[None, None, :] < counts[:, :, None]
            rows[cp]["cone_violation"] = _cone_violation_rows(pts[live], 0.6)
        report[f"stack32_{precision}"] = rows
    # --- trees: FP32, FP64 articulated inertia, compensated sums ---
    gen = torch.Generator(device=device).manual_seed(SEED)
    for precision in ("fp32", "fp64-inertia", "compensated"):
        with nb.World("tree29", n_tree, substeps=SUBSTEPS, velocity_iterations=ITERATIONS, control_dt=CONTROL_DT, seed=SEED,
                      precision=precision) as world:
            rec = world.model()
            if precision == "fp32":
                tree_actions = 0.3 * torch.randn((checkpoints[-1], n_tree, world.action_count), device=device, generator=gen)
            q0, v0, m0 = world.state()
            fr = world.friction_scales()
            gpu = {}
            done, ms = 0, 0.0
            for cp in checkpoints:
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                world.step(tree_actions[done:cp], wait=False)
                e1.record()
                torch.cuda.synchronize(device)
                ms += e0.elapsed_time(e1)
                done = cp
                gpu[cp] = world.state()
            timing[f"tree29_{precision}"] = n_tree * checkpoints[-1] / (ms / 1e3)
            oracle = Oracle(rec, h, SUBSTEPS, ITERATIONS, 0)
            if precision == "fp32":
                # The FP64 replay of the subset, shared by both device modes
                # (same reset state and actions).
                acts_host = tree_actions[:, :subset].cpu().numpy().astype(np.float64)
                replay = {}
                for e in range(subset):
                    q = q0[e].astype(np.float64)
                    v = v0[e].astype(np.float64)
                    man = oracle.env_manifolds(m0, e)
                    replay[(e, 0)] = (q.copy(), v.copy())
                    k = 0
                    for cp in checkpoints:
                        while k < cp:
                            oracle.control_step(q, v, man, acts_host[k, e], float(fr[e]))
                            k += 1
                        replay[(e, cp)] = (q.copy(), v.copy())
            rows = {cp: {"q_drift": 0.0, "energy_drift_gpu_J": 0.0, "energy_drift_oracle_J": 0.0, "cone_violation": 0.0}
                    for cp in checkpoints}
            for e in range(subset):
                energy0 = _tree_energy(oracle, rec, *replay[(e, 0)])
                for cp in checkpoints:
                    q, v = replay[(e, cp)]
                    gq, gv, _ = gpu[cp]
                    r = rows[cp]
                    r["q_drift"] = max(r["q_drift"], float(np.abs(gq[e] - q).max()))
                    r["energy_drift_gpu_J"] = max(r["energy_drift_gpu_J"],
                                                  abs(_tree_energy(oracle, rec, gq[e].astype(np.float64), gv[e].astype(np.float64)) - energy0))
                    r["energy_drift_oracle_J"] = max(r["energy_drift_oracle_J"], abs(_tree_energy(oracle, rec, q, v) - energy0))
            for cp in checkpoints:
                man = gpu[cp][2]
                imp = np.array([[list(man[i].points[p].impulses) if p < man[i].count else [0.0, 0.0, 0.0] for p in range(4)]
                                for i in range(len(man))]).reshape(n_tree, -1, 4, 3)
                rows[cp]["cone_violation"] = _cone_violation_rows(imp, fr[:, None, None].astype(np.float64))
            report[f"tree29_{precision}"] = rows
    line = {
        "metric": "precision report (drift vs the FP64 oracle)",
        "value": (n_stack + n_tree) * checkpoints[-1] / sum(n * checkpoints[-1] / timing[k] for k, n in
                                                        (("stack32_fp32", n_stack), ("tree29_fp32", n_tree))),
        "unit": UNIT,
        "higher_is_better": True,
        "n_gpus": 1,
        "dtype": "f32",
        "data": "synthetic (seeded)",
        "config": {"workload": f"{n_stack} envs of 32-box stacks (0.1 m, 1 kg, mu 0.6, stack yaw U(0, 2 pi), offsets N(0, 2 mm)) "
                               f"plus {n_tree} tree29 envs (PD targets ~ N(0, 0.3)), {checkpoints[-1]} control steps "
                               f"= {4 * checkpoints[-1]} microsteps of 5 ms; oracle subset {subset} stacks and {subset} trees",
                   "checkpoints_control_steps": list(checkpoints)},
        "throughput_env_steps_per_s": timing,
        "report": report,
        "notes": "value: FP32 stacks and FP32 trees run one after the other; drift is the max over the subset at each "
                 "checkpoint; compensated = FP64 articulated inertia plus Kahan position and impulse sums",
    }
    print(json.dumps(line))


def main() -> None:
    parser = argparse.ArgumentParser()
    parser.add_argument("--gpus", type=int, default=1)
    parser.add_argument("--steps", type=int, default=20)
    parser.add_argument("--warmup", type=int, default=3)
    parser.add_argument("--impl", default="native", choices=["native", "reference"])
    parser.add_argument("--no-cpu-baseline", action="store_true")
    parser.add_argument("--envs", type=int, default=0, help="pile workload: environments (default 16384; smaller for profiling)")
    parser.add_argument("--workload", default="tree29",
                        choices=["tree29", "pile", "cylinder_pile", "hull_pile", "mix", "precision", "policy", "task", "quality"],
                        help="tree29 (the headline), pile (36-body piles), cylinder_pile (36-body piles with cylinders: "
                             "GJK / EPA pairs), mix (chains, trees and piles) or precision (box stacks and trees against the "
                             "FP64 oracle) or policy (tree29 closed loop under a native policy) or quality (tree29 with the "
                             "converged FP64 contact solve)")
    parser.add_argument("--headline-only", action="store_true",
                        help="the 29-DoF contact line without the mix and serving measurements")
    parser.add_argument("--serve", action="store_true",
                        help="serving workload: Poisson request stream, latency percentiles (one JSON line)")
    args = parser.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    world_size = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference_arm(args, rank)
        return
    if args.serve:
        if rank == 0:
            run_serving(args)
        return
    if args.workload != "tree29":
        if rank == 0:
            {"pile": run_pile, "cylinder_pile": lambda a: run_pile(a, "cylinder_pile"),
             "hull_pile": lambda a: run_pile(a, "hull_pile"), "mix": run_mix,
             "precision": run_precision, "policy": run_policy, "task": run_task, "quality": run_quality}[args.workload](args)
        return

    run_headline(args, rank, local_rank, world_size)


def run_headline(args, rank: int, local_rank: int, world_size: int) -> None:
    """The 29-DoF contact workload: device-resident throughput, end to end
    through the host-buffer C ABI, roofline, the reference CPU baseline and
    the plain-ABA chain configuration."""

    import torch

    import numi_lab_b200 as nb
    from numi_lab_b200.sharding import HorizonStats, reduce_stats, shard_range

    torch.cuda.set_device(local_rank)
    dist = None
    if world_size > 1:
        import datetime

        import torch.distributed as dist_mod

        dist_mod.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = dist_mod

    device = torch.device("cuda", local_rank)
    # Weak scaling: the job is world_size x ENVS environments of one world;
    # rank r steps its contiguous range of them (reset states of those global
    # environment indices), with no collective on the data path.
    begin, end = shard_range(ENVS * world_size, rank, world_size)
    world = nb.World("tree29", end - begin, substeps=SUBSTEPS, velocity_iterations=ITERATIONS, control_dt=CONTROL_DT, seed=SEED)
    if begin != 0:
        rq, rv, _ = nb.sample_reset("tree29", SEED, SEED, begin, end - begin)
        world.set_state(rq, rv, as_reset_state=True)  # current and reset state
    envs = world.envs
    gen = torch.Generator(device=device).manual_seed(SEED + rank)
    total_steps = args.warmup + args.steps
    actions = 0.3 * torch.randn((total_steps, HORIZON, envs, world.action_count), device=device, generator=gen)
    obs = torch.empty((HORIZON, envs, world.observation_count), device=device)
    status = torch.empty((args.steps, HORIZON, envs), device=device, dtype=torch.int32)
    flush = torch.empty(256 * 1024 * 1024 // 4, device=device, dtype=torch.float32)
    stream = torch.cuda.current_stream(device)

    def barrier():
        torch.cuda.synchronize(device)
        if dist is not None:
            dist.barrier()

    # Warm-up (graph capture happens on the first advance).
    for i in range(args.warmup):
        world.step(actions[i], observations=obs, status=status[0])
    barrier()
    warm_state = world.state()

    # Device-resident timed region: per-step CUDA events, L2 flushed between steps.
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    stops = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    with ClockSampler(device.index if device.index is not None else 0) as clocks:
        barrier()
        for i in range(args.steps):
            flush.fill_(float(i))
            starts[i].record(stream)
            world.step(actions[args.warmup + i], observations=obs, status=status[i])
            stops[i].record(stream)
        barrier()
    failures = int((status != 0).sum().item())
    clock_summary = clocks.summary()
    step_ms = [s_.elapsed_time(e_) for s_, e_ in zip(starts, stops)]
    total_ms = float(sum(step_ms))
    stats = reduce_stats(HorizonStats(envs * HORIZON * args.steps, failures, total_ms), dist, device)
    max_ms = stats.device_ms
    value = stats.env_steps / (max_ms / 1e3)

    # Contact statistics for the algorithmic byte count (one extra advance
    # with counters, outside the timed region).
    world.step(actions[0], wait=True)
    q_, v_, man_ = world.state()
    counts = np.array([m.count for m in man_], np.int64).reshape(envs, world.pair_count)
    mean_points = float(counts.sum(axis=1).mean())
    mean_manifolds = float((counts > 0).sum(axis=1).mean())

    # End to end through the reference-shaped C ABI with host buffers, over
    # the same number of advances as the device-resident figure: each
    # advance copies its actions from pinned host memory to the device, runs
    # the control steps and reads statuses, contacts, observations and the
    # final q back to host memory, where the caller reads them through the
    # pointers the C ABI returns (valid until the next advance).  L2 is
    # flushed before each advance, inside the timed region.
    world.set_state(*warm_state)
    world.set_state_readback(True)
    host_actions = [actions[args.warmup + i].cpu().pin_memory().numpy() for i in range(args.steps)]
    world.advance_host(host_actions[0], raise_on_failure=False, copy=False)  # warm the host path
    barrier()
    t0 = time.perf_counter()
    for i, a in enumerate(host_actions):
        flush.fill_(float(i))
        torch.cuda.synchronize(device)
        world.advance_host(a, raise_on_failure=False, copy=False)
    e2e_stats = reduce_stats(HorizonStats(envs * HORIZON * len(host_actions), 0, 1e3 * (time.perf_counter() - t0)), dist, device)
    e2e_value = e2e_stats.env_steps / (e2e_stats.device_ms / 1e3)
    h2d = HORIZON * envs * world.action_count * 4
    d2h = HORIZON * envs * (4 + 4 + 4 * world.observation_count) + envs * world.nq * 4
    world.set_state_readback(False)
    del host_actions

    chains = world.environment_chains
    launches_per_step = HORIZON * chains  # one control-step launch per chain per control step
    # The chains' launches of one control step run concurrently, so the
    # kernel is timed per control step (all chains, all environments).
    kernel_ms = total_ms / (args.steps * HORIZON)
    bytes_per_env_step = _algorithmic_bytes_per_env_step(world.nq, world.nv, world.action_count, mean_points, mean_manifolds)
    achieved = bytes_per_env_step * envs / (kernel_ms / 1e3) / 1e9
    peaks = _measured_peaks()
    # DRAM bytes of the control step's launches (both environment chains).
    traffic = _profile_value("traffic_bytes_per_control_step")
    # Issue roofline: the kernel's warp instructions per env-step (from the
    # committed ncu summary) at the measured control-step time, against the
    # measured warp-instruction issue rate of this device.
    issue = _issue_peak()
    inst_per_env_step = _profile_value("warp_instructions_per_env_step")
    issue_achieved = inst_per_env_step * envs / (kernel_ms / 1e3) if inst_per_env_step else None

    launch_shape = world.launch_shape()
    world.close()
    plain = plain_aba_chain7(device) if rank == 0 else None
    # The heterogeneous mix (batched vs plain per-config kernels) and the
    # serving stream, on rank 0 (bounded: a few horizons, one arrival rate).
    mix = serving = quality = task_loop = None
    if rank == 0 and not args.headline_only:
        mix_args = argparse.Namespace(steps=min(args.steps, 5), warmup=3, envs=0)
        mix = measure_mix(mix_args, device)
        mix["steps"] = mix_args.steps
        serving = measure_serving(SERVE_RATES[:1] + SERVE_RATES[2:3])
        quality = measure_quality(device)
        loop = measure_closed_loop(argparse.Namespace(steps=min(args.steps, 5), warmup=3, envs=0), task=True)
        task_loop = {k: loop[k] for k in ("value", "unit", "ms_per_step", "steps", "gpu_launches", "clocks", "last_step_transitions")}
        task_loop["config"] = loop["config"]["workload"]

    cpu = None
    if rank == 0 and world_size == 1 and not args.no_cpu_baseline:
        try:
            cpu = _reference_sample(os.cpu_count() or 1, _reference_actions(0))
            cpu.pop("seconds", None)
        except (FileNotFoundError, OSError, RuntimeError) as exc:
            cpu = {"unavailable": str(exc)}

    if rank == 0:
        step_sorted = sorted(step_ms)
        line = {
            "metric": METRIC,
            "value": value,
            "unit": UNIT,
            "n_gpus": world_size,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": max_ms / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic (seeded)",
            "config": _config(world_size),
            "launch": {**dict(zip(("envs_per_cta", "resident_envs_per_sm"), launch_shape)), "environment_chains": chains},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "advances_timed": args.steps},
            "roofline": {
                "bound": "hbm",
                "achieved": achieved,
                "peak": peaks["hbm_gbs"],
                "unit": "GB/s",
                "frac": achieved / peaks["hbm_gbs"],
                "traffic": traffic,
                "peak_source": peaks["source"],
                "algorithmic_bytes_per_env_step": bytes_per_env_step,
                "kernel_ms_per_control_step": kernel_ms,
                "launches_per_control_step": chains,
                "issue_frac": issue_achieved / issue["warp_instructions_per_s"] if issue_achieved else None,
                "issue": {"achieved_warp_instructions_per_s": issue_achieved,
                          "peak_warp_instructions_per_s": issue["warp_instructions_per_s"],
                          "peak_source": "measured (mr_measure_issue_peak: FP32 FMA chains, CUDA events)",
                          "fma_tflops_peak": issue["fma_tflops"],
                          "warp_instructions_per_env_step": inst_per_env_step,
                          "instructions_source": "profiles/control_step_contact_tree29.md (ncu smsp__inst_executed.sum)"},
            },
            "cpu_baseline": cpu,
            "gpu_launches": launches_per_step * args.steps,
            "clocks": {k: clock_summary[k] for k in ("sm_mhz", "sm_max_mhz", "reasons")},
            "latency_ms_per_advance": {"p50": step_sorted[len(step_sorted) // 2],
                                        "p99": step_sorted[min(len(step_sorted) - 1, int(0.99 * len(step_sorted)))]},
            "failed_env_steps": stats.failed_env_steps,
            "mean_active_contacts": mean_points,
            "mean_manifolds": mean_manifolds,
            "plain_aba_chain7": plain,
            "heterogeneous_mix": mix,
            "serving": serving,
            "quality_newton": quality,
            "task_closed_loop": task_loop,
        }
        if quality and cpu and cpu.get("value"):
            # The reference CPU arm runs the same (converged) solver class.
            quality["vs_cpu_baseline"] = quality["value"] / cpu["value"]
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()

if __name__ == "__main__":
    main()
