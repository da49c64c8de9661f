"""world / reset / step API over the numi_b200 task-rollout C ABI.

``World.step`` is the zero-copy path: actions, reset masks and observations
are torch CUDA tensors whose device pointers go straight to the native
library (``mr_task_rollout_advance_device``); work is ordered on torch's
current stream.  ``World.advance_host`` is the reference-shaped path
(``mr_task_rollout_advance``: host spans in, handle-owned results out).

Every physics computation runs in the CUDA library; this module only marshals
pointers and shapes.  A missing library raises ``FileNotFoundError``.
"""

from __future__ import annotations

import ctypes as ct
import os
from dataclasses import dataclass
from typing import Any, Sequence

import numpy as np

from . import native
from .native import MetalRoboError

SOURCES = {
    "chain7": native.MR_RUN_SOURCE_SYNTHETIC_CHAIN7,
    "tree29": native.MR_RUN_SOURCE_SYNTHETIC_TREE29,
    "pile": native.MR_RUN_SOURCE_SYNTHETIC_PILE,
    "stack32": native.MR_RUN_SOURCE_SYNTHETIC_STACK,
    "cylinder_pile": native.MR_RUN_SOURCE_SYNTHETIC_CYLINDER_PILE,
    "pile_gjk": native.MR_RUN_SOURCE_SYNTHETIC_PILE_GJK,
    "hull_pile": native.MR_RUN_SOURCE_SYNTHETIC_HULL_PILE,
}
SCENE_MANIFOLDS = 128      # manifold slots per scene environment
SCENE_SLOT_WORDS = 57      # MRManifoldC words + pair key


def _source_id(source: str | int) -> int:
    if isinstance(source, str):
        if source not in SOURCES:
            raise ValueError(f"unknown source {source!r}; expected one of {sorted(SOURCES)}")
        return SOURCES[source]
    return int(source)


@dataclass
class ModelRecords:
    """Compiled world records (ctypes arrays) of one synthetic world."""

    world: native.ModelWorldC
    joints: Any
    bodies: Any
    dofs: Any
    shapes: Any
    materials: Any
    pairs: Any
    hull_vertices: Any = None  # [n][4] float32 unit-scale hull vertices (convex shapes), or None

    def view(self) -> native.ModelViewC:
        v = native.ModelViewC()
        v.world = self.world
        v.joints = ct.cast(self.joints, ct.POINTER(native.ModelJointC))
        v.bodies = ct.cast(self.bodies, ct.POINTER(native.ModelBodyC))
        v.dofs = ct.cast(self.dofs, ct.POINTER(native.ModelDofC))
        v.shapes = ct.cast(self.shapes, ct.POINTER(native.ModelShapeC))
        v.materials = ct.cast(self.materials, ct.POINTER(native.ModelMaterialC))
        v.pairs = ct.cast(self.pairs, ct.POINTER(native.ModelPairC))
        if self.hull_vertices is not None and len(self.hull_vertices):
            v.hull_vertices = self.hull_vertices.ctypes.data_as(ct.POINTER(ct.c_float))
            v.hull_vertex_capacity = len(self.hull_vertices)
        return v


def _alloc_records(world: native.ModelWorldC) -> ModelRecords:
    return ModelRecords(
        world=world,
        joints=(native.ModelJointC * max(world.joint_count, 1))(),
        bodies=(native.ModelBodyC * max(world.body_count, 1))(),
        dofs=(native.ModelDofC * max(world.nv, 1))(),
        shapes=(native.ModelShapeC * max(world.shape_count, 1))(),
        materials=(native.ModelMaterialC * max(world.material_count, 1))(),
        pairs=(native.ModelPairC * max(world.pair_count, 1))(),
    )


def compile_model(source: str | int, seed: int, *, library: native.Bindings | None = None) -> ModelRecords:
    """Compiles a synthetic world on the host (no GPU needed)."""

    lib = library or native.bindings()
    sid = _source_id(source)
    probe = native.ModelViewC()
    lib.check(lib.lib.mr_compile_synthetic_model(sid, seed, ct.byref(probe)), "mr_compile_synthetic_model")
    records = _alloc_records(probe.world)
    if probe.hull_vertex_count:
        records.hull_vertices = np.zeros((probe.hull_vertex_count, 4), np.float32)
    view = records.view()
    lib.check(lib.lib.mr_compile_synthetic_model(sid, seed, ct.byref(view)), "mr_compile_synthetic_model")
    records.world = view.world
    return records


def sample_reset(
    source: str | int,
    model_seed: int,
    reset_seed: int,
    env_begin: int,
    env_count: int,
    *,
    library: native.Bindings | None = None,
) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Reset states (q, v, friction scale) a rollout samples for these envs."""

    lib = library or native.bindings()
    sid = _source_id(source)
    world = compile_model(sid, model_seed, library=lib).world
    q = np.zeros((env_count, world.nq), np.float32)
    v = np.zeros((env_count, world.nv), np.float32)
    f = np.zeros((env_count,), np.float32)
    lib.check(
        lib.lib.mr_sample_synthetic_reset(
            sid,
            model_seed,
            reset_seed,
            env_begin,
            env_count,
            q.ctypes.data_as(ct.POINTER(ct.c_float)),
            v.ctypes.data_as(ct.POINTER(ct.c_float)),
            f.ctypes.data_as(ct.POINTER(ct.c_float)),
        ),
        "mr_sample_synthetic_reset",
    )
    return q, v, f


def pile_seeds_by_body_count(bodies: Sequence[int], first_seed: int = 0) -> dict[int, int]:
    """The first model seed (from `first_seed` on) whose synthetic pile has
    each requested body count (8-64): the pile source draws its body count
    from the seed."""

    want = {int(n) for n in bodies}
    if not want <= set(range(8, 65)):
        raise ValueError("pile body counts are 8-64")
    out: dict[int, int] = {}
    seed = first_seed
    while want - set(out):
        n = int(compile_model("pile", seed).world.body_count) - 1
        if n in want and n not in out:
            out[n] = seed
        seed += 1
    return out


def policy_pack_c(
    layers: Sequence[tuple[np.ndarray, np.ndarray | None, str]],
    *,
    revision: int,
    action_clip: float,
    policy_id: str = "policy",
    observation_mean: np.ndarray | None = None,
    observation_inverse_std: np.ndarray | None = None,
    observation_clip: float = 0.0,
    critic_layers: Sequence[tuple[np.ndarray, np.ndarray | None, str]] = (),
    critic_observation_mean: np.ndarray | None = None,
    critic_observation_inverse_std: np.ndarray | None = None,
    action_log_std: np.ndarray | None = None,
    action_bias: np.ndarray | None = None,
    action_scale: np.ndarray | None = None,
    contract: tuple[int, int, int, int, int] = (0, 0, 0, 0, 0),
):
    """An MRPolicyPackC over the given arrays, and the list of objects that
    must outlive it.  `layers` are (weights [out][in], bias [out] or None,
    activation name); `contract` is (version, world, task, observation,
    action fingerprints)."""

    keep: list[Any] = []

    def arr(a):
        if a is None:
            return None, 0
        a = np.ascontiguousarray(a, np.float32).reshape(-1)
        keep.append(a)
        return a.ctypes.data_as(ct.POINTER(ct.c_float)), a.size

    def dense(spec):
        out = (native.PolicyDenseLayerC * max(len(spec), 1))()
        for i, (w, b, act) in enumerate(spec):
            w = np.asarray(w, np.float32)
            wp, wn = arr(w)
            bp, bn = arr(b)
            out[i] = native.PolicyDenseLayerC(w.shape[1], w.shape[0], native.POLICY_ACTIVATIONS[act], wp, wn, bp, bn)
        keep.append(out)
        return out, len(spec)

    pk = native.PolicyPackC()
    ident = policy_id.encode()
    keep.append(ident)
    pk.id = ident
    pk.revision = int(revision)
    (pk.contract_version, pk.world_fingerprint, pk.task_fingerprint, pk.observation_fingerprint,
     pk.action_fingerprint) = (int(x) for x in contract)
    pk.layers, pk.layer_count = dense(layers)
    if critic_layers:
        pk.critic_layers, pk.critic_layer_count = dense(critic_layers)
    pk.observation_mean, pk.observation_mean_count = arr(observation_mean)
    pk.observation_inverse_standard_deviation, pk.observation_inverse_standard_deviation_count = arr(observation_inverse_std)
    pk.critic_observation_mean, pk.critic_observation_mean_count = arr(critic_observation_mean)
    (pk.critic_observation_inverse_standard_deviation,
     pk.critic_observation_inverse_standard_deviation_count) = arr(critic_observation_inverse_std)
    pk.action_log_standard_deviation, pk.action_log_standard_deviation_count = arr(action_log_std)
    pk.action_bias, pk.action_bias_count = arr(action_bias)
    pk.action_scale, pk.action_scale_count = arr(action_scale)
    pk.observation_clip = float(observation_clip)
    pk.action_clip = float(action_clip)
    return pk, keep


def write_policy_pack(path: str | os.PathLike[str], layers, *, library: native.Bindings | None = None, **fields) -> None:
    """Writes a PolicyPack file (mr_write_policy_pack); arguments as
    policy_pack_c.  The pack needs an exact contract (version 1, non-zero
    fingerprints)."""

    lib = library or native.bindings()
    pk, keep = policy_pack_c(layers, **fields)
    lib.check(lib.lib.mr_write_policy_pack(ct.byref(pk), os.fsencode(path)), "mr_write_policy_pack")
    del keep


def inspect_policy_pack(path: str | os.PathLike[str], *, library: native.Bindings | None = None) -> tuple[dict, np.ndarray]:
    """Reads a PolicyPack file without a device (mr_policy_pack_inspect):
    its fields and every FP32 table concatenated in file order."""

    lib = library or native.bindings()
    info = native.PolicyPackInfoC()
    lib.check(lib.lib.mr_policy_pack_inspect(os.fsencode(path), ct.byref(info), None, 0), "mr_policy_pack_inspect")
    params = np.zeros(int(info.parameter_count), np.float32)
    lib.check(lib.lib.mr_policy_pack_inspect(os.fsencode(path), ct.byref(info),
                                             params.ctypes.data_as(ct.POINTER(ct.c_float)), params.size),
              "mr_policy_pack_inspect")
    fields = {name: getattr(info, name) for name, _ in native.PolicyPackInfoC._fields_}
    fields["id"] = info.id.decode()
    return fields, params


def policy_rollout_pack_c(*, id: str, task_fingerprint: int, policy_fingerprint: int, policy_revision: int, environment_count: int,
                          control_step_count: int, actor_observations, latents, log_probabilities, values, bootstrap_values,
                          transitions, critic_observations=None, teacher_actions=None, motion_features=None,
                          actor_observation_count: int | None = None, critic_observation_count: int | None = None,
                          action_count: int | None = None, motion_feature_count: int = 0):
    """(MRPolicyRolloutPackC, keepalive) from arrays: observations
    [step][env][features], latents [step][env][actions], log-probabilities
    and values [step][env], bootstrap values [env], transitions a ctypes
    MRTaskTransitionC array [step * env]."""

    keep: list[Any] = []

    def arr(a, width=None):
        if a is None:
            return None, 0
        x = np.ascontiguousarray(a, np.float32).reshape(-1)
        keep.append(x)
        return x.ctypes.data_as(ct.POINTER(ct.c_float)), x.size

    obs = np.asarray(actor_observations, np.float32)
    lat = np.asarray(latents, np.float32)
    b = native.PolicyRolloutBatchC()
    b.control_step_count = control_step_count
    b.actor_observations, b.actor_observation_count = arr(obs)
    b.critic_observations, b.critic_observation_count = arr(obs if critic_observations is None else critic_observations)
    b.motion_features, b.motion_feature_count = arr(motion_features)
    b.teacher_actions, b.teacher_action_count = arr(teacher_actions)
    b.latents, b.latent_count = arr(lat)
    b.log_probabilities, b.log_probability_count = arr(log_probabilities)
    b.values, b.value_count = arr(values)
    b.bootstrap_values, b.bootstrap_value_count = arr(bootstrap_values)
    keep.append(transitions)
    b.transitions = ct.cast(transitions, ct.POINTER(native.TaskTransitionC))
    b.transition_count = len(transitions)
    keep.append(b)
    c = native.PolicyRolloutPackC()
    ident = id.encode()
    keep.append(ident)
    c.id = ident
    c.task_fingerprint, c.policy_fingerprint, c.policy_revision = task_fingerprint, policy_fingerprint, policy_revision
    c.environment_count = environment_count
    c.actor_observation_count = obs.shape[-1] if actor_observation_count is None else actor_observation_count
    crit = obs if critic_observations is None else np.asarray(critic_observations)
    c.critic_observation_count = crit.shape[-1] if critic_observation_count is None else critic_observation_count
    c.action_count = lat.shape[-1] if action_count is None else action_count
    c.motion_feature_count = motion_feature_count
    c.batch = ct.pointer(b)
    return c, keep


def write_policy_rollout_pack(path: str | os.PathLike[str], *, library: native.Bindings | None = None, **fields) -> None:
    """Writes a PolicyRolloutPack (mr_write_policy_rollout_pack)."""

    lib = library or native.bindings()
    c, keep = policy_rollout_pack_c(**fields)
    lib.check(lib.lib.mr_write_policy_rollout_pack(ct.byref(c), os.fsencode(path)), "mr_write_policy_rollout_pack")
    del keep


def inspect_policy_rollout_pack(path: str | os.PathLike[str], *, library: native.Bindings | None = None) -> tuple[dict, np.ndarray]:
    """(fields, actor observations + latents + log-probabilities + values +
    bootstrap values concatenated) of a PolicyRolloutPack file."""

    lib = library or native.bindings()
    info = native.PolicyRolloutPackInfoC()
    lib.check(lib.lib.mr_policy_rollout_pack_inspect(os.fsencode(path), ct.byref(info), None, 0), "mr_policy_rollout_pack_inspect")
    samples = int(info.environment_count) * int(info.control_step_count)
    count = samples * (int(info.actor_observation_count) + int(info.action_count) + 2) + int(info.environment_count)
    params = np.zeros(count, np.float32)
    lib.check(lib.lib.mr_policy_rollout_pack_inspect(os.fsencode(path), ct.byref(info), params.ctypes.data_as(ct.POINTER(ct.c_float)),
                                                     params.size), "mr_policy_rollout_pack_inspect")
    fields = {name: getattr(info, name) for name, _ in native.PolicyRolloutPackInfoC._fields_}
    fields["id"] = info.id.decode()
    return fields, params


def inspect_task_pack(path: str | os.PathLike[str], *, library: native.Bindings | None = None) -> dict:
    """Table counts and episode constants of a TaskPack file (mr_task_pack_inspect)."""

    lib = library or native.bindings()
    info = native.TaskPackInfoC()
    lib.check(lib.lib.mr_task_pack_inspect(os.fsencode(path), ct.byref(info)), "mr_task_pack_inspect")
    fields = {name: getattr(info, name) for name, _ in native.TaskPackInfoC._fields_}
    fields["id"] = info.id.decode()
    return fields


def rewrite_task_pack(source: str | os.PathLike[str], destination: str | os.PathLike[str], *,
                      library: native.Bindings | None = None) -> None:
    """Reads a TaskPack, checks the writer's artifact rules, writes it again (mr_task_pack_rewrite)."""

    lib = library or native.bindings()
    lib.check(lib.lib.mr_task_pack_rewrite(os.fsencode(source), os.fsencode(destination)), "mr_task_pack_rewrite")


def quality_solve(mass: np.ndarray, jacobian: np.ndarray, free_velocity: np.ndarray, target: np.ndarray,
                  regularization: np.ndarray, friction: np.ndarray, *, counts: np.ndarray | None = None,
                  warm: np.ndarray | None = None, max_newton: int = 0, tolerance: float = 0.0,
                  regularization_floor: float = 0.0, library: native.Bindings | None = None):
    """Converged contact solves of a batch of dense problems on the GPU
    (mr_quality_solve_batch).  Shapes: mass [P, nv, nv], jacobian
    [P, 3 cap, nv], free_velocity [P, nv], target / regularization / warm
    [P, 3 cap], friction [P, cap], counts [P] (contacts used per problem).
    Returns (impulses [P, 3 cap], velocity [P, nv], results: list of dicts)."""

    lib = library or native.bindings()
    mass = np.ascontiguousarray(mass, np.float64)
    P, nv = mass.shape[0], mass.shape[1]
    jac = np.ascontiguousarray(jacobian, np.float64).reshape(P, -1, nv)
    cap = jac.shape[1] // 3
    vf = np.ascontiguousarray(free_velocity, np.float64).reshape(P, nv)
    tgt = np.ascontiguousarray(target, np.float64).reshape(P, 3 * cap)
    reg = np.ascontiguousarray(regularization, np.float64).reshape(P, 3 * cap)
    mu = np.ascontiguousarray(friction, np.float64).reshape(P, cap)
    dp = lambda a: a.ctypes.data_as(ct.POINTER(ct.c_double))  # noqa: E731
    cnt = None if counts is None else np.ascontiguousarray(counts, np.uint32).reshape(P)
    wm = None if warm is None else np.ascontiguousarray(warm, np.float64).reshape(P, 3 * cap)
    imp = np.zeros((P, 3 * cap), np.float64)
    vel = np.zeros((P, nv), np.float64)
    res = (native.QualityResultC * P)()
    cfg = native.QualitySolverConfigC(max_newton, 0, tolerance, 0.0, regularization_floor, 0.0)
    lib.check(lib.lib.mr_quality_solve_batch(P, nv, cap, None if cnt is None else cnt.ctypes.data_as(ct.POINTER(ct.c_uint32)),
                                             dp(mass), dp(jac), dp(vf), dp(tgt), dp(reg), dp(mu),
                                             None if wm is None else dp(wm), ct.byref(cfg), dp(imp), dp(vel), res),
              "quality_solve")
    results = [{"code": int(r.code), "newton_iterations": int(r.newton_iterations),
                "line_search_iterations": int(r.line_search_iterations), "scaled_optimality": float(r.scaled_optimality),
                "cone_violation": float(r.cone_violation), "complementarity": float(r.complementarity),
                "objective": float(r.objective)} for r in res]
    return imp, vel, results


# MRTaskTransitionC as a numpy record.
_TRANSITION_DTYPE = np.dtype([
    ("reward", "<f4"), ("tracking_score", "<f4"), ("root_height", "<f4"), ("tilt", "<f4"), ("done", "<u4"), ("timeout", "<u4"),
    ("physics_error", "<u4"), ("termination_reason", "<u4"), ("task_reward", "<f4"), ("base_reward", "<f4"),
    ("joint_velocity_reward", "<f4"), ("joint_acceleration_reward", "<f4"), ("control_reward", "<f4"), ("posture_reward", "<f4"),
    ("energy_reward", "<f4"), ("contact_reward", "<f4"), ("task_outcome_channels", "<f4", (8,)), ("policy_revision", "<u8"),
    ("timeout_bootstrap_value", "<f4"), ("episode_tracking_score", "<f4"), ("difficulty_band", "<u4"), ("terrain_level", "<u4"),
    ("impact_sequence_index", "<u4"), ("impact_event_flags", "<u4"),
])


class World:
    """A batch of environments of one synthetic world on the current CUDA device."""

    def __init__(
        self,
        source: str | int = "tree29",
        envs: int = 1,
        *,
        substeps: int = 4,
        velocity_iterations: int = 8,
        final_velocity_iterations: int = 0,
        control_dt: float = 0.02,
        seed: int = 0,
        precision: str = "fp32",
        difficulty_bands: tuple[int, int] | None = None,
        library: native.Bindings | None = None,
    ) -> None:
        self._lib = library or native.bindings()
        if precision not in native.PRECISION_MODES:
            raise ValueError(f"precision must be one of {sorted(native.PRECISION_MODES)}")
        self.source = _source_id(source)
        manifest = native.default_manifest(
            self.source,
            envs,
            physics_substeps=substeps,
            velocity_iterations=velocity_iterations,
            final_velocity_iterations=final_velocity_iterations,
            control_timestep_seconds=control_dt,
            seed=seed,
        )
        if difficulty_bands is not None:  # the sampled band range of a task's episodes
            manifest.profile.override_difficulty_band_range = 1
            manifest.profile.minimum_difficulty_band, manifest.profile.maximum_difficulty_band = difficulty_bands
        handle = self._lib.lib.mr_create_task_rollout(ct.byref(manifest))
        if not handle:
            raise MetalRoboError(f"mr_create_task_rollout: {self._lib.last_error()}")
        self._handle = ct.c_void_p(handle)
        self.envs = envs
        self.seed = seed
        self.substeps = substeps
        layout = self.layout()
        self.nq = int(layout.nq)
        self.nv = int(layout.nv)
        self.action_count = int(layout.action_count)
        self.observation_count = self.nq + self.nv
        model = native.ModelViewC()
        self._lib.check(self._lib.lib.mr_task_rollout_copy_model(self._handle, ct.byref(model)), "copy_model")
        self.pair_count = int(model.world.pair_count)
        self.scene_bodies = int(layout.scene_body_count)
        self.scene = self.scene_bodies > 0
        self.solver = "temporal_cone"
        self.task = None
        self.set_precision(precision)

    def set_precision(self, precision: str) -> None:
        """"fp32" (reference precision), "fp64-inertia" (FP64 articulated
        inertia) or "compensated" (FP64 articulated inertia plus compensated
        FP32 position and impulse sums)."""

        if precision not in native.PRECISION_MODES:
            raise ValueError(f"precision must be one of {sorted(native.PRECISION_MODES)}")
        self._lib.check(self._lib.lib.mr_task_rollout_set_precision(self._handle, native.PRECISION_MODES[precision]),
                        "set_precision")
        self.precision = precision

    def set_solver(self, solver: str, *, max_newton: int = 0, max_line_search: int = 0, tolerance: float = 0.0,
                   line_search_tolerance: float = 0.0, regularization_floor: float = 0.0) -> None:
        """"temporal_cone" (default, fixed sweep budget) or "quality_newton"
        (every substep's contact problem solved to convergence in FP64;
        articulated contact worlds).  Zero settings take the library's
        defaults (100 Newton steps, 50 line-search evaluations per step,
        tolerance 1e-9, line-search tolerance 0.1, regularisation floor
        1e-6)."""

        if solver not in native.SOLVERS:
            raise ValueError(f"solver must be one of {sorted(native.SOLVERS)}")
        cfg = native.QualitySolverConfigC(max_newton, max_line_search, tolerance, line_search_tolerance, regularization_floor, 0.0)
        self._lib.check(self._lib.lib.mr_task_rollout_set_solver(self._handle, native.SOLVERS[solver], ct.byref(cfg)),
                        "set_solver")
        self.solver = solver

    def quality_diagnostics(self) -> dict[str, float]:
        """Certificates of the last advance's quality solves."""

        out = native.QualityDiagnosticsC()
        self._lib.check(self._lib.lib.mr_task_rollout_quality_diagnostics(self._handle, ct.byref(out)), "quality_diagnostics")
        return {
            "newton_iterations": int(out.maximum_newton_iterations),
            "line_search_iterations": int(out.line_search_iterations),
            "scaled_optimality": float(out.maximum_scaled_optimality),
            "cone_violation": float(out.maximum_cone_violation),
            "complementarity": float(out.maximum_complementarity),
        }

    # -- lifecycle -------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_handle", None) and self._handle.value:
            self._lib.lib.mr_task_rollout_destroy(self._handle)
            self._handle = ct.c_void_p(None)

    def __del__(self) -> None:
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self) -> "World":
        return self

    def __exit__(self, *exc: object) -> None:
        self.close()

    # -- queries ---------------------------------------------------------
    def layout(self) -> native.TaskRolloutLayoutC:
        return self._lib.lib.mr_task_rollout_layout(self._handle)

    def launch_shape(self) -> tuple[int, int]:
        """(environments per CTA, resident environments per SM) of the
        control-step kernel in the current precision mode."""

        wpb, res = ct.c_uint32(), ct.c_uint32()
        self._lib.check(self._lib.lib.mr_task_rollout_launch_shape(self._handle, ct.byref(wpb), ct.byref(res)), "launch_shape")
        return int(wpb.value), int(res.value)

    def device_name(self) -> str:
        name = self._lib.lib.mr_task_rollout_device_name(self._handle)
        return name.decode() if name else ""

    def model(self) -> ModelRecords:
        probe = native.ModelViewC()
        self._lib.check(self._lib.lib.mr_task_rollout_copy_model(self._handle, ct.byref(probe)), "copy_model")
        records = _alloc_records(probe.world)
        if probe.hull_vertex_count:
            records.hull_vertices = np.zeros((probe.hull_vertex_count, 4), np.float32)
        view = records.view()
        self._lib.check(self._lib.lib.mr_task_rollout_copy_model(self._handle, ct.byref(view)), "copy_model")
        records.world = view.world
        return records

    def friction_scales(self) -> np.ndarray:
        out = np.zeros((self.envs,), np.float32)
        self._lib.check(
            self._lib.lib.mr_task_rollout_copy_environment_parameters(self._handle, out.ctypes.data_as(ct.POINTER(ct.c_float))),
            "copy_environment_parameters",
        )
        return out

    # -- state -----------------------------------------------------------
    def reset(self, seed: int | None = None) -> None:
        if seed is not None:
            self.seed = seed
        self._lib.check(self._lib.lib.mr_task_rollout_reset(self._handle, self.seed), "mr_task_rollout_reset")

    def state(self) -> tuple[np.ndarray, np.ndarray, Any]:
        """q, v and the persistent manifolds: a ctypes MRManifoldC array
        [env][pair] for articulated worlds, a float32 array [env][slot][57]
        (manifold words + pair key, sorted by key) for scene worlds."""

        q = np.zeros((self.envs, self.nq), np.float32)
        v = np.zeros((self.envs, self.nv), np.float32)
        if self.scene:
            table = np.zeros((self.envs, SCENE_MANIFOLDS, SCENE_SLOT_WORDS), np.float32)
            self._lib.check(
                self._lib.lib.mr_task_rollout_copy_state(
                    self._handle, q.ctypes.data_as(ct.POINTER(ct.c_float)), v.ctypes.data_as(ct.POINTER(ct.c_float)),
                    ct.c_void_p(table.ctypes.data)),
                "copy_state",
            )
            return q, v, table
        manifolds = (native.ManifoldC * max(self.envs * self.pair_count, 1))()
        self._lib.check(
            self._lib.lib.mr_task_rollout_copy_state(
                self._handle,
                q.ctypes.data_as(ct.POINTER(ct.c_float)),
                v.ctypes.data_as(ct.POINTER(ct.c_float)),
                ct.cast(manifolds, ct.c_void_p) if self.pair_count else None,
            ),
            "copy_state",
        )
        return q, v, manifolds

    def set_state(self, q: np.ndarray, v: np.ndarray, manifolds: Any = None, *, as_reset_state: bool = False) -> None:
        q = np.ascontiguousarray(q, np.float32)
        v = np.ascontiguousarray(v, np.float32)
        if q.shape != (self.envs, self.nq) or v.shape != (self.envs, self.nv):
            raise ValueError("state shapes must be (envs, nq) and (envs, nv)")
        self._lib.check(
            self._lib.lib.mr_task_rollout_set_state(
                self._handle,
                q.ctypes.data_as(ct.POINTER(ct.c_float)),
                v.ctypes.data_as(ct.POINTER(ct.c_float)),
                (ct.c_void_p(np.ascontiguousarray(manifolds, np.float32).ctypes.data) if isinstance(manifolds, np.ndarray)
                 else ct.cast(manifolds, ct.c_void_p)) if manifolds is not None else None,
                1 if as_reset_state else 0,
            ),
            "set_state",
        )

    AUDIT_FIELDS = ("kinetic", "potential", "total", "reference_total", "max_total_drift", "px", "py", "pz", "lx", "ly", "lz",
                    "steps")

    def set_audit(self, enabled: bool) -> None:
        """Per-environment FP64 energy and momentum audit on the device."""

        self._lib.check(self._lib.lib.mr_task_rollout_set_audit(self._handle, 1 if enabled else 0), "set_audit")

    def audit(self) -> np.ndarray:
        """[env, 12] audit records (fields in AUDIT_FIELDS order)."""

        out = np.zeros((self.envs, 12), np.float64)
        self._lib.check(self._lib.lib.mr_task_rollout_copy_audit(self._handle, out.ctypes.data_as(ct.POINTER(ct.c_double)), out.size),
                        "copy_audit")
        return out

    def set_island_labels(self, enabled: bool) -> None:
        """Scene worlds: record each control step's island partition."""

        self._lib.check(self._lib.lib.mr_task_rollout_set_island_labels(self._handle, 1 if enabled else 0), "set_island_labels")

    def island_labels(self) -> np.ndarray:
        """[env, bodies] island index of each body on the last control step's
        final substep (255: in no island)."""

        out = np.zeros((self.envs, 64), np.uint8)
        self._lib.check(self._lib.lib.mr_task_rollout_copy_island_labels(
            self._handle, out.ctypes.data_as(ct.POINTER(ct.c_uint8)), out.size), "copy_island_labels")
        return out[:, : self.scene_bodies].copy()

    # -- stepping ----------------------------------------------------------
    def step(
        self,
        actions: Any,
        reset_mask: Any = None,
        observations: Any = None,
        status: Any = None,
        *,
        wait: bool = False,
    ) -> tuple[Any, Any, native.TaskRolloutAdvanceC | None]:
        """Advances ``actions.shape[0]`` control steps on the device.

        ``actions``: CUDA float32 tensor [steps, envs, action_count] (or
        [envs, action_count] for one step).  Returns (observations [steps,
        envs, nq+nv], status codes [steps, envs], counters or None).
        """

        import torch

        if actions.dim() == 2:
            actions = actions.unsqueeze(0)
        if not actions.is_cuda or actions.dtype != torch.float32 or not actions.is_contiguous():
            raise ValueError("actions must be a contiguous float32 CUDA tensor")
        steps = int(actions.shape[0])
        if tuple(actions.shape[1:]) != (self.envs, self.action_count):
            raise ValueError(f"actions must have shape [steps, {self.envs}, {self.action_count}]")
        device = actions.device
        if observations is None:
            observations = torch.empty((steps, self.envs, self.observation_count), device=device, dtype=torch.float32)
        if status is None:
            status = torch.empty((steps, self.envs), device=device, dtype=torch.int32)
        mask_ptr = None
        if reset_mask is not None:
            if reset_mask.dim() == 1:
                reset_mask = reset_mask.unsqueeze(0)
            if tuple(reset_mask.shape) != (steps, self.envs) or reset_mask.dtype not in (torch.int32, torch.uint32):
                raise ValueError("reset_mask must be an int32 tensor [steps, envs]")
            mask_ptr = ct.c_void_p(reset_mask.contiguous().data_ptr())
        stream = torch.cuda.current_stream(device).cuda_stream
        counters = native.TaskRolloutAdvanceC() if wait else None
        self._lib.check(
            self._lib.lib.mr_task_rollout_advance_device(
                self._handle,
                ct.c_void_p(actions.data_ptr()),
                mask_ptr,
                steps,
                ct.c_void_p(observations.data_ptr()),
                ct.c_void_p(status.data_ptr()),
                ct.c_uint64(stream),
                ct.byref(counters) if counters is not None else None,
            ),
            "mr_task_rollout_advance_device",
        )
        return observations, status, counters

    @property
    def environment_chains(self) -> int:
        """Environment chains (control-step launches per control step) of an articulated advance."""
        return int(self._lib.lib.mr_task_rollout_environment_chains(self._handle))

    # -- native policy ---------------------------------------------------
    def set_policy(
        self,
        layers: Sequence[tuple[np.ndarray, np.ndarray | None, str]],
        *,
        revision: int,
        action_clip: float,
        policy_id: str = "policy",
        observation_mean: np.ndarray | None = None,
        observation_inverse_std: np.ndarray | None = None,
        observation_clip: float = 0.0,
        critic_layers: Sequence[tuple[np.ndarray, np.ndarray | None, str]] = (),
        critic_observation_mean: np.ndarray | None = None,
        critic_observation_inverse_std: np.ndarray | None = None,
        action_log_std: np.ndarray | None = None,
        action_bias: np.ndarray | None = None,
        action_scale: np.ndarray | None = None,
    ) -> None:
        """Installs a dense policy (mr_task_rollout_set_policy).  `layers`
        are (weights [out][in], bias [out] or None, activation name); the
        actor maps [q, v] to the action mean."""

        pk, keep = policy_pack_c(layers, revision=revision, action_clip=action_clip, policy_id=policy_id,
                                 observation_mean=observation_mean, observation_inverse_std=observation_inverse_std,
                                 observation_clip=observation_clip, critic_layers=critic_layers,
                                 critic_observation_mean=critic_observation_mean,
                                 critic_observation_inverse_std=critic_observation_inverse_std, action_log_std=action_log_std,
                                 action_bias=action_bias, action_scale=action_scale)
        self._lib.check(self._lib.lib.mr_task_rollout_set_policy(self._handle, ct.byref(pk)), "mr_task_rollout_set_policy")

    def load_policy_pack(self, path: str | os.PathLike[str]) -> None:
        """Reads a PolicyPack file and installs it (mr_task_rollout_load_policy_pack)."""

        self._lib.check(self._lib.lib.mr_task_rollout_load_policy_pack(self._handle, os.fsencode(path)),
                        "mr_task_rollout_load_policy_pack")

    def clear_policy(self) -> None:
        self._lib.check(self._lib.lib.mr_task_rollout_clear_policy(self._handle), "mr_task_rollout_clear_policy")

    @property
    def policy_revision(self) -> int:
        return int(self._lib.lib.mr_task_rollout_policy_revision(self._handle))

    def step_policy(self, steps: int, *, reset_mask: Any = None, wait: bool = True):
        """Advances `steps` control steps driven by the installed policy on
        the device (no action stream).  Returns (observations, status)."""

        import torch

        device = torch.device("cuda", torch.cuda.current_device())
        observations = torch.empty((steps, self.envs, self.observation_count), device=device, dtype=torch.float32)
        status = torch.empty((steps, self.envs), device=device, dtype=torch.int32)
        mask_ptr = None
        if reset_mask is not None:
            reset_mask = reset_mask.contiguous()
            mask_ptr = ct.c_void_p(reset_mask.data_ptr())
        counters = native.TaskRolloutAdvanceC() if wait else None
        self._lib.check(
            self._lib.lib.mr_task_rollout_advance_device(
                self._handle, None, mask_ptr, steps, ct.c_void_p(observations.data_ptr()), ct.c_void_p(status.data_ptr()),
                ct.c_uint64(torch.cuda.current_stream(device).cuda_stream), ct.byref(counters) if counters is not None else None),
            "mr_task_rollout_advance_device")
        self._last_policy_steps = steps
        return observations, status

    def policy_outputs(self) -> dict[str, np.ndarray] | None:
        """Latents [step][env][action], log-probabilities and values
        [step][env], bootstrap values [env] of the last policy-driven advance
        (copies; after the advance has completed)."""

        L = self._lib.lib
        lat = L.mr_task_rollout_policy_latents(self._handle)
        if not lat:
            return None
        import torch

        torch.cuda.synchronize()
        lp = L.mr_task_rollout_policy_log_probabilities(self._handle)
        steps = self._last_policy_steps
        cells = steps * self.envs
        return {
            "latents": np.ctypeslib.as_array(lat, shape=(cells * self.action_count,)).reshape(steps, self.envs, -1).copy(),
            "log_probabilities": np.ctypeslib.as_array(lp, shape=(cells,)).reshape(steps, self.envs).copy(),
            "values": np.ctypeslib.as_array(L.mr_task_rollout_policy_values(self._handle), shape=(cells,)).reshape(steps, self.envs).copy(),
            "bootstrap_values": np.ctypeslib.as_array(L.mr_task_rollout_bootstrap_policy_values(self._handle), shape=(self.envs,)).copy(),
        }

    # -- task layer ----------------------------------------------------------
    def set_task(self, program) -> None:
        """Installs a task program (``numi_lab_b200.task.TaskProgram``,
        mr_task_rollout_set_task): observations become its actor frames,
        actions its normalised policy actions; every environment starts a
        new episode at the next step."""

        from .task import task_program_c

        record, keep = task_program_c(program)
        self._lib.check(self._lib.lib.mr_task_rollout_set_task(self._handle, ct.byref(record)), "mr_task_rollout_set_task")
        del keep
        self.observation_count = int(self.layout().actor_observation_count)
        self.task = program

    def clear_task(self) -> None:
        self._lib.check(self._lib.lib.mr_task_rollout_clear_task(self._handle), "mr_task_rollout_clear_task")
        self.observation_count = self.nq + self.nv
        self.task = None

    TRANSITION_FIELDS = ("reward", "tracking_score", "root_height", "tilt", "done", "timeout", "physics_error",
                         "termination_reason", "task_reward", "base_reward", "joint_velocity_reward", "joint_acceleration_reward",
                         "control_reward", "posture_reward", "energy_reward", "contact_reward", "episode_tracking_score",
                         "policy_revision", "difficulty_band")

    def transitions(self, steps: int) -> dict[str, np.ndarray]:
        """The last advance's transitions ([step][env] per field; the advance
        must have covered `steps` control steps), copied once its work has
        finished."""

        raw = (native.TaskTransitionC * (steps * self.envs))()
        self._lib.check(self._lib.lib.mr_task_rollout_copy_transitions(self._handle, raw, len(raw)), "mr_task_rollout_copy_transitions")
        arr = np.frombuffer(bytes(raw), dtype=_TRANSITION_DTYPE).reshape(steps, self.envs)
        return {name: arr[name].copy() for name in self.TRANSITION_FIELDS}

    def write_policy_rollout_pack(self, path: str | os.PathLike[str], batch_id: str, observations) -> None:
        """Publishes the last policy-driven advance as a PolicyRolloutPack
        (mr_task_rollout_write_policy_rollout_pack): `observations` are the
        actor frames it returned; latents, log-probabilities, values,
        bootstrap values and transitions are the rollout's own."""

        out = self.policy_outputs()
        if out is None:
            raise MetalRoboError("no policy-driven advance to publish")
        steps = out["latents"].shape[0]
        raw = (native.TaskTransitionC * (steps * self.envs))()
        self._lib.check(self._lib.lib.mr_task_rollout_copy_transitions(self._handle, raw, len(raw)), "mr_task_rollout_copy_transitions")
        frames = observations.cpu().numpy() if hasattr(observations, "cpu") else np.asarray(observations)
        c, keep = policy_rollout_pack_c(id=batch_id, task_fingerprint=0, policy_fingerprint=0, policy_revision=0,
                                        environment_count=self.envs, control_step_count=steps, actor_observations=frames,
                                        latents=out["latents"], log_probabilities=out["log_probabilities"], values=out["values"],
                                        bootstrap_values=out["bootstrap_values"], transitions=raw)
        self._lib.check(self._lib.lib.mr_task_rollout_write_policy_rollout_pack(self._handle, c.batch, batch_id.encode(), os.fsencode(path)),
                        "mr_task_rollout_write_policy_rollout_pack")
        del keep

    def set_state_readback(self, enabled: bool) -> None:
        self._lib.check(self._lib.lib.mr_task_rollout_set_state_readback(self._handle, 1 if enabled else 0), "set_state_readback")

    def advance_host(
        self,
        actions: np.ndarray | None,
        reset_masks: np.ndarray | None = None,
        *,
        raise_on_failure: bool = True,
        copy: bool = True,
        steps: int | None = None,
        evaluate_final_policy: bool = False,
    ) -> dict[str, Any]:
        """Reference-shaped synchronous advance with host buffers.

        With ``copy=False`` the returned arrays are views of the rollout's
        own result memory, valid until the next advance, reset or close --
        the C ABI's rule for the pointers it returns (c_api.h:680-681)."""

        if actions is None:
            # Policy-driven: no action stream.
            if steps is None:
                raise ValueError("steps is required without actions")
            actions = np.zeros((0,), np.float32)
            self._last_policy_steps = int(steps)
        else:
            actions = np.ascontiguousarray(actions, np.float32)
            steps = actions.shape[0] if actions.ndim == 3 else 1
        counters = native.TaskRolloutAdvanceC()
        masks_ptr = None
        mask_count = 0
        if reset_masks is not None:
            reset_masks = np.ascontiguousarray(reset_masks, np.uint32)
            masks_ptr = reset_masks.ctypes.data_as(ct.POINTER(ct.c_uint32))
            mask_count = reset_masks.size
        rc = self._lib.lib.mr_task_rollout_advance(
            self._handle,
            actions.ctypes.data_as(ct.POINTER(ct.c_float)),
            actions.size,
            masks_ptr,
            mask_count,
            steps,
            self.policy_revision if evaluate_final_policy else 0,
            1 if evaluate_final_policy else 0,
            ct.byref(counters),
        )
        if rc != 0 and (raise_on_failure or counters.control_step_count == 0):
            raise MetalRoboError(f"mr_task_rollout_advance: {self._lib.last_error()}")
        cells = steps * self.envs
        out: dict[str, Any] = {"counters": counters, "rc": rc}

        def view(ptr, count, shape):
            if not ptr:
                return None
            a = np.ctypeslib.as_array(ptr, shape=(count,)).reshape(shape)
            return a.copy() if copy else a

        out["status"] = view(self._lib.lib.mr_task_rollout_status_codes(self._handle), cells, (steps, self.envs))
        out["contacts"] = view(self._lib.lib.mr_task_rollout_active_contacts(self._handle), cells, (steps, self.envs))
        obs = self._lib.lib.mr_task_rollout_actor_observations(self._handle)
        if obs:
            out["observations"] = view(obs, cells * self.observation_count, (steps, self.envs, self.observation_count))
            out["final_q"] = view(self._lib.lib.mr_task_rollout_final_q(self._handle), self.envs * self.nq, (self.envs, self.nq))
        return out


class Batch:
    """Several worlds advanced together: one persistent launch per horizon
    over every environment of every world (mr_create_batch).  The worlds
    keep their state; close the batch before them."""

    def __init__(self, worlds: Sequence["World"], *, library: native.Bindings | None = None) -> None:
        self._lib = library or native.bindings()
        self.worlds = list(worlds)
        handles = (ct.c_void_p * len(self.worlds))(*[w._handle.value for w in self.worlds])
        handle = self._lib.lib.mr_create_batch(handles, len(self.worlds))
        if not handle:
            raise MetalRoboError(f"mr_create_batch: {self._lib.last_error()}")
        self._handle = ct.c_void_p(handle)

    def close(self) -> None:
        if getattr(self, "_handle", None) and self._handle.value:
            self._lib.lib.mr_batch_destroy(self._handle)
            self._handle = ct.c_void_p(None)

    def __del__(self) -> None:
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self) -> "Batch":
        return self

    def __exit__(self, *exc: object) -> None:
        self.close()

    @staticmethod
    def _pointers(tensors) -> Any:
        arr = (ct.c_void_p * len(tensors))(*[t.data_ptr() if t is not None else None for t in tensors])
        return ct.cast(arr, ct.POINTER(ct.c_void_p)), arr

    def step(self, actions: Sequence[Any], reset_masks: Sequence[Any] | None = None, status: Sequence[Any] | None = None) -> None:
        """Advances every world by actions[w].shape[0] control steps on torch's
        current stream (actions[w]: CUDA float32 [steps, envs, action_count];
        a world without actions takes an empty [steps, envs, 0] tensor)."""

        import torch

        steps = int(actions[0].shape[0])
        for w, a in zip(self.worlds, actions):
            if a.shape[:2] != (steps, w.envs) or a.dtype != torch.float32 or not a.is_cuda or not a.is_contiguous():
                raise ValueError("actions[w] must be contiguous CUDA float32 [steps, envs, action_count]")
        acts, _keep_a = self._pointers([a if a.shape[-1] > 0 else None for a in actions])
        masks, _keep_m = self._pointers(reset_masks) if reset_masks is not None else (None, None)
        stats, _keep_s = self._pointers(status) if status is not None else (None, None)
        stream = torch.cuda.current_stream().cuda_stream
        self._lib.check(self._lib.lib.mr_batch_advance(self._handle, steps, acts, masks, stats, stream), "mr_batch_advance")

    def tune(self, actions: Sequence[Any]) -> None:
        steps = int(actions[0].shape[0])
        acts, _keep = self._pointers([a if a.shape[-1] > 0 else None for a in actions])
        self._lib.check(self._lib.lib.mr_batch_tune(self._handle, steps, acts), "mr_batch_tune")

    def launch_shape(self) -> dict:
        out = native.BatchLaunchShapeC()
        self._lib.check(self._lib.lib.mr_batch_launch_shape(self._handle, ct.byref(out)), "mr_batch_launch_shape")
        return {name: getattr(out, name) for name, _ in out._fields_}

    def world_costs(self) -> np.ndarray:
        out = np.zeros(len(self.worlds), np.float32)
        self._lib.check(self._lib.lib.mr_batch_world_costs(self._handle, out.ctypes.data_as(ct.POINTER(ct.c_float)), out.size),
                        "mr_batch_world_costs")
        return out

