"""ORACLE — test infrastructure only.

ctypes loaders for
  * ``oracle/liboracle.so``: this project's plain-C FP64 restatement of
    numi-lab's microstep (oracle/oracle.c), and
  * ``oracle/_ref/libnumiref.so``: the reference's own FP64 CPU core compiled
    from its sources with oracle/ref_harness.cpp (built by oracle/Makefile
    where the reference sources exist; the built file travels with the repo
    snapshot).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this package, and only as the checker.  The product library never loads it.
"""

from __future__ import annotations

import ctypes as ct
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent
ORACLE_LIB = HERE / "liboracle.so"
REF_LIB = HERE / "_ref" / "libnumiref.so"
REFERENCE_SOURCES = Path(os.environ.get("NUMI_REFERENCE_ROOT", "/root/reference"))

MAX_CONTACTS = 32
MANIFOLD_POINTS = 4
CONTACT_ROW = 24  # doubles per contact row (oracle_articulated_contacts, ref_articulated_contacts)


class OraclePoint(ct.Structure):
    _fields_ = [
        ("anchor_a", ct.c_double * 3),
        ("anchor_b", ct.c_double * 3),
        ("feature_a", ct.c_uint32),
        ("feature_b", ct.c_uint32),
        ("life", ct.c_uint32),
        ("reserved", ct.c_uint32),
        ("impulses", ct.c_double * 3),
    ]


class OracleManifold(ct.Structure):
    _fields_ = [
        ("normal_local", ct.c_double * 3),
        ("age", ct.c_double),
        ("tangent_local", ct.c_double * 3),
        ("count", ct.c_uint32),
        ("reserved", ct.c_uint32),
        ("points", OraclePoint * MANIFOLD_POINTS),
    ]


class OracleContact(ct.Structure):
    _fields_ = [
        ("pair", ct.c_uint32),
        ("point", ct.c_uint32),
        ("feature_a", ct.c_uint32),
        ("feature_b", ct.c_uint32),
        ("body", ct.c_uint32),
        ("new_impact", ct.c_uint32),
        ("separation", ct.c_double),
        ("normal", ct.c_double * 3),
        ("impulses", ct.c_double * 3),
    ]


class OracleTrace(ct.Structure):
    _fields_ = [
        ("status", ct.c_uint32),
        ("failing_index", ct.c_uint32),
        ("failing_substep", ct.c_uint32),
        ("contact_count", ct.c_uint32),
        ("island_count", ct.c_uint32),
        ("manifold_count", ct.c_uint32),
        ("max_contacts", ct.c_uint32),
        ("band_decisions", ct.c_uint32),
        ("max_cone_violation", ct.c_double),
        ("max_normal_residual", ct.c_double),
        ("min_decision_margin", ct.c_double),
        ("contacts", OracleContact * MAX_CONTACTS),
        ("quality_newton", ct.c_uint32),
        ("quality_line_search", ct.c_uint32),
    ]


def set_rounding_noise(seed: int) -> None:
    """Test-only Monte Carlo rounding mode of the C restatement on this
    thread: seed != 0 perturbs every FP32-rounded intermediate by a random
    relative 2^-24 (one rounding to nearest); 0 is exact FP64."""

    lib = ct.CDLL(str(ORACLE_LIB))
    lib.oracle_set_rounding_noise.argtypes = [ct.c_uint64]
    lib.oracle_set_rounding_noise(int(seed) & 0xFFFFFFFFFFFFFFFF)


def build(reference: bool = True) -> None:
    """Compiles the checker libraries (the C restatement always; the
    reference core when its sources are present)."""

    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    if reference and (REFERENCE_SOURCES / "src" / "core").is_dir():
        subprocess.run(["make", "-s", "-j8", "-C", str(HERE), "ref", f"REF={REFERENCE_SOURCES}"], check=True)


_DP = ct.POINTER(ct.c_double)


def _dp(a: np.ndarray):
    return a.ctypes.data_as(_DP)


class QualityConfig(ct.Structure):
    """OracleQualityConfig (the library's defaults)."""

    _fields_ = [
        ("max_newton", ct.c_int32),
        ("max_line_search", ct.c_int32),
        ("tolerance", ct.c_double),
        ("line_search_tolerance", ct.c_double),
        ("regularization_floor", ct.c_double),
    ]


def quality_config(max_newton: int = 100, max_line_search: int = 50, tolerance: float = 1e-9, line_search_tolerance: float = 0.1,
                   regularization_floor: float = 1e-6) -> QualityConfig:
    return QualityConfig(max_newton, max_line_search, tolerance, line_search_tolerance, regularization_floor)


class QualityOutcome(ct.Structure):
    _fields_ = [
        ("status", ct.c_uint32),
        ("newton", ct.c_uint32),
        ("line_search", ct.c_uint32),
        ("reserved", ct.c_uint32),
        ("residual", ct.c_double),
        ("cone", ct.c_double),
        ("complementarity", ct.c_double),
        ("objective", ct.c_double),
    ]


def _oracle_lib():
    if not ORACLE_LIB.is_file():
        build(reference=False)
    lib = ct.CDLL(str(ORACLE_LIB))
    lib.oracle_quality_dense.restype = ct.c_uint32
    lib.oracle_quality_dense.argtypes = [ct.c_uint32, ct.c_uint32] + [_DP] * 7 + [ct.POINTER(QualityConfig), _DP, _DP,
                                                                                   ct.POINTER(QualityOutcome)]
    lib.oracle_world_set_quality.argtypes = [ct.c_void_p, ct.POINTER(QualityConfig)]
    return lib


def quality_dense(mass, jacobian, free_velocity, target, reg, mu, warm=None, cfg: QualityConfig | None = None):
    """The oracle's converged contact solve of one dense problem (the inputs
    of mr_quality_solve_batch for one problem, nc = len(mu)).  Returns
    (status, impulses [3 nc], velocity [nv], outcome)."""

    lib = _oracle_lib()
    mass = np.ascontiguousarray(mass, np.float64)
    nv, nc = mass.shape[0], len(mu)
    lam = np.zeros(3 * nc)
    vel = np.zeros(nv)
    out = QualityOutcome()
    st = lib.oracle_quality_dense(nv, nc, _dp(mass), _dp(np.ascontiguousarray(jacobian, np.float64)),
                                  _dp(np.ascontiguousarray(free_velocity, np.float64)), _dp(np.ascontiguousarray(target, np.float64)),
                                  _dp(np.ascontiguousarray(reg, np.float64)), _dp(np.ascontiguousarray(mu, np.float64)),
                                  None if warm is None else _dp(np.ascontiguousarray(warm, np.float64)),
                                  ct.byref(cfg or quality_config()), _dp(lam), _dp(vel), ct.byref(out))
    return int(st), lam, vel, out


def reference_quality_solve(inverse_mass, free_velocity, jacobian, mu, target, reg):
    """The reference's solveQualityContactProblem on one dense problem.
    Returns (status, impulses, velocity, certificates dict)."""

    if not REF_LIB.is_file():
        raise FileNotFoundError(f"{REF_LIB} is missing; build it with `make -C oracle ref` where the reference sources exist")
    lib = ct.CDLL(str(REF_LIB))
    lib.ref_quality_solve.restype = ct.c_int
    lib.ref_quality_solve.argtypes = [ct.c_uint32, _DP, _DP, ct.c_uint32] + [_DP] * 7 + [ct.POINTER(ct.c_uint32)]
    inverse_mass = np.ascontiguousarray(inverse_mass, np.float64)
    nv, n = inverse_mass.shape[0], len(mu)
    imp = np.zeros(3 * n)
    vel = np.zeros(nv)
    cert = np.zeros(8)
    iters = ct.c_uint32(0)
    st = lib.ref_quality_solve(nv, _dp(inverse_mass), _dp(np.ascontiguousarray(free_velocity, np.float64)), n,
                               _dp(np.ascontiguousarray(jacobian, np.float64)), _dp(np.ascontiguousarray(mu, np.float64)),
                               _dp(np.ascontiguousarray(target, np.float64)), _dp(np.ascontiguousarray(reg, np.float64)),
                               _dp(imp), _dp(vel), _dp(cert), ct.byref(iters))
    names = ("kkt", "natural_residual", "primal_cone", "dual_cone", "complementarity", "gap", "objective", "normal")
    return int(st), imp, vel, dict(zip(names, cert.tolist()), iterations=int(iters.value))


def _ref_lib():
    if not REF_LIB.is_file():
        raise FileNotFoundError(f"{REF_LIB} is missing; build it with `make -C oracle ref` where the reference sources exist")
    return ct.CDLL(str(REF_LIB))


def reference_write_policy_pack(pack, path) -> None:
    """The reference's writePolicyPack on a pack given as an MRPolicyPackC
    (numi_lab_b200.native.PolicyPackC)."""

    lib = _ref_lib()
    lib.ref_write_policy_pack.restype = ct.c_int
    lib.ref_write_policy_pack.argtypes = [ct.c_void_p, ct.c_char_p, ct.c_char_p, ct.c_size_t]
    err = ct.create_string_buffer(512)
    st = lib.ref_write_policy_pack(ct.addressof(pack), os.fsencode(path), err, len(err))
    if st != 0:
        raise ValueError(f"reference writePolicyPack failed ({st}): {err.value.decode()}")


def reference_write_policy_rollout_pack(pack, path) -> None:
    """The reference's writePolicyRolloutPack on a pack given as an
    MRPolicyRolloutPackC (numi_lab_b200.native.PolicyRolloutPackC)."""

    lib = _ref_lib()
    lib.ref_write_policy_rollout_pack.restype = ct.c_int
    lib.ref_write_policy_rollout_pack.argtypes = [ct.c_void_p, ct.c_char_p, ct.c_char_p, ct.c_size_t]
    err = ct.create_string_buffer(512)
    st = lib.ref_write_policy_rollout_pack(ct.addressof(pack), os.fsencode(path), err, len(err))
    if st != 0:
        raise ValueError(f"reference writePolicyRolloutPack failed ({st}): {err.value.decode()}")


def reference_inspect_policy_rollout_pack(path, parameter_count: int = 0):
    """The reference's readPolicyRolloutPack in the layout of
    mr_policy_rollout_pack_inspect: (fields, actor observations, latents,
    log-probabilities, values and bootstrap values concatenated)."""

    from numi_lab_b200 import native

    lib = _ref_lib()
    lib.ref_policy_rollout_pack_inspect.restype = ct.c_int
    lib.ref_policy_rollout_pack_inspect.argtypes = [ct.c_char_p, ct.c_void_p, ct.POINTER(ct.c_float), ct.c_size_t, ct.c_char_p,
                                                    ct.c_size_t]
    info = native.PolicyRolloutPackInfoC()
    err = ct.create_string_buffer(512)
    params = np.zeros(parameter_count, np.float32)
    st = lib.ref_policy_rollout_pack_inspect(os.fsencode(path), ct.addressof(info),
                                             params.ctypes.data_as(ct.POINTER(ct.c_float)) if parameter_count else None,
                                             params.size, err, len(err))
    if st != 0:
        raise ValueError(f"reference readPolicyRolloutPack failed ({st}): {err.value.decode()}")
    fields = {name: getattr(info, name) for name, _ in native.PolicyRolloutPackInfoC._fields_}
    fields["id"] = info.id.decode()
    return fields, params


def reference_write_task_pack(variant: int, path) -> None:
    """A TaskPack filled field by field in the harness (0: every table and
    program used; 1: the smallest valid pack), written by the reference's
    writeTaskPack."""

    lib = _ref_lib()
    lib.ref_write_task_pack.restype = ct.c_int
    lib.ref_write_task_pack.argtypes = [ct.c_int, ct.c_char_p, ct.c_char_p, ct.c_size_t]
    err = ct.create_string_buffer(512)
    st = lib.ref_write_task_pack(variant, os.fsencode(path), err, len(err))
    if st != 0:
        raise ValueError(f"reference writeTaskPack failed ({st}): {err.value.decode()}")


def reference_inspect_task_pack(path) -> dict:
    """The reference's readTaskPack in the layout of mr_task_pack_inspect."""

    from numi_lab_b200 import native

    lib = _ref_lib()
    lib.ref_task_pack_inspect.restype = ct.c_int
    lib.ref_task_pack_inspect.argtypes = [ct.c_char_p, ct.c_void_p, ct.c_char_p, ct.c_size_t]
    info = native.TaskPackInfoC()
    err = ct.create_string_buffer(512)
    st = lib.ref_task_pack_inspect(os.fsencode(path), ct.addressof(info), err, len(err))
    if st != 0:
        raise ValueError(f"reference readTaskPack failed ({st}): {err.value.decode()}")
    fields = {name: getattr(info, name) for name, _ in native.TaskPackInfoC._fields_}
    fields["id"] = info.id.decode()
    return fields


def reference_rewrite_task_pack(source, destination) -> None:
    """The reference's readTaskPack then writeTaskPack."""

    lib = _ref_lib()
    lib.ref_task_pack_rewrite.restype = ct.c_int
    lib.ref_task_pack_rewrite.argtypes = [ct.c_char_p, ct.c_char_p, ct.c_char_p, ct.c_size_t]
    err = ct.create_string_buffer(512)
    st = lib.ref_task_pack_rewrite(os.fsencode(source), os.fsencode(destination), err, len(err))
    if st != 0:
        raise ValueError(f"reference TaskPack rewrite failed ({st}): {err.value.decode()}")


def reference_capacity_profile_bytes() -> int:
    lib = _ref_lib()
    lib.ref_capacity_profile_bytes.restype = ct.c_size_t
    return int(lib.ref_capacity_profile_bytes())


def reference_inspect_policy_pack(path):
    """The reference's readPolicyPack: (fields, FP32 tables in file order)
    in the layout of mr_policy_pack_inspect."""

    from numi_lab_b200 import native

    lib = _ref_lib()
    lib.ref_policy_pack_inspect.restype = ct.c_int
    lib.ref_policy_pack_inspect.argtypes = [ct.c_char_p, ct.c_void_p, ct.POINTER(ct.c_float), ct.c_size_t, ct.c_char_p,
                                            ct.c_size_t]
    info = native.PolicyPackInfoC()
    err = ct.create_string_buffer(512)
    st = lib.ref_policy_pack_inspect(os.fsencode(path), ct.addressof(info), None, 0, err, len(err))
    if st != 0:
        raise ValueError(f"reference readPolicyPack failed ({st}): {err.value.decode()}")
    params = np.zeros(int(info.parameter_count), np.float32)
    lib.ref_policy_pack_inspect(os.fsencode(path), ct.addressof(info), params.ctypes.data_as(ct.POINTER(ct.c_float)), params.size,
                                err, len(err))
    fields = {name: getattr(info, name) for name, _ in native.PolicyPackInfoC._fields_}
    fields["id"] = info.id.decode()
    return fields, params


class Oracle:
    """The C restatement, bound to one compiled world."""

    def __init__(self, records, h: float, substeps: int, velocity_iterations: int, final_velocity_iterations: int) -> None:
        if not ORACLE_LIB.is_file():
            build(reference=False)
        lib = ct.CDLL(str(ORACLE_LIB))
        self.lib = lib
        lib.oracle_world_create.restype = ct.c_void_p
        lib.oracle_world_create.argtypes = [ct.c_void_p] * 7 + [ct.c_double, ct.c_uint32, ct.c_uint32, ct.c_uint32]
        lib.oracle_world_destroy.argtypes = [ct.c_void_p]
        lib.oracle_control_step.restype = ct.c_uint32
        lib.oracle_control_step.argtypes = [ct.c_void_p, _DP, _DP, ct.c_void_p, _DP, ct.c_double, ct.c_int, _DP, _DP, ct.c_void_p]
        lib.oracle_aba.restype = ct.c_uint32
        lib.oracle_aba.argtypes = [ct.c_void_p, _DP, _DP, _DP, _DP]
        lib.oracle_mass_matrix.restype = ct.c_uint32
        lib.oracle_mass_matrix.argtypes = [ct.c_void_p, _DP, _DP]
        lib.oracle_body_states.restype = ct.c_uint32
        lib.oracle_body_states.argtypes = [ct.c_void_p, _DP, _DP, _DP]
        lib.oracle_point_jacobian.restype = ct.c_uint32
        lib.oracle_point_jacobian.argtypes = [ct.c_void_p, _DP, ct.c_uint32, _DP, _DP, _DP]
        lib.oracle_drive_efforts.argtypes = [ct.c_void_p, _DP, _DP, _DP, _DP]
        lib.oracle_project_cone.argtypes = [_DP, ct.c_double, ct.c_double, _DP]
        lib.oracle_invert3x3.restype = ct.c_int
        lib.oracle_invert3x3.argtypes = [_DP, _DP]
        lib.oracle_manifold_from_device.argtypes = [ct.c_void_p, ct.c_void_p, ct.c_uint32]
        lib.oracle_manifold_to_device.argtypes = [ct.c_void_p, ct.c_void_p, ct.c_uint32]
        lib.oracle_temporal_cone_dense.argtypes = [ct.c_uint32, _DP, _DP, _DP, ct.c_uint32, _DP]
        self.records = records
        w = records.world
        self.nq, self.nv, self.na, self.np = int(w.nq), int(w.nv), int(w.action_count), int(w.pair_count)
        self.h = h
        self.handle = lib.oracle_world_create(
            ct.byref(records.world),
            ct.cast(records.joints, ct.c_void_p),
            ct.cast(records.bodies, ct.c_void_p),
            ct.cast(records.dofs, ct.c_void_p),
            ct.cast(records.shapes, ct.c_void_p),
            ct.cast(records.materials, ct.c_void_p),
            ct.cast(records.pairs, ct.c_void_p),
            h,
            substeps,
            velocity_iterations,
            final_velocity_iterations,
        )
        if not self.handle:
            raise RuntimeError("oracle_world_create failed")
        lib.oracle_world_set_quality.argtypes = [ct.c_void_p, ct.POINTER(QualityConfig)]

    def set_quality(self, cfg: QualityConfig | None) -> None:
        """Converged contact solves (cfg) or the temporalCone sweeps (None)."""

        self._quality = cfg
        self.lib.oracle_world_set_quality(self.handle, ct.byref(cfg) if cfg is not None else None)

    def __del__(self) -> None:
        try:
            if self.handle:
                self.lib.oracle_world_destroy(self.handle)
        except Exception:
            pass

    def new_manifolds(self, count: int = 1):
        return (OracleManifold * max(count * self.np, 1))()

    def manifolds_from_device(self, device_manifolds, count: int):
        out = (OracleManifold * max(count, 1))()
        self.lib.oracle_manifold_from_device(ct.cast(device_manifolds, ct.c_void_p), ct.cast(out, ct.c_void_p), count)
        return out

    def env_manifolds(self, device_manifolds, env: int):
        """Oracle copy of environment `env`'s slots of a device manifold array."""

        out = (OracleManifold * max(self.np, 1))()
        if self.np:
            size = ct.sizeof(device_manifolds._type_)
            src = ct.c_void_p(ct.addressof(device_manifolds) + env * self.np * size)
            self.lib.oracle_manifold_from_device(src, ct.cast(out, ct.c_void_p), self.np)
        return out

    def control_step(self, q: np.ndarray, v: np.ndarray, manifolds, actions: np.ndarray, friction: float,
                     reset: bool = False, reset_q: np.ndarray | None = None, reset_v: np.ndarray | None = None):
        """One control step of one env; q, v (float64) and manifolds in place."""

        assert q.dtype == np.float64 and v.dtype == np.float64
        trace = OracleTrace()
        act = np.ascontiguousarray(actions, np.float64)
        rq = np.ascontiguousarray(reset_q if reset_q is not None else q, np.float64)
        rv = np.ascontiguousarray(reset_v if reset_v is not None else v, np.float64)
        status = self.lib.oracle_control_step(
            self.handle, _dp(q), _dp(v), ct.cast(manifolds, ct.c_void_p) if manifolds is not None else None,
            _dp(act), float(friction), 1 if reset else 0, _dp(rq), _dp(rv), ct.byref(trace))
        return int(status), trace

    def aba(self, q, v, tau) -> tuple[int, np.ndarray]:
        out = np.zeros(self.nv)
        st = self.lib.oracle_aba(self.handle, _dp(np.ascontiguousarray(q, np.float64)), _dp(np.ascontiguousarray(v, np.float64)),
                                 _dp(np.ascontiguousarray(tau, np.float64)), _dp(out))
        return int(st), out

    def body_states(self, q: np.ndarray, v: np.ndarray) -> np.ndarray:
        """[nb][13]: world COM position, orientation xyzw, linear and angular velocity."""

        out = np.zeros((int(self.records.world.body_count), 13))
        st = self.lib.oracle_body_states(self.handle, _dp(np.ascontiguousarray(q, np.float64)), _dp(np.ascontiguousarray(v, np.float64)),
                                         _dp(out))
        if st != 0:
            raise ValueError(f"oracle_body_states failed ({st})")
        return out

    def mass_matrix(self, q) -> np.ndarray:
        out = np.zeros((self.nv, self.nv))
        self.lib.oracle_mass_matrix(self.handle, _dp(np.ascontiguousarray(q, np.float64)), _dp(out))
        return out

    def point_jacobian(self, q, body: int, local) -> tuple[np.ndarray, np.ndarray]:
        wp = np.zeros(3)
        J = np.zeros((3, self.nv))
        self.lib.oracle_point_jacobian(self.handle, _dp(np.ascontiguousarray(q, np.float64)), body,
                                       _dp(np.ascontiguousarray(local, np.float64)), _dp(wp), _dp(J))
        return wp, J

    def drive_efforts(self, q, v, actions) -> np.ndarray:
        out = np.zeros(self.nv)
        self.lib.oracle_drive_efforts(self.handle, _dp(np.ascontiguousarray(q, np.float64)), _dp(np.ascontiguousarray(v, np.float64)),
                                      _dp(np.ascontiguousarray(actions, np.float64)), _dp(out))
        return out

    def project_cone(self, impulse, mu_u: float, mu_v: float) -> np.ndarray:
        out = np.zeros(3)
        self.lib.oracle_project_cone(_dp(np.ascontiguousarray(impulse, np.float64)), mu_u, mu_v, _dp(out))
        return out

    def invert3x3(self, m) -> tuple[bool, np.ndarray]:
        out = np.zeros(9)
        ok = self.lib.oracle_invert3x3(_dp(np.ascontiguousarray(m, np.float64).reshape(9)), _dp(out))
        return bool(ok), out.reshape(3, 3)

    def articulated_contacts(self, q, vf, manifolds, friction: float, speculative: bool = False):
        """Collision + ConstraintIR rows at (q, vf); manifolds updated in place.
        Returns (status, raw [n, 16], rows [m, CONTACT_ROW])."""

        L = self.lib
        if not getattr(self, "_contacts_bound", False):
            L.oracle_articulated_contacts.restype = ct.c_uint32
            L.oracle_articulated_contacts.argtypes = [ct.c_void_p, _DP, _DP, ct.c_void_p, ct.c_double, ct.c_int, _DP, ct.c_uint32,
                                                      ct.POINTER(ct.c_uint32), _DP, ct.c_uint32, ct.POINTER(ct.c_uint32)]
            self._contacts_bound = True
        raw = np.zeros((256, 16))
        rows = np.zeros((MAX_CONTACTS * 4, CONTACT_ROW))
        nr, nc = ct.c_uint32(0), ct.c_uint32(0)
        st = L.oracle_articulated_contacts(self.handle, _dp(np.ascontiguousarray(q, np.float64)), _dp(np.ascontiguousarray(vf, np.float64)),
                                           ct.cast(manifolds, ct.c_void_p), float(friction), 1 if speculative else 0, _dp(raw), 256,
                                           ct.byref(nr), _dp(rows), rows.shape[0], ct.byref(nc))
        return int(st), raw[: nr.value].copy(), rows[: nc.value].copy()

    def temporal_cone_dense(self, W, u0, mu, iterations: int, lam0=None) -> np.ndarray:
        n = len(mu)
        lam = np.zeros(3 * n) if lam0 is None else np.array(lam0, np.float64)
        self.lib.oracle_temporal_cone_dense(n, _dp(np.ascontiguousarray(W, np.float64)), _dp(np.ascontiguousarray(u0, np.float64)),
                                            _dp(np.ascontiguousarray(mu, np.float64)), iterations, _dp(lam))
        return lam


class Reference:
    """The reference's own FP64 CPU core (compiled from its sources)."""

    def __init__(self, records, h: float, friction: float = 1.0) -> None:
        if not REF_LIB.is_file():
            raise FileNotFoundError(f"{REF_LIB} is missing; build it with `make -C oracle ref` where the reference sources exist")
        lib = ct.CDLL(str(REF_LIB))
        self.lib = lib
        lib.ref_model_create.restype = ct.c_void_p
        lib.ref_model_create.argtypes = [ct.c_void_p] * 6 + [ct.c_double, ct.c_double, ct.c_char_p, ct.c_size_t]
        lib.ref_model_destroy.argtypes = [ct.c_void_p]
        lib.ref_forward_dynamics.restype = ct.c_int
        lib.ref_forward_dynamics.argtypes = [ct.c_void_p, _DP, _DP, _DP, _DP]
        lib.ref_mass_matrix.restype = ct.c_int
        lib.ref_mass_matrix.argtypes = [ct.c_void_p, _DP, _DP]
        lib.ref_point_jacobian.restype = ct.c_int
        lib.ref_point_jacobian.argtypes = [ct.c_void_p, _DP, ct.c_uint32, _DP, _DP, _DP]
        lib.ref_integrate.restype = ct.c_int
        lib.ref_integrate.argtypes = [ct.c_void_p, _DP, _DP, _DP]
        lib.ref_conic_solve.restype = ct.c_int
        lib.ref_conic_solve.argtypes = [ct.c_uint32, _DP, _DP, ct.c_uint32, _DP, _DP, _DP, _DP, _DP, _DP, _DP]
        lib.ref_run.restype = ct.c_double
        lib.ref_run.argtypes = [ct.c_void_p, ct.c_uint32, _DP, _DP, ct.POINTER(ct.c_float), ct.c_uint32, ct.c_uint32,
                                ct.c_uint32, ct.c_int, ct.POINTER(ct.c_uint64)]
        w = records.world
        self.nq, self.nv = int(w.nq), int(w.nv)
        err = ct.create_string_buffer(512)
        self.handle = lib.ref_model_create(
            ct.byref(records.world), ct.cast(records.joints, ct.c_void_p), ct.cast(records.bodies, ct.c_void_p),
            ct.cast(records.dofs, ct.c_void_p), ct.cast(records.shapes, ct.c_void_p), ct.cast(records.materials, ct.c_void_p),
            h, friction, err, len(err))
        if not self.handle:
            raise RuntimeError(err.value.decode())

    def __del__(self) -> None:
        try:
            if self.handle:
                self.lib.ref_model_destroy(self.handle)
        except Exception:
            pass

    def forward_dynamics(self, q, v, tau) -> tuple[int, np.ndarray]:
        out = np.zeros(self.nv)
        st = self.lib.ref_forward_dynamics(self.handle, _dp(np.ascontiguousarray(q, np.float64)), _dp(np.ascontiguousarray(v, np.float64)),
                                           _dp(np.ascontiguousarray(tau, np.float64)), _dp(out))
        return st, out

    def mass_matrix(self, q) -> np.ndarray:
        out = np.zeros((self.nv, self.nv))
        self.lib.ref_mass_matrix(self.handle, _dp(np.ascontiguousarray(q, np.float64)), _dp(out))
        return out

    def point_jacobian(self, q, body: int, local) -> tuple[np.ndarray, np.ndarray]:
        wp = np.zeros(3)
        J = np.zeros((3, self.nv))
        self.lib.ref_point_jacobian(self.handle, _dp(np.ascontiguousarray(q, np.float64)), body,
                                    _dp(np.ascontiguousarray(local, np.float64)), _dp(wp), _dp(J))
        return wp, J

    def integrate(self, q, v, tau) -> int:
        return self.lib.ref_integrate(self.handle, _dp(q), _dp(v), _dp(np.ascontiguousarray(tau, np.float64)))

    def conic_solve(self, inverse_mass, free_velocity, jac, mu, target, reg):
        n = len(mu)
        imp = np.zeros(3 * n)
        vel = np.zeros(self.nv if inverse_mass.shape[0] == self.nv else inverse_mass.shape[0])
        viol = ct.c_double(0.0)
        nv = inverse_mass.shape[0]
        st = self.lib.ref_conic_solve(nv, _dp(np.ascontiguousarray(inverse_mass, np.float64)),
                                      _dp(np.ascontiguousarray(free_velocity, np.float64)), n,
                                      _dp(np.ascontiguousarray(jac, np.float64)), _dp(np.ascontiguousarray(mu, np.float64)),
                                      _dp(np.ascontiguousarray(target, np.float64)), _dp(np.ascontiguousarray(reg, np.float64)),
                                      _dp(imp), _dp(vel), ct.byref(viol))
        return st, imp, vel, viol.value

    def contact_cache(self):
        """A persistent-manifold cache for articulated_contacts (one per environment)."""

        L = self.lib
        L.ref_contact_cache_create.restype = ct.c_void_p
        L.ref_contact_cache_destroy.argtypes = [ct.c_void_p]
        handle = L.ref_contact_cache_create()

        class _Cache:
            def __init__(self, h):
                self.handle = h

            def __del__(self):
                try:
                    L.ref_contact_cache_destroy(self.handle)
                except Exception:
                    pass

        return _Cache(handle)

    def articulated_contacts(self, cache, q, vf):
        """The reference CPU world step's collision and ConstraintIR
        evaluation at (q, vf).  Returns (status, raw [n, 16], manifolds
        [m, 58], rows [k, CONTACT_ROW]); shape indices are record indices."""

        L = self.lib
        L.ref_articulated_contacts.restype = ct.c_int
        L.ref_articulated_contacts.argtypes = [ct.c_void_p, ct.c_void_p, _DP, _DP, ct.c_uint32, _DP, ct.POINTER(ct.c_uint32),
                                               ct.c_uint32, _DP, ct.POINTER(ct.c_uint32), ct.c_uint32, _DP, ct.POINTER(ct.c_uint32)]
        raw, man, rows = np.zeros((256, 16)), np.zeros((128, 58)), np.zeros((256, CONTACT_ROW))
        nr, nm, nc = ct.c_uint32(0), ct.c_uint32(0), ct.c_uint32(0)
        st = L.ref_articulated_contacts(self.handle, cache.handle, _dp(np.ascontiguousarray(q, np.float64)),
                                        _dp(np.ascontiguousarray(vf, np.float64)), 256, _dp(raw), ct.byref(nr), 128, _dp(man),
                                        ct.byref(nm), 256, _dp(rows), ct.byref(nc))
        return int(st), raw[: nr.value].copy(), man[: nm.value].copy(), rows[: nc.value].copy()

    def run(self, q: np.ndarray, v: np.ndarray, actions: np.ndarray, substeps: int, threads: int, solver: int = 1):
        """Steps every env for actions.shape[0] control steps; returns (seconds, failed)."""

        envs = q.shape[0]
        steps = actions.shape[0]
        failed = ct.c_uint64(0)
        acts = np.ascontiguousarray(actions, np.float32)
        secs = self.lib.ref_run(self.handle, envs, _dp(q), _dp(v), acts.ctypes.data_as(ct.POINTER(ct.c_float)), steps, substeps,
                                threads, solver, ct.byref(failed))
        return secs, int(failed.value)


def reference_islands(dynamic: np.ndarray, pairs: np.ndarray) -> tuple[int, np.ndarray]:
    """buildConstraintIslands (ConstraintSolver.cpp:848) over a contact set of
    (bodyA, bodyB) pairs: (island count, island index per body, 0xffffffff
    for a body in no island)."""

    lib = ct.CDLL(str(REF_LIB))
    lib.ref_build_islands.restype = ct.c_uint32
    lib.ref_build_islands.argtypes = [ct.c_uint32, ct.POINTER(ct.c_uint8), ct.c_uint32, ct.POINTER(ct.c_uint32),
                                      ct.POINTER(ct.c_uint32)]
    dyn = np.ascontiguousarray(dynamic, np.uint8)
    pr = np.ascontiguousarray(pairs, np.uint32).reshape(-1)
    out = np.zeros(len(dyn), np.uint32)
    n = lib.ref_build_islands(len(dyn), dyn.ctypes.data_as(ct.POINTER(ct.c_uint8)), len(pr) // 2,
                              pr.ctypes.data_as(ct.POINTER(ct.c_uint32)), out.ctypes.data_as(ct.POINTER(ct.c_uint32)))
    return int(n), out


class ReferenceBatch:
    """One reference model per environment, each with that environment's
    friction scale, stepped together by the reference's CPU world step
    (stepControlledArticulatedWorldCpu) on `threads` host threads."""

    def __init__(self, records, h: float, friction: np.ndarray) -> None:
        self.models = [Reference(records, h, float(f)) for f in np.asarray(friction, np.float64)]
        lib = self.models[0].lib
        lib.ref_run_envs.restype = ct.c_double
        lib.ref_run_envs.argtypes = [ct.POINTER(ct.c_void_p), ct.c_uint32, _DP, _DP, ct.POINTER(ct.c_float), ct.c_uint32,
                                     ct.c_uint32, ct.c_uint32, ct.c_int, ct.POINTER(ct.c_uint64)]
        self.lib = lib
        self.handles = (ct.c_void_p * len(self.models))(*[m.handle for m in self.models])

    def run(self, q: np.ndarray, v: np.ndarray, actions: np.ndarray, substeps: int, threads: int, solver: int = 1):
        """Steps env e (q[e], v[e], float64, in place) for actions.shape[0]
        control steps; returns (seconds, failed substeps)."""

        envs = q.shape[0]
        assert envs == len(self.models) and q.dtype == np.float64 and v.dtype == np.float64
        failed = ct.c_uint64(0)
        acts = np.ascontiguousarray(actions, np.float32)
        secs = self.lib.ref_run_envs(self.handles, envs, _dp(q), _dp(v), acts.ctypes.data_as(ct.POINTER(ct.c_float)),
                                     actions.shape[0], substeps, threads, solver, ct.byref(failed))
        return secs, int(failed.value)


SCENE_MANIFOLDS = 128
SCENE_SLOT_WORDS = 57


class OracleSceneSlot(ct.Structure):
    _fields_ = [("key", ct.c_uint32), ("reserved", ct.c_uint32), ("m", OracleManifold)]


class OracleSceneTrace(ct.Structure):
    _fields_ = [
        ("status", ct.c_uint32),
        ("failing_index", ct.c_uint32),
        ("contact_count", ct.c_uint32),
        ("manifold_count", ct.c_uint32),
        ("raw_count", ct.c_uint32),
        ("candidate_pairs", ct.c_uint32),
        ("islands", ct.c_uint32),
        ("band_decisions", ct.c_uint32),
        ("min_decision_margin", ct.c_double),
        ("island_contacts", ct.c_uint32),
        ("island_pairs", ct.c_int32 * 512),
        ("island_of", ct.c_uint32 * 64),
    ]


class SceneTable:
    """Persistent manifolds of one pile environment, sorted by pair key."""

    def __init__(self) -> None:
        self.slots = (OracleSceneSlot * SCENE_MANIFOLDS)()
        self.count = ct.c_uint32(0)

    def keys(self) -> list[int]:
        return [int(self.slots[i].key) for i in range(self.count.value)]


class SceneOracle:
    """The C restatement of the free-body (pile) control step."""

    def __init__(self, records, h: float, substeps: int, velocity_iterations: int, final_velocity_iterations: int) -> None:
        if not ORACLE_LIB.is_file():
            build(reference=False)
        lib = ct.CDLL(str(ORACLE_LIB))
        self.lib = lib
        lib.oracle_scene_create.restype = ct.c_void_p
        lib.oracle_scene_create.argtypes = [ct.c_void_p] * 6 + [ct.c_uint32, ct.c_double, ct.c_uint32, ct.c_uint32, ct.c_uint32]
        lib.oracle_scene_destroy.argtypes = [ct.c_void_p]
        lib.oracle_scene_step.restype = ct.c_uint32
        lib.oracle_scene_step.argtypes = [ct.c_void_p, _DP, _DP, ct.c_void_p, ct.POINTER(ct.c_uint32), ct.c_double, ct.c_void_p]
        lib.oracle_scene_collide.restype = ct.c_uint32
        lib.oracle_scene_collide.argtypes = [ct.c_void_p, _DP, ct.c_void_p, ct.POINTER(ct.c_uint32), _DP, ct.c_uint32,
                                             ct.POINTER(ct.c_uint32)]
        lib.oracle_scene_table_from_device.argtypes = [ct.POINTER(ct.c_float), ct.c_uint32, ct.c_void_p]
        lib.oracle_scene_raw_contacts.restype = ct.c_uint32
        lib.oracle_scene_raw_contacts.argtypes = [ct.c_void_p, _DP, ct.c_uint32, ct.c_uint32, ct.c_double, ct.c_double, _DP]
        lib.oracle_scene_pair_query.restype = ct.c_uint32
        lib.oracle_scene_pair_query.argtypes = [ct.c_void_p, _DP, ct.c_uint32, ct.c_uint32, ct.c_uint32, _DP,
                                                ct.POINTER(ct.c_uint32), ct.POINTER(ct.c_uint32)]
        self.records = records
        w = records.world
        self.nb = int(w.body_count) - 1
        self.h = h
        hull = getattr(records, "hull_vertices", None)
        self._hull = None if hull is None else np.ascontiguousarray(hull, np.float32)
        self.handle = lib.oracle_scene_create(
            ct.byref(records.world), ct.cast(records.bodies, ct.c_void_p), ct.cast(records.shapes, ct.c_void_p),
            ct.cast(records.materials, ct.c_void_p), ct.cast(records.pairs, ct.c_void_p),
            None if self._hull is None else self._hull.ctypes.data_as(ct.c_void_p),
            0 if self._hull is None else len(self._hull), h, substeps, velocity_iterations, final_velocity_iterations)
        if not self.handle:
            raise RuntimeError("oracle_scene_create failed")

    def __del__(self) -> None:
        try:
            if self.handle:
                self.lib.oracle_scene_destroy(self.handle)
        except Exception:
            pass

    def table_from_device(self, words: np.ndarray, count: int) -> SceneTable:
        """Oracle copy of one environment's device manifold table ([slot][57] float32)."""

        t = SceneTable()
        w = np.ascontiguousarray(words, np.float32)
        self.lib.oracle_scene_table_from_device(w.ctypes.data_as(ct.POINTER(ct.c_float)), int(count), ct.cast(t.slots, ct.c_void_p))
        t.count.value = int(count)
        return t

    def step(self, q: np.ndarray, v: np.ndarray, table: SceneTable, friction: float):
        """One control step of one env; q, v (float64) and table in place."""

        assert q.dtype == np.float64 and v.dtype == np.float64
        trace = OracleSceneTrace()
        status = self.lib.oracle_scene_step(self.handle, _dp(q), _dp(v), ct.cast(table.slots, ct.c_void_p), ct.byref(table.count),
                                            float(friction), ct.byref(trace))
        return int(status), trace

    def collide(self, q: np.ndarray, table: SceneTable, raw_cap: int = 1024):
        """Narrowphase + manifold update over all compiled pairs; returns (status, raw rows [n, 16])."""

        raw = np.zeros((raw_cap, 16))
        n = ct.c_uint32(0)
        st = self.lib.oracle_scene_collide(self.handle, _dp(np.ascontiguousarray(q, np.float64)), ct.cast(table.slots, ct.c_void_p),
                                           ct.byref(table.count), _dp(raw), raw_cap, ct.byref(n))
        return int(st), raw[: n.value].copy()

    def raw_contacts(self, q: np.ndarray, a: int, b: int, margin_a: float = 0.0, margin_b: float = 0.0) -> np.ndarray:
        out = np.zeros((8, 12))
        n = self.lib.oracle_scene_raw_contacts(self.handle, _dp(np.ascontiguousarray(q, np.float64)), a, b, margin_a, margin_b,
                                               _dp(out))
        return out[:n].copy()

    def pair_query(self, q: np.ndarray, a: int, b: int, pair_class: int) -> tuple[int, np.ndarray, int]:
        """Raw contacts of pair (a, b) under `pair_class` (11: support-mapped GJK / EPA / MPR);
        (status, rows [n, 12], path: 0 GJK distance, 3 EPA, 1 MPR)."""

        out = np.zeros((8, 12))
        st, path = ct.c_uint32(0), ct.c_uint32(0)
        n = self.lib.oracle_scene_pair_query(self.handle, _dp(np.ascontiguousarray(q, np.float64)), a, b, pair_class, _dp(out),
                                             ct.byref(st), ct.byref(path))
        return int(st.value), out[:n].copy(), int(path.value)


class ReferenceScene:
    """The reference's FP64 collision oracle (collideCpuReference) over one pile."""

    def __init__(self, records) -> None:
        if not REF_LIB.is_file():
            raise FileNotFoundError(f"{REF_LIB} is missing; build it with `make -C oracle ref` where the reference sources exist")
        lib = ct.CDLL(str(REF_LIB))
        self.lib = lib
        lib.ref_scene_create.restype = ct.c_void_p
        lib.ref_scene_create.argtypes = [ct.c_void_p] * 3 + [ct.c_char_p, ct.c_size_t]
        lib.ref_scene_destroy.argtypes = [ct.c_void_p]
        lib.ref_scene_collide.restype = ct.c_int
        lib.ref_scene_collide.argtypes = [ct.c_void_p, _DP, ct.c_uint32, _DP, ct.POINTER(ct.c_uint32), ct.c_uint32, _DP,
                                          ct.POINTER(ct.c_uint32)]
        err = ct.create_string_buffer(512)
        self.handle = lib.ref_scene_create(ct.byref(records.world), ct.cast(records.bodies, ct.c_void_p),
                                           ct.cast(records.shapes, ct.c_void_p), err, len(err))
        if not self.handle:
            raise RuntimeError(err.value.decode())

    def __del__(self) -> None:
        try:
            if self.handle:
                self.lib.ref_scene_destroy(self.handle)
        except Exception:
            pass

    def collide(self, q: np.ndarray, raw_cap: int = 1024, manifold_cap: int = 512):
        """Returns (status, raw rows [n, 16], manifold rows [m, 58]); manifolds persist across calls."""

        raw = np.zeros((raw_cap, 16))
        man = np.zeros((manifold_cap, 58))
        nr, nm = ct.c_uint32(0), ct.c_uint32(0)
        st = self.lib.ref_scene_collide(self.handle, _dp(np.ascontiguousarray(q, np.float64)), raw_cap, _dp(raw), ct.byref(nr),
                                        manifold_cap, _dp(man), ct.byref(nm))
        return int(st), raw[: nr.value].copy(), man[: nm.value].copy()
