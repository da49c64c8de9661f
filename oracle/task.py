"""Oracle for the task layer -- test infrastructure only (tests/ and the
smoke check import it; the product never does).

An FP64 restatement, one environment at a time, of the reference's task
kernels for the operator subset the device evaluates
(src/metal/LocomotionTask.metal):

* ``observe``  -- mr_locomotion_task_observe (:2184-3440): the reset test
  (:2329-2333), reset pose from default_q plus the randomization operators
  (:2337-2770), the new episode's state (:2947-3010) and its actor frame
  (writeFrame :1190-1330 on the reset state, :3070-3098);
* ``apply``    -- mr_locomotion_task_apply_actions (:3442-3674);
* ``complete`` -- mr_locomotion_task_complete (:3904-6745): reward inputs
  (:4376-4500), reward operators (:4700-5960), breakdown lanes (:5985-6046),
  terminations (:6064-6160), command schedule and state (:6388-6440), next
  actor frame and joint history (:6478-6630), transition (:6697-6742);
  the contact groups' metrics (:4104-4370) from the committed contacts and
  the contact-group rewards (:5405-5553).

Draws use the reference's keyed counter hash (randomUnit :121-152): a key of
seed, environment, episode, control step and channel through SplitMix64's
finaliser, the top 24 bits scaled to [0, 1).

Parity unpinned against the reference itself: the reference evaluates its
task program only in Metal shaders (there is no CPU path to run here).  The
restatement is checked against closed forms in tests/test_task_oracle.py and
the device against it in tests/test_task_gpu.py.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

M64 = (1 << 64) - 1
M32 = (1 << 32) - 1
TWO_PI = 2.0 * math.pi

OBS_ROOT_ANGULAR, OBS_GRAVITY, OBS_COMMAND, OBS_JOINT_ERROR, OBS_JOINT_VELOCITY, OBS_PREVIOUS_ACTION = 0, 1, 2, 3, 4, 5
OBS_ROOT_LINEAR, OBS_ROOT_HEIGHT, OBS_GAIT_PHASE, OBS_DELAYED_ACTION, OBS_JOINT_FD_VELOCITY = 6, 7, 14, 26, 27
NORMALIZE = 1
R_LINEAR, R_YAW, R_CONSTANT, R_VERTICAL, R_ROLL_PITCH, R_TILT, R_HEIGHT_ERROR = 0, 1, 2, 3, 4, 5, 6
R_JOINT_VELOCITY, R_JOINT_ACCELERATION, R_ACTION_RATE, R_LIMIT_SQUARED = 7, 8, 9, 10
R_POSTURE_SQUARED, R_POSTURE_ABSOLUTE, R_GRAVITY_HORIZONTAL, R_LIMIT_ABSOLUTE = 12, 17, 18, 20
R_HEIGHT_NORMALIZED, R_HEIGHT_PROGRESS, R_UPRIGHTNESS = 21, 22, 23
R_GAIT_MATCH, R_SWING_CLEARANCE, R_SUPPORT_SLIP, R_FORBIDDEN, R_FOOT_CLEARANCE = 13, 14, 15, 16, 19
OBS_CONTACT_METRIC, OBS_CONTACT_WRENCH, OBS_SUPPORT_SENSE = 8, 13, 18
T_MIN_HEIGHT, T_MAX_TILT, T_CONTACT_GROUP = 0, 1, 2
SUPPORT, FORBIDDEN = 1, 2
ALL_GROUPS = 0xFFFFFFFF
MANIFOLD_POINTS = 4
REASON_CONTINUING, REASON_TIMEOUT, REASON_PHYSICS_ERROR = 0, 4, 5
RND_ROOT_POSITION, RND_ROOT_YAW, RND_ACTION_POSITION, RND_VELOCITY = 0, 1, 2, 3
RND_ACTION_VELOCITY, RND_ROOT_HEIGHT, RND_JOINT_POSITION = 9, 10, 12
RND_ACTION_DELAY, RND_OBSERVATION_DELAY = 7, 8


def mix64(x: int) -> int:
    """SplitMix64's finaliser (LocomotionTask.metal:121-130)."""

    x = (x + 0x9E3779B97F4A7C15) & M64
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & M64
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & M64
    return x ^ (x >> 31)


def unit_draw(seed: int, env: int, episode: int, step: int, channel: int) -> float:
    """randomUnit (:132-152): the counters are 32-bit before widening."""

    key = seed & M64
    key ^= (((env + 1) & M32) * 0xD2B74407B1CE6E93) & M64
    key ^= (((episode + 1) & M32) * 0xCA5A826395121157) & M64
    key ^= (((step + 1) & M32) * 0x9E3779B185EBCA87) & M64
    key ^= (((channel + 1) & M32) * 0x94D049BB133111EB) & M64
    return float((mix64(key) >> 40) & 0xFFFFFF) / 16777216.0


def signed_draw(*args) -> float:
    return 2.0 * unit_draw(*args) - 1.0


def range_draw(seed, env, episode, step, channel, lower, upper) -> float:
    return lower + (upper - lower) * unit_draw(seed, env, episode, step, channel)


def rotate(q, v):
    u = np.asarray(q[:3], np.float64)
    t = 2.0 * np.cross(u, v)
    return np.asarray(v, np.float64) + q[3] * t + np.cross(u, t)


def rotate_inverse(q, v):
    u = np.asarray(q[:3], np.float64)
    t = 2.0 * np.cross(u, v)
    return np.asarray(v, np.float64) - q[3] * t + np.cross(u, t)


def quat_product(a, b):
    return np.array([a[3] * b[0] + a[0] * b[3] + a[1] * b[2] - a[2] * b[1],
                     a[3] * b[1] - a[0] * b[2] + a[1] * b[3] + a[2] * b[0],
                     a[3] * b[2] + a[0] * b[1] - a[1] * b[0] + a[2] * b[3],
                     a[3] * b[3] - a[0] * b[0] - a[1] * b[1] - a[2] * b[2]])


def normalized_or(v, fallback):
    l2 = float(np.dot(v, v))
    return np.asarray(v, np.float64) / math.sqrt(l2) if l2 > 1.0e-12 and math.isfinite(l2) else np.asarray(fallback, np.float64)


def stable_tangent(n):
    a = np.abs(n)
    ref = np.array([1.0, 0.0, 0.0]) if a[0] <= a[1] and a[0] <= a[2] else (np.array([0.0, 1.0, 0.0]) if a[1] <= a[2] else
                                                                           np.array([0.0, 0.0, 1.0]))
    t = np.cross(ref, n)
    return t / np.linalg.norm(t)


@dataclass
class EnvState:
    """One environment's task record (MRTaskStateGPU's used lanes) plus its
    delay line [history][na], joint history [2][na] and next actor frame."""

    history: np.ndarray
    previous_joint: np.ndarray
    frame: np.ndarray
    episode_step: int = 0
    episode: int = 0
    command_steps: int = 0
    initialized: bool = False
    pending_reset: bool = False
    last_reason: int = 0
    command: np.ndarray = field(default_factory=lambda: np.zeros(3))
    phase: float = 0.0
    previous_height: float = 0.0
    episode_return: float = 0.0
    episode_tracking: float = 0.0
    air: np.ndarray = field(default_factory=lambda: np.zeros(8))
    critic: np.ndarray = field(default_factory=lambda: np.zeros(0))
    action_delay: int = 0
    observation_delay: int = 0
    band: int = 0


class TaskOracle:
    """The task layer over one rollout: `program` a numi_lab_b200.task.TaskProgram."""

    def __init__(self, program, *, nq: int, nv: int, dt: float, seed: int, fixed_root: bool, limit_lower, limit_upper,
                 terminations: bool = True, records=None, world=None, physics_dt: float = 0.0,
                 band_range: tuple[int, int] | None = None) -> None:
        """`records` (compiled world) and `world` (an oracle.Oracle of it,
        for body states) serve the contact groups; `physics_dt` is the
        microstep; `band_range` the rollout's sampled difficulty bands
        (None: every band)."""

        self.p = program
        self.nq, self.nv, self.dt, self.seed, self.fixed_root = nq, nv, float(dt), int(seed), fixed_root
        self.na = len(program.actions)
        self.nobs = len(program.actor)
        self.L = int(program.action_history)
        self.H = int(getattr(program, "observation_history", 1))  # stacked actor frames, oldest first
        self.delay = min(int(program.action_delay_steps), self.L - 2)
        self.lo = np.asarray(limit_lower, np.float64)
        self.hi = np.asarray(limit_upper, np.float64)
        self.default_q = np.asarray(program.default_q, np.float64)
        self.terminations = program.terminations if terminations else []
        self.bands = max(int(getattr(program, "difficulty_band_count", 1)), 1)
        self.band_range = band_range
        self.records, self.world, self.physics_dt = records, world, float(physics_dt)
        self.groups = list(getattr(program, "contact_groups", []))
        self.metrics = np.zeros((len(self.groups), 12))
        if records is not None:
            self.ground = 0.0
            for i in range(int(records.world.shape_count)):
                sh = records.shapes[i]
                if int(sh.shape_type) == 3:
                    pose = np.array(records.bodies[int(sh.body)].static_pose, np.float64)
                    self.ground = float(pose[2] + rotate(pose[4:8] / np.linalg.norm(pose[4:8]), np.array(sh.local_position[:3], np.float64))[2])
                    self.plane_pose = (pose[:3], pose[4:8] / np.linalg.norm(pose[4:8]))
                    break

    # -- contact groups (LocomotionTask.metal:4104-4370) -------------------------
    def contact_metrics(self, st: EnvState, q, v, manifolds) -> np.ndarray:
        """[group][12] metrics of one finished step from its committed
        manifolds (MRManifoldC, one per compiled pair): force (forbidden
        groups: the hard-contact flag), slip, air time, clearance, CoP x, y,
        then the wrench in the reference body's frame.  Updates st.air."""

        rec = self.records
        bs = self.world.body_states(np.asarray(q, np.float64), np.asarray(v, np.float64))
        ng = len(self.groups)
        imp, hard = np.zeros(ng), np.zeros(ng)
        F, Mo, Pw = np.zeros((ng, 3)), np.zeros((ng, 3)), np.zeros((ng, 3))
        for pidx in range(int(rec.world.pair_count)):
            pr = rec.pairs[pidx]
            sa, sb = rec.shapes[int(pr.shape_a)], rec.shapes[int(pr.shape_b)]
            body = int(sa.body)
            if int(rec.bodies[int(sb.body)].articulated) or not int(rec.bodies[body].articulated):
                continue
            m = manifolds[pidx]
            count = int(m.count)
            if count <= 0:
                continue
            ra, ca = bs[body, 3:7], bs[body, :3]
            n = rotate(ra, np.array(m.normal_local, np.float64))
            n = n / np.linalg.norm(n)
            t = rotate(ra, np.array(m.tangent_local, np.float64))
            t = t - np.dot(t, n) * n
            t = t / np.linalg.norm(t) if np.dot(t, t) > 1e-12 else stable_tangent(n)
            b = np.cross(n, t)
            for i in range(min(count, MANIFOLD_POINTS)):
                pt = m.points[i]
                pa = ca + rotate(ra, np.array(pt.anchor_a, np.float64))
                pb = self.plane_pose[0] + rotate(self.plane_pose[1], np.array(pt.anchor_b, np.float64))
                pw = 0.5 * (pa + pb)
                ln, lt, lb = (float(x) for x in pt.impulses)
                fo = -(n * ln + t * lt + b * lb)
                a = abs(ln)
                for g, G in enumerate(self.groups):
                    if body not in G.bodies:
                        continue
                    imp[g] += a
                    hard[g] = max(hard[g], a)
                    F[g] += fo
                    Mo[g] += np.cross(pw, fo)
                    Pw[g] += a * pw
        out = np.zeros((ng, 12))
        for g, G in enumerate(self.groups):
            rb = G.reference_body
            cr, rr, vr, wr = bs[rb, :3], bs[rb, 3:7], bs[rb, 7:10], bs[rb, 10:13]
            ref = cr + rotate(rr, np.array(G.local_reference[:3], np.float64))
            Fw, Mw = F[g] / self.physics_dt, Mo[g] / self.physics_dt
            out[g, 6:9] = rotate_inverse(rr, Fw)
            out[g, 9:12] = rotate_inverse(rr, Mw - np.cross(ref, Fw))
            if G.flags & SUPPORT:
                force = imp[g] / self.physics_dt
                touching = force > self.p.support_force_threshold
                koff = rotate(rr, np.array(G.kinematic_reference[:3], np.float64))
                kv = vr + np.cross(wr, koff)
                out[g, 0] = force
                out[g, 1] = math.hypot(kv[0], kv[1]) if touching else 0.0
                out[g, 2] = 0.0 if touching else st.air[g] + self.dt
                out[g, 3] = ref[2] - G.local_reference[3] - self.ground
                if imp[g] > 1e-6:
                    cl = rotate_inverse(rr, Pw[g] - imp[g] * ref)
                    out[g, 4:6] = cl[:2] / imp[g]
            elif G.flags & FORBIDDEN:
                out[g, 0] = 1.0 if hard[g] / self.physics_dt > self.p.support_force_threshold else 0.0
        st.air[:ng] = out[:, 2]
        return out

    @staticmethod
    def desired_support(G, phase: float) -> bool:
        x = math.fmod(phase + G.gait_phase_offset, TWO_PI)
        if x < 0.0:
            x += TWO_PI
        return x / TWO_PI < G.stance_fraction

    def new_state(self) -> EnvState:
        return EnvState(np.zeros((self.L, self.na)), np.zeros((2, self.na)), np.zeros((self.H, self.nobs)))

    # -- root frame (:396-478) ------------------------------------------------
    def root(self, q, v):
        if self.fixed_root:
            z = np.zeros(3)
            return np.array([0.0, 0.0, 0.0, 1.0]), z, z, z
        o = np.asarray(q[3:7], np.float64)
        off = rotate(o, np.asarray(self.p.root_reference, np.float64))
        ang = np.asarray(v[3:6], np.float64)
        return o, np.asarray(q[:3], np.float64) + off, np.asarray(v[:3], np.float64) + np.cross(ang, off), ang

    @staticmethod
    def gravity(o):
        down = np.array([0.0, 0.0, -1.0])
        return normalized_or(rotate_inverse(o, down), down)

    def clean(self, op, q, v, st: EnvState, raw_slot: int, previous_q, metrics=None) -> float:
        o, pos, lin, ang = self.root(q, v)
        c = op.component
        b = self.p.actions[op.source] if op.opcode in (OBS_JOINT_ERROR, OBS_JOINT_VELOCITY, OBS_JOINT_FD_VELOCITY) else None
        if op.opcode == OBS_ROOT_ANGULAR:
            value = rotate_inverse(o, ang)[c]
        elif op.opcode == OBS_GRAVITY:
            value = self.gravity(o)[c]
        elif op.opcode == OBS_COMMAND:
            value = st.command[c] if c < 3 else 0.0
        elif op.opcode == OBS_JOINT_ERROR:
            value = q[b.q_index] - self.default_q[b.q_index]
        elif op.opcode == OBS_JOINT_VELOCITY:
            value = v[b.v_index]
        elif op.opcode == OBS_JOINT_FD_VELOCITY:
            value = (q[b.q_index] - previous_q[op.source]) / self.dt
        elif op.opcode == OBS_PREVIOUS_ACTION:
            value = st.history[raw_slot, op.source]
        elif op.opcode == OBS_DELAYED_ACTION:
            value = st.history[raw_slot - c, op.source]
        elif op.opcode == OBS_ROOT_LINEAR:
            value = rotate_inverse(o, lin)[c]
        elif op.opcode == OBS_ROOT_HEIGHT:
            value = pos[2]
        elif op.opcode == OBS_CONTACT_METRIC:
            value = metrics[op.source, c] if metrics is not None else 0.0
        elif op.opcode == OBS_CONTACT_WRENCH:
            value = metrics[op.source, 6 + c] if metrics is not None else 0.0
        elif op.opcode == OBS_SUPPORT_SENSE:
            total = signed = slip = 0.0
            for g, G in enumerate(self.groups):
                if metrics is None or not G.flags & SUPPORT:
                    continue
                load = max(metrics[g, 0], 0.0)
                total += load
                signed += load * math.cos(G.gait_phase_offset)
                slip = max(slip, max(metrics[g, 1], 0.0))
            value = total if c == 0 else ((signed / total if total > 1e-6 else 0.0) if c == 1 else slip)
        elif op.opcode == OBS_GAIT_PHASE:
            value = (math.sin(st.phase) if c == 0 else math.cos(st.phase)) if np.linalg.norm(st.command) >= 0.1 else 0.0
        else:
            raise ValueError(f"opcode {op.opcode} is outside the subset")
        return op.scale * float(value) + op.offset

    def frame(self, env, q, v, st: EnvState, raw_slot: int, previous_q, episode: int, step: int, metrics=None) -> np.ndarray:
        """writeFrame (:1190-1330)."""

        g = np.array([0.0, 0.0, -1.0])
        have = False
        for op in self.p.actor:
            if op.opcode == OBS_GRAVITY and op.flags & NORMALIZE:
                g[op.component] = self.clean(op, q, v, st, raw_slot, previous_q, metrics) + op.noise_amplitude * signed_draw(
                    self.seed, env, episode, step, op.noise_channel)
                have = True
        if have:
            g = normalized_or(g, [0.0, 0.0, -1.0])
        out = np.zeros(self.nobs)
        for i, op in enumerate(self.p.actor):
            if op.opcode == OBS_GRAVITY and op.flags & NORMALIZE:
                out[i] = g[op.component]
            else:
                out[i] = self.clean(op, q, v, st, raw_slot, previous_q, metrics) + op.noise_amplitude * signed_draw(
                    self.seed, env, episode, step, op.noise_channel)
        return out

    def critic_frame(self, q, v, st: EnvState, raw_slot: int, previous_q, metrics=None) -> np.ndarray:
        """writeCriticFrame (:1403-1456): the critic operators' clean values."""

        return np.array([self.clean(op, q, v, st, raw_slot, previous_q, metrics) for op in getattr(self.p, "critic", [])])

    def duration_steps(self, env, episode, step, channel) -> int:
        lo, hi = self.p.command_duration_seconds
        return max(1, int(math.floor(range_draw(self.seed, env, episode, step, channel, lo, hi) / self.dt)))

    def sample_band(self, env, episode) -> int:
        """sampledDifficultyBand (LocomotionTask.metal:1537-1568)."""

        lo, hi = (0, 0xFFFFFFFF) if self.band_range is None else self.band_range
        lo = min(lo, self.bands - 1)
        hi = max(lo, min(self.bands - 1 if hi == 0xFFFFFFFF else hi, self.bands - 1))
        n = hi - lo + 1
        if n == 1:
            return lo
        u = unit_draw(self.seed, env, episode, 0, 15) ** max(float(getattr(self.p, "band_sampling_exponent", 1.0)), 0.01)
        return lo + min(int(math.floor(u * n)), n - 1)

    def sample_command(self, env, episode, step, band: int = 0) -> np.ndarray:
        """sampledCommand (:1570-1615): each band widens the range by the
        step, within the limits."""

        p = self.p
        step_k = getattr(p, "command_band_step", (0.0, 0.0, 0.0))
        lim_lo = getattr(p, "command_limit_lower", None) or p.command_lower
        lim_hi = getattr(p, "command_limit_upper", None) or p.command_upper
        lower = [max(p.command_lower[k] - band * step_k[k], lim_lo[k]) for k in range(3)]
        upper = [min(p.command_upper[k] + band * step_k[k], lim_hi[k]) for k in range(3)]
        cmd = np.array([range_draw(self.seed, env, episode, step, 16 + k, lower[k], upper[k]) for k in range(3)])
        if unit_draw(self.seed, env, episode, step, 19) < self.p.standing_probability:
            cmd[:] = 0.0
        return cmd

    # -- the three stages --------------------------------------------------------
    def observe(self, env: int, st: EnvState, q, v, mask: bool):
        """Returns (reset, reset_q, reset_v, observation)."""

        reset = (not st.initialized) or st.pending_reset or bool(mask)
        if not reset:
            return False, None, None, st.frame.reshape(-1).copy()
        episode = st.episode + 1
        rq = self.default_q.copy()
        st.action_delay, st.observation_delay = self.delay, 0
        st.band = self.sample_band(env, episode)
        rv = np.zeros(self.nv)
        for k, op in enumerate(self.p.randomization):
            ch = 2048 + k
            if st.band < getattr(op, "minimum_band", 0):
                continue
            a, b = op.parameters[0], op.parameters[1]
            if op.opcode == RND_ROOT_POSITION:
                for c in range(3):
                    rq[c] += op.parameters[c] * signed_draw(self.seed, env, episode, 0, ch + c)
            elif op.opcode == RND_ROOT_YAW:
                half = 0.5 * range_draw(self.seed, env, episode, 0, ch, a, b)
                rq[3:7] = quat_product([0.0, 0.0, math.sin(half), math.cos(half)], self.default_q[3:7])
            elif op.opcode == RND_ROOT_HEIGHT:
                rq[2] = range_draw(self.seed, env, episode, 0, ch, a, b)
            elif op.opcode == RND_JOINT_POSITION:
                rq[op.target] = range_draw(self.seed, env, episode, 0, ch, a, b)
            elif op.opcode == RND_ACTION_POSITION:
                for i, bd in enumerate(self.p.actions):
                    x = self.default_q[bd.q_index] + range_draw(self.seed, env, episode, 0, ch + i, a, b)
                    rq[bd.q_index] = min(max(x, bd.lower_target), bd.upper_target)
            elif op.opcode == RND_VELOCITY:
                for i in range(self.nv):
                    rv[i] = range_draw(self.seed, env, episode, 0, ch + i, a, b)
            elif op.opcode in (RND_ACTION_DELAY, RND_OBSERVATION_DELAY):
                lo_d = int(max(op.parameters[0], 0.0))
                hi_d = int(max(op.parameters[1], op.parameters[0]))
                d = lo_d + int(math.floor((hi_d - lo_d + 1) * unit_draw(self.seed, env, episode, 0, ch)))
                if op.opcode == RND_ACTION_DELAY:
                    st.action_delay = min(d, self.L - 1)
                else:
                    st.observation_delay = min(d, int(getattr(self.p, "maximum_observation_delay", 0)), 8)
            elif op.opcode == RND_ACTION_VELOCITY:
                for i, bd in enumerate(self.p.actions):
                    rv[bd.v_index] = range_draw(self.seed, env, episode, 0, ch + i, a, b)
            else:
                raise ValueError(f"randomization opcode {op.opcode} is outside the subset")
        st.history[:] = 0.0
        st.air[:] = 0.0
        st.previous_joint[0] = 0.0
        st.previous_joint[1] = [rq[bd.q_index] for bd in self.p.actions]
        st.episode_step, st.episode = 0, episode
        st.command_steps = self.duration_steps(env, episode, 0, 32)
        st.initialized, st.pending_reset, st.last_reason = True, False, REASON_CONTINUING
        st.command = self.sample_command(env, episode, 0, st.band)
        st.phase = 0.0
        st.previous_height = self.root(rq, rv)[1][2]
        st.episode_return = st.episode_tracking = 0.0
        first = self.frame(env, rq, rv, st, self.L - 2, st.previous_joint[1], episode, 0)
        st.critic = self.critic_frame(rq, rv, st, self.L - 2, st.previous_joint[1])
        st.frame = np.tile(first, (self.H, 1))  # every history slot the reset frame (:3072-3098)
        return True, rq, rv, st.frame.reshape(-1).copy()

    def apply(self, st: EnvState, actions) -> np.ndarray:
        """Drive targets [na] for the physics step (:3520-3668)."""

        filt, raw_last = self.L - 1, self.L - 2
        targets = np.zeros(self.na)
        for a, b in enumerate(self.p.actions):
            for d in range(raw_last):
                st.history[d, a] = st.history[d + 1, a]
            previous = st.history[filt, a]
            resp = min(max(1.0 - math.exp(-self.dt / b.response_time_seconds), 0.0), 1.0) if b.response_time_seconds > 0.0 else 1.0
            st.history[raw_last, a] = float(actions[a])
            delayed = st.history[raw_last - min(st.action_delay, raw_last), a]
            st.history[filt, a] = previous + (delayed - previous) * resp
            targets[a] = min(max(self.default_q[b.q_index] + b.scale * st.history[filt, a], b.lower_target), b.upper_target)
        return targets

    def complete(self, env: int, st: EnvState, q, v, status: int, manifolds=None) -> dict:
        """Reward, termination, schedule and the next actor frame of one
        finished physics step; returns the transition's fields."""

        p, dt = self.p, self.dt
        physics_error = status != 0
        o, pos, lin, ang = self.root(q, v)
        base_linear = rotate_inverse(o, lin)
        base_angular = rotate_inverse(o, ang)
        g = self.gravity(o)
        height = pos[2]
        tilt = math.atan2(math.hypot(g[0], g[1]), max(-g[2], 1.0e-6))
        yx, yy = 1.0 - 2.0 * (o[1] * o[1] + o[2] * o[2]), 2.0 * (o[3] * o[2] + o[0] * o[1])
        ys = 1.0 / math.sqrt(max(yx * yx + yy * yy, 1.0e-12))
        yx, yy = yx * ys, yy * ys
        fx, fy = yx * lin[0] + yy * lin[1], -yy * lin[0] + yx * lin[1]
        tracking_error = (fx - st.command[0]) ** 2 + (fy - st.command[1]) ** 2
        yaw_error = (base_angular[2] - st.command[2]) ** 2
        raw_last, raw_prev = self.L - 2, self.L - 3
        vel2 = acc2 = rate2 = lim2 = 0.0
        for a, b in enumerate(p.actions):
            rate2 += (st.history[raw_last, a] - st.history[raw_prev, a]) ** 2
            x, xd = q[b.q_index], v[b.v_index]
            acc = (xd - st.previous_joint[0, a]) / dt
            lower, upper = max(self.lo[a] - x, 0.0), max(x - self.hi[a], 0.0)
            vel2 += xd * xd
            acc2 += acc * acc
            lim2 += lower * lower + upper * upper
        phase = math.fmod(st.phase + TWO_PI * dt / p.gait_period_seconds, TWO_PI)
        moving = float(np.linalg.norm(st.command)) > 0.1
        gm = self.contact_metrics(st, q, v, manifolds) if self.groups else None
        reward = 0.0
        b0, b1 = np.zeros(4), np.zeros(4)
        for r in p.rewards:
            op, w = r.opcode, r.weight
            if op == R_LINEAR:
                value = math.exp(-tracking_error / max(r.parameters[0], 1.0e-8))
            elif op == R_YAW:
                value = math.exp(-yaw_error / max(r.parameters[0], 1.0e-8))
            elif op == R_CONSTANT:
                value = 1.0
            elif op == R_VERTICAL:
                value = base_linear[2] ** 2
            elif op == R_ROLL_PITCH:
                value = base_angular[0] ** 2 + base_angular[1] ** 2
            elif op == R_TILT:
                value = tilt * tilt
            elif op == R_GRAVITY_HORIZONTAL:
                value = g[0] ** 2 + g[1] ** 2
            elif op == R_HEIGHT_ERROR:
                value = (height - p.base_height_target) ** 2
            elif op == R_HEIGHT_NORMALIZED:
                value = min(max(height / max(p.base_height_target, 1.0e-6), 0.0), 1.0)
            elif op == R_HEIGHT_PROGRESS:
                value = min(max((height - st.previous_height) / dt, -2.0), 2.0)
            elif op == R_UPRIGHTNESS:
                value = min(max(-g[2], 0.0), 1.0) ** 2
            elif op == R_JOINT_VELOCITY:
                value = vel2
            elif op == R_JOINT_ACCELERATION:
                value = acc2
            elif op == R_ACTION_RATE:
                value = rate2
            elif op == R_LIMIT_SQUARED:
                value = lim2
            elif op == R_LIMIT_ABSOLUTE:
                soft = min(max(r.parameters[0], 1.0e-6), 1.0)
                value = 0.0
                for a, b in enumerate(p.actions):
                    center, half = 0.5 * (self.lo[a] + self.hi[a]), 0.5 * (self.hi[a] - self.lo[a]) * soft
                    x = q[b.q_index]
                    value += max(center - half - x, 0.0) + max(x - center - half, 0.0)
            elif op in (R_GAIT_MATCH, R_SWING_CLEARANCE, R_SUPPORT_SLIP, R_FORBIDDEN, R_FOOT_CLEARANCE):
                acc, count = 0.0, 0.0
                for g, G in enumerate(self.groups):
                    if r.group != ALL_GROUPS and r.group != g:
                        continue
                    m = gm[g]
                    support = bool(G.flags & SUPPORT)
                    if op == R_GAIT_MATCH and support:
                        acc += 1.0 if self.desired_support(G, phase) == (m[0] > p.support_force_threshold) else 0.0
                    elif op == R_SWING_CLEARANCE and support and not self.desired_support(G, phase):
                        acc += math.exp(-((m[3] - p.clearance_target) ** 2) / max(r.parameters[0], 1e-8))
                        count += 1.0
                    elif op == R_SUPPORT_SLIP and support:
                        acc += m[1]
                    elif op == R_FORBIDDEN and G.flags & FORBIDDEN:
                        acc = max(acc, m[0])
                    elif op == R_FOOT_CLEARANCE and support:
                        bs = self.world.body_states(np.asarray(q, np.float64), np.asarray(v, np.float64))
                        rb = G.reference_body
                        off = rotate(bs[rb, 3:7], np.array(G.kinematic_reference[:3], np.float64))
                        vel = bs[rb, 7:10] + np.cross(bs[rb, 10:13], off)
                        e = bs[rb, 2] + off[2] - p.clearance_target
                        acc += e * e * math.tanh(r.parameters[1] * math.hypot(vel[0], vel[1]))
                if op == R_FOOT_CLEARANCE:
                    value = math.exp(-acc / max(r.parameters[0], 1e-8))
                elif op == R_SWING_CLEARANCE:
                    value = acc / max(count, 1.0) if moving else 0.0
                elif op == R_GAIT_MATCH:
                    value = acc if moving else 0.0
                else:
                    value = acc
            elif op in (R_POSTURE_SQUARED, R_POSTURE_ABSOLUTE):
                members = p.joint_groups[r.group]
                errs = [q[p.actions[m].q_index] - self.default_q[p.actions[m].q_index] for m in members]
                value = (sum(e * e for e in errs) / max(len(errs), 1)) if op == R_POSTURE_SQUARED else sum(abs(e) for e in errs)
            else:
                raise ValueError(f"reward opcode {op} is outside the subset")
            c = w * value
            reward += c
            if op in (R_LINEAR, R_YAW, R_CONSTANT, R_GAIT_MATCH, R_SWING_CLEARANCE, R_FOOT_CLEARANCE):
                b0[0] += c
            elif op in (R_SUPPORT_SLIP, R_FORBIDDEN):
                b1[3] += c
            elif op == R_JOINT_VELOCITY:
                b0[2] += c
            elif op == R_JOINT_ACCELERATION:
                b0[3] += c
            elif op == R_ACTION_RATE:
                b1[0] += c
            elif op in (R_LIMIT_SQUARED, R_LIMIT_ABSOLUTE, R_POSTURE_SQUARED, R_POSTURE_ABSOLUTE):
                b1[1] += c
            else:
                b0[1] += c
        steps = st.episode_step + 1
        timeout = steps >= p.maximum_episode_steps
        done, reason, priority, penalty = False, REASON_CONTINUING, 0, 0.0
        for t in self.terminations:
            top = self.bands - 1 if getattr(t, "maximum_band", 0xFFFFFFFF) == 0xFFFFFFFF else t.maximum_band
            if st.band < getattr(t, "minimum_band", 0) or st.band > top:
                continue
            trig = (height < t.threshold if t.opcode == T_MIN_HEIGHT else tilt > t.threshold if t.opcode == T_MAX_TILT
                    else gm[t.group, 0] > t.threshold if t.opcode == T_CONTACT_GROUP else False)
            if trig and (not done or t.priority >= priority):
                done, reason, priority, penalty = True, t.reason, t.priority, t.failure_penalty
        if timeout:
            done, reason = True, REASON_TIMEOUT
        if physics_error:
            done, reason = True, REASON_PHYSICS_ERROR
        if done and reason not in (REASON_TIMEOUT, REASON_PHYSICS_ERROR):
            reward += penalty
            b0[1] += penalty
        reward *= dt
        b0 *= dt
        b1 *= dt
        tracking = math.exp(-tracking_error / 0.25)
        yaw_tracking = math.exp(-yaw_error / 0.25)
        episode_tracking = st.episode_tracking + tracking
        episode_score = episode_tracking / max(steps, 1)
        episode_return = st.episode_return + reward
        if not done and st.command_steps <= 1:
            st.command = self.sample_command(env, st.episode, steps, st.band)
            st.command_steps = self.duration_steps(env, st.episode, steps, 64)
        elif not done:
            st.command_steps -= 1
        st.episode_step = steps
        st.pending_reset = done
        st.last_reason = reason
        st.phase = phase
        st.previous_height = height
        st.episode_return = 0.0 if done else episode_return
        st.episode_tracking = 0.0 if done else episode_tracking
        if not done or (timeout and not physics_error):
            st.frame = np.vstack([st.frame[1:], self.frame(env, q, v, st, raw_last, st.previous_joint[1], st.episode, steps, gm)[None]])
            if st.observation_delay and self.H > 1:
                st.frame[-1] = st.frame[self.H - 1 - min(st.observation_delay, self.H - 1)]
            st.critic = self.critic_frame(q, v, st, raw_last, st.previous_joint[1], gm)
            for a, b in enumerate(p.actions):
                st.previous_joint[0, a] = v[b.v_index]
                st.previous_joint[1, a] = q[b.q_index]
        return {
            "reward": reward, "tracking_score": 0.5 * (tracking + yaw_tracking), "root_height": height, "tilt": tilt,
            "difficulty_band": st.band, "done": int(done), "timeout": int(timeout), "physics_error": int(physics_error), "termination_reason": reason,
            "task_reward": b0[0], "base_reward": b0[1], "joint_velocity_reward": b0[2], "joint_acceleration_reward": b0[3],
            "control_reward": b1[0], "posture_reward": b1[1], "energy_reward": b1[2], "contact_reward": b1[3],
            "episode_tracking_score": episode_score if done and not physics_error else 0.0,
            "contact_metrics": gm,
        }
