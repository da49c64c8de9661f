"""Task programs for the task layer (``World.set_task``).

A ``TaskProgram`` holds the tables of the reference's compiled task program
(include/metalrobo/task_program_types.h: action bindings, actor observation,
reward, termination and randomization operators, joint groups) for the
operator subset the device evaluates; ``task_program_c`` marshals it into the
``MRTaskProgramC`` record of ``mr_task_rollout_set_task``.
``locomotion_task`` composes a velocity-tracking locomotion task over an
articulated world's actuated joints, shaped like the reference's Unitree G1
locomotion tasks (src/core/LocomotionWorld.cpp:1180-1215 actor frame,
:2000-2110 reward and termination operators).

Operator codes are the reference's values (``native.TASK_*``).
"""

from __future__ import annotations

import ctypes as ct
from dataclasses import dataclass, field
from typing import Any, Sequence

import numpy as np

from . import native

# MRTaskObservationOpcode / MRTaskRewardOpcode / MRTaskTerminationOpcode /
# MRTaskTerminationReason / MRTaskRandomizationOpcode (the evaluated subset).
OBSERVE = {
    "root_angular_velocity_local": 0, "projected_gravity": 1, "command": 2, "joint_position_error": 3, "joint_velocity": 4,
    "previous_action": 5, "root_linear_velocity_local": 6, "root_height": 7, "contact_metric": 8, "contact_wrench_local": 13,
    "gait_phase": 14, "support_sense": 18, "delayed_action": 26, "joint_finite_difference_velocity": 27,
}
NORMALIZE_VECTOR3 = 1
REWARD = {
    "linear_velocity_tracking": 0, "yaw_velocity_tracking": 1, "constant": 2, "root_vertical_velocity_squared": 3,
    "root_roll_pitch_velocity_squared": 4, "tilt_squared": 5, "root_height_error_squared": 6, "joint_velocity_squared": 7,
    "joint_acceleration_squared": 8, "action_rate_squared": 9, "joint_limit_violation_squared": 10,
    "joint_group_posture_squared": 12, "gait_contact_match": 13, "swing_clearance": 14, "support_slip": 15, "forbidden_contact": 16,
    "joint_group_posture_absolute": 17, "projected_gravity_horizontal_squared": 18, "foot_clearance": 19,
    "joint_limit_violation_absolute": 20, "root_height_normalized": 21, "root_height_progress": 22, "uprightness": 23,
}
TERMINATE = {"minimum_root_height": 0, "maximum_tilt": 1, "contact_group": 2}
CONTACT_SUPPORT, CONTACT_FORBIDDEN = 1, 2
ALL_GROUPS = 0xFFFFFFFF
REASON = {"continuing": 0, "height": 1, "tilt": 2, "contact": 3, "timeout": 4, "physics_error": 5}
RANDOMIZE = {
    "root_position": 0, "root_yaw": 1, "action_position": 2, "velocity": 3, "action_delay": 7, "observation_delay": 8,
    "action_velocity": 9, "root_height": 10, "joint_position": 12,
}


@dataclass
class ActionBinding:
    dof: int
    q_index: int
    v_index: int
    scale: float
    lower_target: float
    upper_target: float
    response_time_seconds: float = 0.0


@dataclass
class Observation:
    opcode: int
    source: int = 0
    component: int = 0
    flags: int = 0
    scale: float = 1.0
    offset: float = 0.0
    noise_amplitude: float = 0.0
    noise_channel: int = 0


@dataclass
class Reward:
    opcode: int
    weight: float
    parameters: tuple[float, float, float] = (0.0, 0.0, 0.0)
    group: int = 0


@dataclass
class Termination:
    opcode: int
    reason: int
    priority: int
    threshold: float
    failure_penalty: float = 0.0
    group: int = 0
    minimum_band: int = 0
    maximum_band: int = 0xFFFFFFFF  # every band from minimum_band up


@dataclass
class ContactGroup:
    bodies: list[int]
    flags: int
    reference_body: int
    local_reference: tuple[float, float, float, float] = (0.0, 0.0, 0.0, 0.0)
    kinematic_reference: tuple[float, float, float] = (0.0, 0.0, 0.0)
    gait_phase_offset: float = 0.0
    stance_fraction: float = 0.5


@dataclass
class Randomization:
    opcode: int
    parameters: tuple[float, float, float, float] = (0.0, 0.0, 0.0, 0.0)
    target: int = 0
    minimum_band: int = 0  # skipped in episodes of a lower difficulty band


@dataclass
class TaskProgram:
    actions: list[ActionBinding]
    actor: list[Observation]
    default_q: np.ndarray
    critic: list[Observation] = field(default_factory=list)  # the critic's own clean frame (empty: the actor history)
    rewards: list[Reward] = field(default_factory=list)
    terminations: list[Termination] = field(default_factory=list)
    randomization: list[Randomization] = field(default_factory=list)
    joint_groups: list[list[int]] = field(default_factory=list)  # action indices
    contact_groups: list[ContactGroup] = field(default_factory=list)
    support_force_threshold: float = 1.0
    clearance_target: float = 0.08
    maximum_episode_steps: int = 500
    action_history: int = 3
    action_delay_steps: int = 0
    observation_history: int = 1  # actor frames stacked per observation, oldest first
    maximum_observation_delay: int = 0
    base_height_target: float = 0.0
    gait_period_seconds: float = 0.8
    root_reference: tuple[float, float, float] = (0.0, 0.0, 0.0)
    command_lower: tuple[float, float, float] = (0.0, 0.0, 0.0)
    command_upper: tuple[float, float, float] = (0.0, 0.0, 0.0)
    standing_probability: float = 0.0
    command_duration_seconds: tuple[float, float] = (1.0, 1.0)
    difficulty_band_count: int = 1
    band_sampling_exponent: float = 1.0
    command_limit_lower: tuple[float, float, float] | None = None  # None: command_lower
    command_limit_upper: tuple[float, float, float] | None = None  # None: command_upper
    command_band_step: tuple[float, float, float] = (0.0, 0.0, 0.0)
    task_fingerprint: int = 0


def task_program_c(program: TaskProgram) -> tuple[native.TaskProgramC, list[Any]]:
    """(record, keepalive): the record points into the keepalive arrays."""

    keep: list[Any] = []

    def table(cls, rows, fill):
        arr = (cls * max(len(rows), 1))()
        for i, row in enumerate(rows):
            fill(arr[i], row)
        keep.append(arr)
        return ct.cast(arr, ct.POINTER(cls)), len(rows)

    def fill_action(c, b: ActionBinding):
        c.dof_index, c.q_index, c.v_index = b.dof, b.q_index, b.v_index
        c.scale, c.lower_target, c.upper_target, c.response_time_seconds = b.scale, b.lower_target, b.upper_target, b.response_time_seconds

    def fill_obs(c, o: Observation):
        c.opcode, c.source, c.component, c.flags = o.opcode, o.source, o.component, o.flags
        c.transform_scale, c.transform_offset, c.noise_amplitude, c.noise_channel = o.scale, o.offset, o.noise_amplitude, o.noise_channel

    def fill_reward(c, r: Reward):
        c.opcode, c.group, c.weight = r.opcode, r.group, r.weight
        c.parameters[:] = list(r.parameters)

    def fill_term(c, t: Termination):
        c.opcode, c.reason, c.priority, c.threshold, c.failure_penalty = t.opcode, t.reason, t.priority, t.threshold, t.failure_penalty
        c.group, c.minimum_band, c.maximum_band = t.group, t.minimum_band, t.maximum_band

    def fill_random(c, r: Randomization):
        c.opcode, c.target, c.minimum_band = r.opcode, r.target, r.minimum_band
        c.parameters[:] = list(r.parameters)

    p = native.TaskProgramC()
    p.actions, p.action_count = table(native.TaskActionBindingC, program.actions, fill_action)
    p.actor, p.actor_count = table(native.TaskObservationOperatorC, program.actor, fill_obs)
    p.critic, p.critic_count = table(native.TaskObservationOperatorC, program.critic, fill_obs)
    p.rewards, p.reward_count = table(native.TaskRewardOperatorC, program.rewards, fill_reward)
    p.terminations, p.termination_count = table(native.TaskTerminationOperatorC, program.terminations, fill_term)
    p.randomization, p.randomization_count = table(native.TaskRandomizationOperatorC, program.randomization, fill_random)
    members: list[int] = []
    groups = []
    for g in program.joint_groups:
        groups.append((len(members), len(g)))
        members.extend(int(a) for a in g)

    def fill_group(c, g):
        c.first, c.count = g

    p.joint_groups, p.joint_group_count = table(native.TaskIndexGroupC, groups, fill_group)
    m = np.ascontiguousarray(members if members else [0], np.uint32)
    keep.append(m)
    p.joint_members, p.joint_member_count = m.ctypes.data_as(ct.POINTER(ct.c_uint32)), len(members)
    bodies: list[int] = []
    cgroups = []
    for g in program.contact_groups:
        cgroups.append((len(bodies), g))
        bodies.extend(int(b) for b in g.bodies)

    def fill_cgroup(c, item):
        first, g = item
        c.first, c.count, c.flags, c.reference_body = first, len(g.bodies), g.flags, g.reference_body
        c.local_reference[:] = list(g.local_reference)
        c.kinematic_reference[:] = list(g.kinematic_reference) + [0.0]
        c.gait_phase_offset, c.stance_fraction = g.gait_phase_offset, g.stance_fraction

    p.contact_groups, p.contact_group_count = table(native.TaskContactGroupC, cgroups, fill_cgroup)
    cm = np.ascontiguousarray(bodies if bodies else [0], np.uint32)
    keep.append(cm)
    p.contact_members, p.contact_member_count = cm.ctypes.data_as(ct.POINTER(ct.c_uint32)), len(bodies)
    p.support_force_threshold = program.support_force_threshold
    p.clearance_target = program.clearance_target
    dq = np.ascontiguousarray(program.default_q, np.float32)
    keep.append(dq)
    p.default_q, p.default_q_count = dq.ctypes.data_as(ct.POINTER(ct.c_float)), dq.size
    p.maximum_episode_steps = program.maximum_episode_steps
    p.action_history = program.action_history
    p.action_delay_steps = program.action_delay_steps
    p.observation_history = program.observation_history
    p.maximum_observation_delay = program.maximum_observation_delay
    p.base_height_target = program.base_height_target
    p.gait_period_seconds = program.gait_period_seconds
    p.root_reference[:] = list(program.root_reference)
    p.command_lower[:] = list(program.command_lower)
    p.command_upper[:] = list(program.command_upper)
    p.standing_probability = program.standing_probability
    p.command_duration_seconds[:] = list(program.command_duration_seconds)
    p.difficulty_band_count = program.difficulty_band_count
    p.band_sampling_exponent = program.band_sampling_exponent
    p.command_limit_lower[:] = list(program.command_limit_lower or program.command_lower)
    p.command_limit_upper[:] = list(program.command_limit_upper or program.command_upper)
    p.command_band_step[:] = list(program.command_band_step)
    p.task_fingerprint = program.task_fingerprint
    return p, keep


def action_bindings(records, *, scale: float = 0.25, response_time_seconds: float = 0.0) -> list[ActionBinding]:
    """One joint-position binding per world action (the actuated DoFs in
    order), targets clamped to the DoF's position limits."""

    w = records.world
    out = []
    for d in range(int(w.nv)):
        dof = records.dofs[d]
        if not int(dof.flags) & int(native.MR_DOF_FLAG_ACTUATED):
            continue
        lo, hi = float(dof.limits[0]), float(dof.limits[1])
        if not (np.isfinite(lo) and np.isfinite(hi)):
            lo, hi = -1.0e6, 1.0e6
        out.append(ActionBinding(d, int(dof.q_index), d, scale, lo, hi, response_time_seconds))
    if len(out) != int(w.action_count):
        raise ValueError("actuated DoFs do not match the world's action count")
    return out


def foot_contact_groups(records, *, forbidden_bodies: Sequence[int] = (0,), stance_fraction: float = 0.6) -> list[ContactGroup]:
    """Support groups for the bodies that carry box collision shapes (the
    feet of the synthetic humanoid tree), each referenced at its box's sole
    centre, alternating gait phase; then one forbidden group over
    `forbidden_bodies` (the torso by default), referenced at the first."""

    groups = []
    for i in range(int(records.world.shape_count)):
        sh = records.shapes[i]
        if int(sh.shape_type) != 2 or int(sh.body) >= int(records.world.body_count) - 1:
            continue
        body = int(sh.body)
        sole = (float(sh.local_position[0]), float(sh.local_position[1]), float(sh.local_position[2]) - float(sh.dimensions[2]), 0.0)
        groups.append(ContactGroup([body], CONTACT_SUPPORT, body, sole, (0.0, 0.0, 0.0), np.pi * (len(groups) % 2), stance_fraction))
    if forbidden_bodies:
        groups.append(ContactGroup(list(forbidden_bodies), CONTACT_FORBIDDEN, int(forbidden_bodies[0])))
    return groups


def locomotion_task(records, default_q: np.ndarray, *, base_height: float | None = None, maximum_episode_steps: int = 500,
                    action_scale: float = 0.25, response_time_seconds: float = 0.0, action_history: int = 3,
                    action_delay_steps: int = 0, noise: float = 0.0, min_height_fraction: float = 0.6,
                    max_tilt: float = 1.22173048, groups: Sequence[Sequence[int]] | None = None,
                    contact_groups: Sequence[ContactGroup] | None = None, support_force_threshold: float = 1.0,
                    clearance_target: float = 0.08, observation_history: int = 1) -> TaskProgram:
    """Velocity-tracking locomotion over every actuated joint of an
    articulated world with a floating root.  Actor frame (per the reference's
    G1 legs frame): raw action one step back, command xyz + extension lane,
    joint position errors, finite-difference joint velocities, normalised
    projected gravity, gait phase sin/cos, root angular velocity in the root
    frame; with `contact_groups`, each support group's normal force and air
    time, and the gait-contact, foot-clearance, swing-clearance, support-slip
    and forbidden-contact rewards of the reference's G1 tasks, and a
    forbidden group's contact ending the episode."""

    actions = action_bindings(records, scale=action_scale, response_time_seconds=response_time_seconds)
    na = len(actions)
    dq = np.asarray(default_q, np.float32)
    height = float(dq[2]) if base_height is None else float(base_height)
    ch = iter(range(1000, 100000))

    def obs(opcode, source=0, component=0, **kw):
        return Observation(OBSERVE[opcode], source, component, noise_channel=next(ch), noise_amplitude=kw.pop("noise", noise), **kw)

    actor = [obs("delayed_action", a, 1, noise=0.0) for a in range(na)]
    actor += [obs("command", 0, c, noise=0.0) for c in range(4)]
    actor += [obs("joint_position_error", a) for a in range(na)]
    actor += [obs("joint_finite_difference_velocity", a, scale=0.05) for a in range(na)]
    actor += [obs("projected_gravity", 0, c, flags=NORMALIZE_VECTOR3) for c in range(3)]
    actor += [obs("gait_phase", 0, c, noise=0.0) for c in range(2)]
    actor += [obs("root_angular_velocity_local", 0, c, scale=0.25) for c in range(3)]
    if groups is None:
        half = na // 2
        groups = [list(range(0, half)), list(range(half, na))]
    rewards = [
        Reward(REWARD["linear_velocity_tracking"], 1.0, (0.25, 0.0, 0.0)),
        Reward(REWARD["yaw_velocity_tracking"], 0.5, (0.25, 0.0, 0.0)),
        Reward(REWARD["constant"], 0.15),
        Reward(REWARD["root_vertical_velocity_squared"], -2.0),
        Reward(REWARD["root_roll_pitch_velocity_squared"], -0.05),
        Reward(REWARD["projected_gravity_horizontal_squared"], -5.0),
        Reward(REWARD["root_height_error_squared"], -10.0),
        Reward(REWARD["joint_velocity_squared"], -0.001),
        Reward(REWARD["joint_acceleration_squared"], -2.5e-7),
        Reward(REWARD["action_rate_squared"], -0.05),
        Reward(REWARD["joint_limit_violation_absolute"], -5.0, (0.9, 0.0, 0.0)),
        Reward(REWARD["joint_group_posture_absolute"], -1.0, group=0),
        Reward(REWARD["joint_group_posture_squared"], -0.1, group=1),
        Reward(REWARD["uprightness"], 0.2),
        Reward(REWARD["root_height_progress"], 0.05),
    ]
    terminations = [
        Termination(TERMINATE["minimum_root_height"], REASON["height"], 1, min_height_fraction * height, -2.0),
        Termination(TERMINATE["maximum_tilt"], REASON["tilt"], 2, max_tilt, -2.0),
    ]
    cgroups = list(contact_groups or [])
    for g, cg in enumerate(cgroups):
        if cg.flags & CONTACT_SUPPORT:
            actor.append(obs("contact_metric", g, 0, scale=0.002))
            actor.append(obs("contact_metric", g, 2, noise=0.0))
    if cgroups:
        actor += [obs("support_sense", 0, c, scale=0.002 if c == 0 else 1.0, noise=0.0) for c in range(3)]
    if cgroups:
        rewards += [
            Reward(REWARD["gait_contact_match"], 0.5, group=ALL_GROUPS),
            Reward(REWARD["foot_clearance"], 1.0, (0.05, 2.0, 0.0), group=ALL_GROUPS),
            Reward(REWARD["swing_clearance"], 0.25, (0.01, 0.0, 0.0), group=ALL_GROUPS),
            Reward(REWARD["support_slip"], -0.2, group=ALL_GROUPS),
            Reward(REWARD["forbidden_contact"], -1.0, group=ALL_GROUPS),
        ]
        for g, cg in enumerate(cgroups):
            if cg.flags & CONTACT_FORBIDDEN:
                terminations.append(Termination(TERMINATE["contact_group"], REASON["contact"], 3, 0.5, -2.0, group=g))
    randomization = [
        Randomization(RANDOMIZE["root_yaw"], (-np.pi, np.pi, 0.0, 0.0)),
        Randomization(RANDOMIZE["action_position"], (-0.1, 0.1, 0.0, 0.0)),
        Randomization(RANDOMIZE["action_velocity"], (-0.2, 0.2, 0.0, 0.0)),
    ]
    return TaskProgram(actions=actions, actor=actor, default_q=dq, rewards=rewards, terminations=terminations,
                       randomization=randomization, joint_groups=[list(g) for g in groups], contact_groups=cgroups,
                       support_force_threshold=support_force_threshold, clearance_target=clearance_target,
                       maximum_episode_steps=maximum_episode_steps, action_history=action_history,
                       action_delay_steps=action_delay_steps, observation_history=observation_history,
                       base_height_target=height, gait_period_seconds=0.8,
                       command_lower=(-0.5, -0.3, -0.5), command_upper=(1.0, 0.3, 0.5), standing_probability=0.1,
                       command_duration_seconds=(2.0, 5.0), task_fingerprint=0x7A5C0001)
