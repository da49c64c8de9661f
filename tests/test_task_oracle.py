"""The task layer's oracle (oracle/task.py) against closed forms: its draw
hash against SplitMix64's published outputs, observations of known poses,
rewards, terminations and their priorities, the action delay line and
first-order response, the command schedule and the reset draws.  No device
work."""

from __future__ import annotations

import math

import numpy as np
import pytest

import numi_lab_b200 as nb
from numi_lab_b200 import task as T
from oracle.task import TaskOracle, mix64, unit_draw

DT = 0.02


def _splitmix64(state: int, n: int) -> list[int]:
    out, M = [], (1 << 64) - 1
    for _ in range(n):
        state = (state + 0x9E3779B97F4A7C15) & M
        z = state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M
        out.append(z ^ (z >> 31))
    return out


def test_draw_hash_is_splitmix64():
    # SplitMix64 from state 0: its first output is the published 0xE220A8397B1DCDAF.
    assert mix64(0) == 0xE220A8397B1DCDAF
    seq = _splitmix64(12345, 4)
    state = 12345
    for k in range(4):
        assert mix64((state + k * 0x9E3779B97F4A7C15) & ((1 << 64) - 1)) == seq[k]
    draws = np.array([unit_draw(7, e, 1, s, c) for e in range(8) for s in range(8) for c in range(16)])
    assert np.all((draws >= 0.0) & (draws < 1.0))
    assert abs(draws.mean() - 0.5) < 0.03
    assert len(np.unique(draws)) == draws.size  # every coordinate its own draw
    assert np.all(draws * 16777216.0 == np.floor(draws * 16777216.0))  # 24-bit grid


@pytest.fixture(scope="module")
def tree():
    rec = nb.compile_model("tree29", 0)
    dq = np.zeros(int(rec.world.nq))
    dq[2], dq[6] = 0.9, 1.0
    prog = T.locomotion_task(rec, dq, noise=0.0)
    lo = [float(rec.dofs[b.dof].limits[0]) for b in prog.actions]
    hi = [float(rec.dofs[b.dof].limits[1]) for b in prog.actions]
    return rec, prog, lo, hi


def _oracle(prog, rec, lo, hi, **kw):
    return TaskOracle(prog, nq=int(rec.world.nq), nv=int(rec.world.nv), dt=DT, seed=kw.pop("seed", 3), fixed_root=False,
                      limit_lower=lo, limit_upper=hi, **kw)


def _quat_axis(axis, angle):
    a = np.asarray(axis, float) / np.linalg.norm(axis)
    return np.concatenate([a * math.sin(angle / 2), [math.cos(angle / 2)]])


def test_observations_of_known_poses(tree):
    rec, prog, lo, hi = tree
    o = _oracle(prog, rec, lo, hi)
    st = o.new_state()
    st.command = np.array([0.5, 0.0, 0.2])
    st.phase = 1.0
    q = prog.default_q.astype(float).copy()
    v = np.zeros(int(rec.world.nv))
    ops = {(op.opcode, op.component): op for op in prog.actor}

    def val(opcode, component=0, source=0):
        op = T.Observation(opcode, source, component)
        return o.clean(op, q, v, st, o.L - 2, st.previous_joint[1])

    assert [val(1, c) for c in range(3)] == pytest.approx([0.0, 0.0, -1.0])
    q[3:7] = _quat_axis([1, 0, 0], math.pi / 2)  # rolled 90 degrees: gravity along -y in the body frame
    assert [val(1, c) for c in range(3)] == pytest.approx([0.0, -1.0, 0.0], abs=1e-12)
    q[3:7] = _quat_axis([0, 0, 1], math.pi / 2)  # yawed 90 degrees
    v[0:3] = [1.0, 0.0, 0.0]  # world +x is body -y
    v[3:6] = [0.0, 0.0, 0.7]
    assert [val(6, c) for c in range(3)] == pytest.approx([0.0, -1.0, 0.0], abs=1e-12)
    assert [val(0, c) for c in range(3)] == pytest.approx([0.0, 0.0, 0.7], abs=1e-12)
    assert val(7) == pytest.approx(0.9)
    assert [val(2, c) for c in range(4)] == [0.5, 0.0, 0.2, 0.0]
    assert [val(14, c) for c in range(2)] == pytest.approx([math.sin(1.0), math.cos(1.0)])
    st.command = np.array([0.05, 0.0, 0.0])  # below 0.1: the phase is gated off
    assert [val(14, c) for c in range(2)] == [0.0, 0.0]
    b = prog.actions[3]
    q[b.q_index] = prog.default_q[b.q_index] + 0.25
    st.previous_joint[1, 3] = q[b.q_index] - 0.01
    v[b.v_index] = 2.0
    assert val(3, source=3) == pytest.approx(0.25)
    assert val(27, source=3) == pytest.approx(0.01 / DT)
    assert val(4, source=3) == 2.0
    st.history[:, 5] = [0.1, 0.2, 0.3]
    assert val(5, source=5) == 0.2 and val(26, 1, source=5) == 0.1  # newest raw slot and one back
    assert ops[(3, 0)].scale == 1.0


def test_rewards_and_terminations_of_known_states(tree):
    rec, prog, lo, hi = tree
    o = _oracle(prog, rec, lo, hi)
    st = o.new_state()
    q = prog.default_q.astype(float).copy()
    st.initialized, st.command, st.command_steps = True, np.zeros(3), 50
    st.previous_height = q[2]
    v = np.zeros(int(rec.world.nv))
    t = o.complete(0, st, q, v, 0)
    # Upright at the target height, still, zero command: tracking terms 1,
    # the constant, uprightness 1; every penalty 0.
    weights = {r.opcode: r.weight for r in prog.rewards}
    expect = DT * (weights[0] + weights[1] + weights[2] + weights[23])
    assert t["reward"] == pytest.approx(expect, rel=1e-12)
    assert t["task_reward"] == pytest.approx(DT * (weights[0] + weights[1] + weights[2]), rel=1e-12)
    assert t["done"] == 0 and t["termination_reason"] == 0 and t["tracking_score"] == pytest.approx(1.0)
    # Below the height threshold: done, reason height, penalty -2.
    st2 = o.new_state()
    st2.initialized, st2.command_steps, st2.previous_height = True, 50, 0.9
    q2 = q.copy()
    q2[2] = 0.3
    t2 = o.complete(0, st2, q2, v, 0)
    assert t2["done"] == 1 and t2["termination_reason"] == 1 and st2.pending_reset
    # Tilted past 1.22 rad and low: both trigger, tilt (priority 2) wins.
    st3 = o.new_state()
    st3.initialized, st3.command_steps = True, 50
    q3 = q2.copy()
    q3[3:7] = _quat_axis([0, 1, 0], 1.4)
    t3 = o.complete(0, st3, q3, v, 0)
    assert t3["termination_reason"] == 2 and t3["tilt"] == pytest.approx(1.4, abs=1e-9)
    # A physics error overrides every reason and pays no penalty.
    st4 = o.new_state()
    st4.initialized, st4.command_steps = True, 50
    t4 = o.complete(0, st4, q3, v, 3)
    assert t4["termination_reason"] == 5 and t4["physics_error"] == 1
    assert t4["reward"] == pytest.approx(t3["reward"] - DT * (-2.0), rel=1e-9)
    # Timeout on the last episode step, with the episode's mean tracking score.
    st5 = o.new_state()
    st5.initialized, st5.command_steps, st5.episode_step = True, 50, prog.maximum_episode_steps - 1
    st5.episode_tracking = 3.0
    t5 = o.complete(0, st5, q, v, 0)
    assert t5["timeout"] == 1 and t5["termination_reason"] == 4
    assert t5["episode_tracking_score"] == pytest.approx((3.0 + 1.0) / prog.maximum_episode_steps)


def test_delay_line_and_first_order_response(tree):
    rec, prog0, lo, hi = tree
    dq = prog0.default_q
    tau = 0.05
    prog = T.locomotion_task(rec, dq, response_time_seconds=tau, action_history=5, action_delay_steps=2)
    o = _oracle(prog, rec, lo, hi)
    st = o.new_state()
    st.action_delay = o.delay  # a reset sets it (no ACTION_DELAY operator here)
    alpha = 1.0 - math.exp(-DT / tau)
    seq = [0.4, -0.2, 0.9, 0.1, 0.0]
    filt = 0.0
    for k, a in enumerate(seq):
        targets = o.apply(st, np.full(o.na, a))
        delayed = seq[k - 2] if k >= 2 else 0.0
        filt = filt + (delayed - filt) * alpha
        b = prog.actions[0]
        assert st.history[-1, 0] == pytest.approx(filt)
        assert targets[0] == pytest.approx(min(max(dq[b.q_index] + b.scale * filt, b.lower_target), b.upper_target))
        assert st.history[o.L - 2, 0] == a  # the newest raw action


def test_command_schedule_and_reset_draws(tree):
    rec, prog, lo, hi = tree
    o = _oracle(prog, rec, lo, hi, seed=11)
    q = prog.default_q.astype(float).copy()
    v = np.zeros(int(rec.world.nv))
    lo_s, hi_s = prog.command_duration_seconds
    for env in range(6):
        st = o.new_state()
        reset, rq, rv, obs = o.observe(env, st, q, v, False)
        assert reset and st.episode == 1 and st.episode_step == 0
        assert math.floor(lo_s / DT) <= st.command_steps <= math.floor(hi_s / DT)
        assert np.all(st.command == 0.0) or all(prog.command_lower[k] <= st.command[k] <= prog.command_upper[k] for k in range(3))
        # Yaw about +z only: the reset root stays upright.
        assert rq[3] == pytest.approx(0.0) and rq[4] == pytest.approx(0.0) and np.linalg.norm(rq[3:7]) == pytest.approx(1.0)
        for b in prog.actions:
            assert abs(rq[b.q_index] - prog.default_q[b.q_index]) <= 0.1 + 1e-12
            assert abs(rv[b.v_index]) <= 0.2 + 1e-12
        assert np.allclose(st.previous_joint[1], [rq[b.q_index] for b in prog.actions])
        # The first command lasts command_steps control steps.
        first, n = st.command.copy(), st.command_steps
        for k in range(n - 1):
            o.complete(env, st, rq, rv, 0)
            assert np.array_equal(st.command, first), k
        o.complete(env, st, rq, rv, 0)
        assert st.episode_step == n
        # Same environment, same episode: the same draws.
        st_again = o.new_state()
        _, rq2, _, obs2 = o.observe(env, st_again, q, v, False)
        assert np.array_equal(rq, rq2) and np.array_equal(obs, obs2)


def test_contact_group_metrics_of_a_hand_made_foot_contact(tree):
    """A foot pressed flat on the ground by four equal normal impulses at its
    sole corners: force = 4 lambda / h, the centre of pressure at the corners'
    centre in the foot frame, the wrench's force straight up in that frame,
    no slip for a still foot, clearance from the sole point."""

    from oracle import Oracle
    from numi_lab_b200 import native

    rec, prog0, lo, hi = tree
    groups = T.foot_contact_groups(rec)
    prog = T.locomotion_task(rec, prog0.default_q, contact_groups=groups, support_force_threshold=1.0)
    h = DT / 4
    world = Oracle(rec, h, 4, 8, 0)
    o = TaskOracle(prog, nq=int(rec.world.nq), nv=int(rec.world.nv), dt=DT, seed=1, fixed_root=False, limit_lower=lo,
                   limit_upper=hi, records=rec, world=world, physics_dt=h)
    st = o.new_state()
    q = prog.default_q.astype(float).copy()
    v = np.zeros(int(rec.world.nv))
    bs = world.body_states(q, v)
    foot = groups[0].reference_body
    pair = next(i for i in range(int(rec.world.pair_count)) if int(rec.shapes[int(rec.pairs[i].shape_a)].body) == foot)
    mans = (native.ManifoldC * int(rec.world.pair_count))()
    m = mans[pair]
    rot = bs[foot, 3:7]
    m.normal_local[:] = list(rotate_inverse_np(rot, np.array([0.0, 0.0, -1.0])))
    m.tangent_local[:] = list(rotate_inverse_np(rot, np.array([1.0, 0.0, 0.0])))
    m.count = 4
    sole = np.array(groups[0].local_reference[:3])
    corners = [sole + np.array([sx * 0.05, sy * 0.02, 0.0]) + np.array([0.01, 0.0, 0.0]) for sx in (-1, 1) for sy in (-1, 1)]
    lam = 0.3
    for i, c in enumerate(corners):
        m.points[i].anchor_a[:] = list(c)
        m.points[i].anchor_b[:] = list(bs[foot, :3] + rotate_np(rot, c))
        m.points[i].impulses[:] = [lam, 0.0, 0.0]
    gm = o.contact_metrics(st, q, v, mans)
    assert gm[0, 0] == pytest.approx(4 * lam / h)
    assert gm[0, 1] == 0.0 and gm[0, 2] == 0.0  # still foot, in contact
    # (anchors are stored as FP32)
    assert gm[0, 4] == pytest.approx(0.01, abs=1e-7) and gm[0, 5] == pytest.approx(0.0, abs=1e-7)
    np.testing.assert_allclose(gm[0, 6:9], rotate_inverse_np(rot, np.array([0.0, 0.0, 4 * lam / h])), rtol=1e-6, atol=1e-5)
    sole_world = bs[foot, :3] + rotate_np(rot, sole)
    assert gm[0, 3] == pytest.approx(sole_world[2] - o.ground)
    # The other foot is in the air: its air time grows by the control step.
    assert gm[1, 0] == 0.0 and gm[1, 2] == pytest.approx(DT)
    gm2 = o.contact_metrics(st, q, v, (native.ManifoldC * int(rec.world.pair_count))())
    assert gm2[0, 2] == pytest.approx(DT) and gm2[1, 2] == pytest.approx(2 * DT)
    assert gm[2, 0] == 0.0  # the forbidden group (torso) does not touch


def rotate_np(qv, v):
    from oracle.task import rotate

    return rotate(np.asarray(qv, float), np.asarray(v, float))


def rotate_inverse_np(qv, v):
    from oracle.task import rotate_inverse

    return rotate_inverse(np.asarray(qv, float), np.asarray(v, float))


def test_difficulty_bands_widen_commands_and_filter_operators(tree):
    """sampledDifficultyBand and sampledCommand: bands stay in the sampled
    range, the exponent skews them towards the low end, each band widens
    the command range by its step within the limits, and band-filtered
    randomization and termination operators apply only inside their bands."""

    import dataclasses

    rec, prog, lo, hi = tree
    prog = dataclasses.replace(prog, difficulty_band_count=6, band_sampling_exponent=3.0, command_band_step=(0.25, 0.1, 0.0),
                               command_limit_lower=(-1.0, -0.4, -0.5), command_limit_upper=(1.5, 0.4, 0.5), standing_probability=0.0,
                               randomization=[T.Randomization(T.RANDOMIZE["root_height"], (0.9, 0.95, 0.0, 0.0), minimum_band=3)],
                               terminations=[T.Termination(T.TERMINATE["minimum_root_height"], T.REASON["height"], 1, 1e9,
                                                           minimum_band=1, maximum_band=2)])
    q = prog.default_q.astype(float).copy()
    v = np.zeros(int(rec.world.nv))
    for band_range, allowed in ((None, range(6)), ((2, 4), range(2, 5)), ((4, 0xFFFFFFFF), range(4, 6)), ((9, 9), [5])):
        o = TaskOracle(prog, nq=int(rec.world.nq), nv=int(rec.world.nv), dt=DT, seed=3, fixed_root=False, limit_lower=lo,
                       limit_upper=hi, band_range=band_range)
        counts = np.zeros(6, int)
        for env in range(400):
            st = o.new_state()
            _, rq, rv, _ = o.observe(env, st, q, v, False)
            assert st.band in allowed, (band_range, st.band)
            counts[st.band] += 1
            b = st.band
            for k in range(3):
                lower = max(prog.command_lower[k] - b * prog.command_band_step[k], prog.command_limit_lower[k])
                upper = min(prog.command_upper[k] + b * prog.command_band_step[k], prog.command_limit_upper[k])
                assert lower - 1e-12 <= st.command[k] <= upper + 1e-12
            # The root height draw applies from band 3 on.
            assert (0.9 <= rq[2] <= 0.95) if b >= 3 else rq[2] == q[2]
            # The always-true height termination fires only in bands 1-2.
            t = o.complete(env, st, rq, rv, 0)
            assert t["difficulty_band"] == b
            assert (t["termination_reason"] == T.REASON["height"]) == (1 <= b <= 2)
        if band_range is None:
            # u^3 puts 1/6^(1/3) = 55 % of the episodes in band 0.
            assert counts[0] > 180 and counts[5] < counts[0] / 3
