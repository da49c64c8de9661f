// The task layer's three kernels around each control step, one warp per
// environment for observe and complete, one thread per (environment,
// action) for apply.  They restate, for the operator subset of
// include/numi_b200.h, src/metal/LocomotionTask.metal:
//   observe   :2184-3440  reset draw (:2330-3120), actor frame (:1190-1330)
//   apply     :3442-3674  delay line, first-order response, target clamp
//   complete  :3904-6745  reward operators (:4700-6060), terminations
//                         (:6064-6160), command schedule (:6388-6420),
//                         next actor frame and joint history (:6478-6630)
// All arithmetic is FP32 like the reference's shaders; draws use the
// reference's keyed SplitMix64 counter hash (randomUnit, :121-152).
#include "task.h"

#include <cmath>

namespace numi {
namespace {

constexpr float kTwoPi = 6.28318530717958647692f;
constexpr int kTaskWarps = 4;  // environments per CTA
constexpr int kApplyThreads = 256;

// SplitMix64's finaliser over a key built from the draw's coordinates.
__device__ __forceinline__ unsigned long long mix64(unsigned long long x) {
    x += 0x9e3779b97f4a7c15ull;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}

__device__ __forceinline__ float unit_draw(unsigned long long seed, unsigned env, unsigned episode, unsigned step, unsigned channel) {
    unsigned long long key = seed;
    key ^= static_cast<unsigned long long>(env + 1u) * 0xd2b74407b1ce6e93ull;
    key ^= static_cast<unsigned long long>(episode + 1u) * 0xca5a826395121157ull;
    key ^= static_cast<unsigned long long>(step + 1u) * 0x9e3779b185ebca87ull;
    key ^= static_cast<unsigned long long>(channel + 1u) * 0x94d049bb133111ebull;
    return static_cast<float>(static_cast<unsigned>(mix64(key) >> 40)) * (1.0f / 16777216.0f);
}

__device__ __forceinline__ float signed_draw(unsigned long long seed, unsigned env, unsigned episode, unsigned step, unsigned channel) {
    return 2.0f * unit_draw(seed, env, episode, step, channel) - 1.0f;
}

__device__ __forceinline__ float range_draw(unsigned long long seed, unsigned env, unsigned episode, unsigned step, unsigned channel,
                                            float lower, float upper) {
    return lower + (upper - lower) * unit_draw(seed, env, episode, step, channel);
}

__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator*(float s, float3 a) { return make_float3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float lane3(float3 a, unsigned i) { return i == 0u ? a.x : (i == 1u ? a.y : a.z); }

__device__ __forceinline__ float3 rotate(float4 q, float3 v) {
    const float3 u = make_float3(q.x, q.y, q.z);
    const float3 t = 2.0f * cross3(u, v);
    return v + q.w * t + cross3(u, t);
}

__device__ __forceinline__ float3 rotate_inverse(float4 q, float3 v) {
    const float3 u = make_float3(q.x, q.y, q.z);
    const float3 t = 2.0f * cross3(u, v);
    return v - q.w * t + cross3(u, t);
}

__device__ __forceinline__ float4 quat_product(float4 a, float4 b) {
    return make_float4(a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y, a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x,
                       a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w, a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z);
}

__device__ __forceinline__ float3 normalized_or(float3 v, float3 fallback) {
    const float l2 = dot3(v, v);
    return l2 > 1.0e-12f && isfinite(l2) ? rsqrtf(l2) * v : fallback;
}

__device__ __forceinline__ float mixf(float x, float y, float a) { return x + (y - x) * a; }

__device__ __forceinline__ float warp_sum(float x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}

// Root link frame of the selected articulation (LocomotionTask.metal:396-478).
struct Root {
    float4 orientation;
    float3 position;
    float3 linear;   // world linear velocity of the link origin
    float3 angular;  // world angular velocity
};

__device__ __forceinline__ Root root_frame(const TaskProgramDevice& P, const float* q, const float* v) {
    Root r;
    if (P.fixed_root) {
        r.orientation = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
        r.position = r.linear = r.angular = make_float3(0.0f, 0.0f, 0.0f);
        return r;
    }
    r.orientation = make_float4(q[3], q[4], q[5], q[6]);
    const float3 offset = rotate(r.orientation, make_float3(P.root_reference[0], P.root_reference[1], P.root_reference[2]));
    r.position = make_float3(q[0], q[1], q[2]) + offset;
    r.angular = make_float3(v[3], v[4], v[5]);
    r.linear = make_float3(v[0], v[1], v[2]) + cross3(r.angular, offset);
    return r;
}

__device__ __forceinline__ float3 projected_gravity(const Root& r) {
    const float3 down = make_float3(0.0f, 0.0f, -1.0f);
    return normalized_or(rotate_inverse(r.orientation, down), down);
}

// One operator's clean value (cleanObservation, :594-1188, the subset):
// transform applied, no noise.  `raw` points at the delay line's newest raw
// slot; `previous_q` at the joint positions of the last step's end.
__device__ float clean_observation(const TaskProgramDevice& P, const MRTaskObservationOperatorC& op, const Root& r, const float* q,
                                   const float* v, const TaskEnvState& st, const float* raw, const float* previous_q,
                                   const float* metrics) {
    float value = 0.0f;
    const unsigned c = op.component;
    switch (op.opcode) {
    case MR_TASK_OBSERVE_ROOT_ANGULAR_VELOCITY_LOCAL:
        value = lane3(rotate_inverse(r.orientation, r.angular), c);
        break;
    case MR_TASK_OBSERVE_PROJECTED_GRAVITY:
        value = lane3(projected_gravity(r), c);
        break;
    case MR_TASK_OBSERVE_COMMAND:
        value = c < 3u ? st.command[c] : 0.0f;  // the command extension lanes stay zero
        break;
    case MR_TASK_OBSERVE_JOINT_POSITION_ERROR: {
        const int qi = static_cast<int>(P.actions[op.source].q_index);
        value = q[qi] - P.default_q[qi];
        break;
    }
    case MR_TASK_OBSERVE_JOINT_VELOCITY:
        value = v[P.actions[op.source].v_index];
        break;
    case MR_TASK_OBSERVE_JOINT_FINITE_DIFFERENCE_VELOCITY:
        value = (q[P.actions[op.source].q_index] - previous_q[op.source]) / P.dt;
        break;
    case MR_TASK_OBSERVE_PREVIOUS_ACTION:
        value = raw[op.source];
        break;
    case MR_TASK_OBSERVE_DELAYED_ACTION:
        value = raw[static_cast<int>(op.source) - static_cast<int>(op.component) * P.na];
        break;
    case MR_TASK_OBSERVE_ROOT_LINEAR_VELOCITY_LOCAL:
        value = lane3(rotate_inverse(r.orientation, r.linear), c);
        break;
    case MR_TASK_OBSERVE_ROOT_HEIGHT:
        value = r.position.z;
        break;
    case MR_TASK_OBSERVE_CONTACT_METRIC:  // the group's compact metrics (zero on a reset frame)
        value = metrics ? metrics[op.source * kTaskGroupMetrics + c] : 0.0f;
        break;
    case MR_TASK_OBSERVE_CONTACT_WRENCH_LOCAL:
        value = metrics ? metrics[op.source * kTaskGroupMetrics + 6 + c] : 0.0f;
        break;
    case MR_TASK_OBSERVE_SUPPORT_SENSE: {  // total support load, phase-signed balance, largest slip (:1082-1116)
        float total = 0.0f, signed_load = 0.0f, slip = 0.0f;
        for (int g = 0; metrics && g < P.ncontact_groups; ++g) {
            const MRTaskContactGroupC G = P.contact_groups[g];
            if ((G.flags & MR_TASK_CONTACT_SUPPORT) == 0u) continue;
            const float load = fmaxf(metrics[g * kTaskGroupMetrics], 0.0f);
            total += load;
            signed_load += load * cosf(G.gait_phase_offset);
            slip = fmaxf(slip, fmaxf(metrics[g * kTaskGroupMetrics + 1], 0.0f));
        }
        value = c == 0u ? total : (c == 1u ? (total > 1.0e-6f ? signed_load / total : 0.0f) : slip);
        break;
    }
    case MR_TASK_OBSERVE_GAIT_PHASE: {
        const float magnitude = sqrtf(st.command[0] * st.command[0] + st.command[1] * st.command[1] + st.command[2] * st.command[2]);
        if (magnitude >= 0.1f) value = c == 0u ? sinf(st.phase) : cosf(st.phase);
        break;
    }
    default:
        break;
    }
    return op.transform_scale * value + op.transform_offset;
}

// The actor frame (writeFrame, :1190-1330): lanes over operators.  The
// gravity operators flagged NORMALIZE_VECTOR3 publish the unit vector of
// their noisy components.
__device__ void write_frame(const TaskProgramDevice& P, const float* q, const float* v, const TaskEnvState& st, const float* raw,
                            const float* previous_q, const float* metrics, unsigned env, unsigned episode, unsigned step, float* frame,
                            int lane) {
    const Root r = root_frame(P, q, v);
    float3 g = make_float3(0.0f, 0.0f, -1.0f);
    bool have = false;
    for (int i = 0; i < P.nobs; ++i) {
        const MRTaskObservationOperatorC op = P.actor[i];
        if (op.opcode != MR_TASK_OBSERVE_PROJECTED_GRAVITY || (op.flags & MR_TASK_OBSERVATION_NORMALIZE_VECTOR3) == 0u) continue;
        const float value = clean_observation(P, op, r, q, v, st, raw, previous_q, metrics) +
                            op.noise_amplitude * signed_draw(P.seed, env, episode, step, op.noise_channel);
        if (op.component == 0u) g.x = value;
        else if (op.component == 1u) g.y = value;
        else g.z = value;
        have = true;
    }
    if (have) g = normalized_or(g, make_float3(0.0f, 0.0f, -1.0f));
    for (int i = lane; i < P.nobs; i += 32) {
        const MRTaskObservationOperatorC op = P.actor[i];
        if (op.opcode == MR_TASK_OBSERVE_PROJECTED_GRAVITY && (op.flags & MR_TASK_OBSERVATION_NORMALIZE_VECTOR3) != 0u) {
            frame[i] = lane3(g, op.component);
            continue;
        }
        frame[i] = clean_observation(P, op, r, q, v, st, raw, previous_q, metrics) +
                   op.noise_amplitude * signed_draw(P.seed, env, episode, step, op.noise_channel);
    }
}

// The critic's frame (writeCriticFrame, :1403-1456): clean values, lanes
// over operators.
__device__ void write_critic(const TaskProgramDevice& P, const float* q, const float* v, const TaskEnvState& st, const float* raw,
                             const float* previous_q, const float* metrics, float* out, int lane) {
    const Root r = root_frame(P, q, v);
    for (int i = lane; i < P.ncritic; i += 32) out[i] = clean_observation(P, P.critic[i], r, q, v, st, raw, previous_q, metrics);
}

// durationSteps (:1484-1508).
__device__ __forceinline__ unsigned duration_steps(const TaskProgramDevice& P, unsigned env, unsigned episode, unsigned step,
                                                   unsigned channel) {
    const float seconds = range_draw(P.seed, env, episode, step, channel, P.duration_min, P.duration_max);
    const float steps = floorf(seconds / P.dt);
    return steps >= 1.0f ? static_cast<unsigned>(steps) : 1u;
}

// sampledDifficultyBand (:1537-1568).
__device__ __forceinline__ unsigned sample_band(const TaskProgramDevice& P, unsigned env, unsigned episode) {
    const unsigned count = static_cast<unsigned>(max(P.bands, 1));
    const unsigned lo = min(static_cast<unsigned>(P.band_min), count - 1u);
    const unsigned req = P.band_max < 0 ? count - 1u : static_cast<unsigned>(P.band_max);
    const unsigned hi = max(lo, min(req, count - 1u));
    const unsigned n = hi - lo + 1u;
    if (n == 1u) return lo;
    const float u = powf(unit_draw(P.seed, env, episode, 0u, 15u), fmaxf(P.band_exponent, 0.01f));
    return lo + min(static_cast<unsigned>(floorf(u * static_cast<float>(n))), n - 1u);
}

// sampledCommand (:1570-1615): each band widens the range by the step,
// within the limits.
__device__ __forceinline__ void sample_command(const TaskProgramDevice& P, unsigned env, unsigned episode, unsigned step, unsigned band,
                                               float* out) {
    const float b = static_cast<float>(band);
    for (unsigned k = 0; k < 3u; ++k) {
        const float lower = fmaxf(P.command_lower[k] - b * P.command_step[k], P.command_limit_lower[k]);
        const float upper = fminf(P.command_upper[k] + b * P.command_step[k], P.command_limit_upper[k]);
        out[k] = range_draw(P.seed, env, episode, step, 16u + k, lower, upper);
    }
    if (unit_draw(P.seed, env, episode, step, 19u) < P.standing_probability) out[0] = out[1] = out[2] = 0.0f;
}

__device__ __forceinline__ float3 shfl3(float3 a, int src) {
    return make_float3(__shfl_sync(0xffffffffu, a.x, src), __shfl_sync(0xffffffffu, a.y, src), __shfl_sync(0xffffffffu, a.z, src));
}
__device__ __forceinline__ float4 shfl4(float4 a, int src) {
    return make_float4(__shfl_sync(0xffffffffu, a.x, src), __shfl_sync(0xffffffffu, a.y, src), __shfl_sync(0xffffffffu, a.z, src),
                       __shfl_sync(0xffffffffu, a.w, src));
}
__device__ __forceinline__ float4 normalized4(float4 a) {
    const float s = rsqrtf(fmaxf(a.x * a.x + a.y * a.y + a.z * a.z + a.w * a.w, 1.0e-30f));
    return make_float4(a.x * s, a.y * s, a.z * s, a.w * s);
}
__device__ __forceinline__ float3 xyz3(float4 a) { return make_float3(a.x, a.y, a.z); }

// World COM position, orientation and twist of body `lane` (the tree's
// forward kinematics, the articulated step's formulas: revolute joints turn
// about their axis, prismatic ones slide along it).
struct BodyFrame {
    float3 c, v, w;
    float4 r;
};

__device__ BodyFrame body_frames(const DeviceModel& M, const float* q, const float* v, int lane) {
    BodyFrame f;
    f.c = f.v = f.w = make_float3(0.0f, 0.0f, 0.0f);
    f.r = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
    const bool mine = lane < M.nb;
    if (lane == 0 && M.floating) {
        f.c = make_float3(q[0], q[1], q[2]);
        f.r = normalized4(make_float4(q[3], q[4], q[5], q[6]));
        f.v = make_float3(v[0], v[1], v[2]);
        f.w = make_float3(v[3], v[4], v[5]);
    }
    const int depth = mine ? static_cast<int>(M.tables.depth[lane]) : -1;
    const int par = mine && lane > 0 ? M.parent[lane] : lane;
    for (int l = 1; l <= M.n_levels; ++l) {
        const float3 cp = shfl3(f.c, par), wp = shfl3(f.w, par), vp = shfl3(f.v, par);
        const float4 qp = shfl4(f.r, par);
        if (depth == l) {
            const int dof = M.body_dof[lane];
            const bool has = dof >= 0, prismatic = M.joint_type[lane] == MR_JOINT_PRISMATIC;
            const float3 axis = xyz3(M.axis[lane]);
            const float4 pj = quat_product(qp, M.parent_rotation[lane]);
            float4 motion = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
            float qj = 0.0f, qdj = 0.0f;
            if (has) {
                qj = q[M.dof_q[dof]];
                qdj = v[dof];
                if (!prismatic) {
                    float sh, ch;
                    sincosf(0.5f * qj, &sh, &ch);
                    motion = make_float4(axis.x * sh, axis.y * sh, axis.z * sh, ch);
                }
            }
            const float4 rb = normalized4(quat_product(quat_product(pj, motion), M.child_rotation_conj[lane]));
            const float3 ja = rotate(pj, axis);
            float3 jp = cp + rotate(qp, xyz3(M.parent_anchor[lane]));
            if (prismatic) jp = jp + qj * ja;
            const float3 ca = rotate(rb, xyz3(M.child_anchor[lane]));
            const float3 wb = wp + ((has && !prismatic) ? qdj * ja : make_float3(0.0f, 0.0f, 0.0f));
            f.v = vp + cross3(wp, jp - cp) + (prismatic ? qdj * ja : make_float3(0.0f, 0.0f, 0.0f)) - cross3(wb, ca);
            f.c = jp - ca;
            f.r = rb;
            f.w = wb;
        }
    }
    return f;
}

// The contact groups' compact metrics of this step (the reduction of
// LocomotionTask.metal:4104-4370 over the committed final-microstep
// contacts): out[g][0..5] force (forbidden groups: the hard-contact flag),
// slip, air time, clearance, CoP x, y; out[g][6..11] wrench in the
// reference body's frame.  `air` holds and receives each group's air time.
__device__ void contact_metrics(const TaskProgramDevice& P, const BodyFrame& f, const float* manifolds, float* air, float* out,
                                int lane) {
    const DeviceModel& M = *P.model;
    float imp[kTaskMaxGroups], hard[kTaskMaxGroups], F[kTaskMaxGroups][3], Mo[kTaskMaxGroups][3], Pw[kTaskMaxGroups][3];
#pragma unroll
    for (int g = 0; g < kTaskMaxGroups; ++g) {
        imp[g] = hard[g] = 0.0f;
        F[g][0] = F[g][1] = F[g][2] = Mo[g][0] = Mo[g][1] = Mo[g][2] = Pw[g][0] = Pw[g][1] = Pw[g][2] = 0.0f;
    }
    for (int p0 = 0; p0 < M.np; p0 += 32) {
        const int pair = p0 + lane;
        const bool live = pair < M.np;
        const int sa = live ? M.pair_a[pair] : 0, sb = live ? M.pair_b[pair] : 0;
        const int body = live ? M.shape_body[sa] : -1;
        const float4 ra = shfl4(f.r, body >= 0 ? body : 0);
        const float3 ca = shfl3(f.c, body >= 0 ? body : 0);
        if (!live || body < 0 || M.shape_body[sb] >= 0) continue;
        const float* m = manifolds + static_cast<size_t>(pair) * kManifoldWords;
        const int count = __float_as_int(m[7]);
        if (count <= 0) continue;
        float3 n = rotate(ra, make_float3(m[0], m[1], m[2]));
        n = rsqrtf(fmaxf(dot3(n, n), 1.0e-30f)) * n;
        float3 t = rotate(ra, make_float3(m[4], m[5], m[6]));
        t = t - dot3(t, n) * n;
        if (dot3(t, t) > 1.0e-12f) {
            t = rsqrtf(dot3(t, t)) * t;
        } else {  // the solver's stable tangent of the normal
            const float3 an = make_float3(fabsf(n.x), fabsf(n.y), fabsf(n.z));
            const float3 ref = an.x <= an.y && an.x <= an.z ? make_float3(1.0f, 0.0f, 0.0f)
                               : an.y <= an.z              ? make_float3(0.0f, 1.0f, 0.0f)
                                                           : make_float3(0.0f, 0.0f, 1.0f);
            t = cross3(ref, n);
            t = rsqrtf(fmaxf(dot3(t, t), 1.0e-30f)) * t;
        }
        const float3 b = cross3(n, t);
        const float3 pb0 = xyz3(M.static_body_position[sb]);
        const float4 rb0 = M.static_body_rotation[sb];
        for (int i = 0; i < count && i < kManifoldPoints; ++i) {
            const float* pt = m + 8 + i * 12;
            const float3 pa = ca + rotate(ra, make_float3(pt[0], pt[1], pt[2]));
            const float3 pw = 0.5f * (pa + pb0 + rotate(rb0, make_float3(pt[3], pt[4], pt[5])));
            const float ln = pt[9], lt = pt[10], lb = pt[11];
            // Impulse on the robot (shape A): -(n ln + t lt + b lb).
            const float3 fo = make_float3(-(n.x * ln + t.x * lt + b.x * lb), -(n.y * ln + t.y * lt + b.y * lb),
                                          -(n.z * ln + t.z * lt + b.z * lb));
            const float3 mo = cross3(pw, fo);
            const float a = fabsf(ln);
            for (int g = 0; g < P.ncontact_groups; ++g) {
                const MRTaskContactGroupC G = P.contact_groups[g];
                bool member = false;
                for (unsigned k = 0; k < G.count; ++k) member = member || P.contact_members[G.first + k] == static_cast<unsigned>(body);
                if (!member) continue;
                imp[g] += a;
                hard[g] = fmaxf(hard[g], a);
                F[g][0] += fo.x; F[g][1] += fo.y; F[g][2] += fo.z;
                Mo[g][0] += mo.x; Mo[g][1] += mo.y; Mo[g][2] += mo.z;
                Pw[g][0] += a * pw.x; Pw[g][1] += a * pw.y; Pw[g][2] += a * pw.z;
            }
        }
    }
    const float inv_h = 1.0f / P.physics_dt;
    for (int g = 0; g < P.ncontact_groups; ++g) {
        const MRTaskContactGroupC G = P.contact_groups[g];
        const float si = warp_sum(imp[g]);
        float hg = hard[g];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) hg = fmaxf(hg, __shfl_xor_sync(0xffffffffu, hg, o));
        const float3 Fw = inv_h * make_float3(warp_sum(F[g][0]), warp_sum(F[g][1]), warp_sum(F[g][2]));
        const float3 Mw = inv_h * make_float3(warp_sum(Mo[g][0]), warp_sum(Mo[g][1]), warp_sum(Mo[g][2]));
        const float3 Pa = make_float3(warp_sum(Pw[g][0]), warp_sum(Pw[g][1]), warp_sum(Pw[g][2]));
        const int rbody = static_cast<int>(G.reference_body);
        const float3 cr = shfl3(f.c, rbody), vr = shfl3(f.v, rbody), wr = shfl3(f.w, rbody);
        const float4 rr = shfl4(f.r, rbody);
        const float3 ref = cr + rotate(rr, xyz3(make_float4(G.local_reference[0], G.local_reference[1], G.local_reference[2], 0.0f)));
        float* o = out + g * kTaskGroupMetrics;
        const float3 fl = rotate_inverse(rr, Fw);
        const float3 tl = rotate_inverse(rr, Mw - cross3(ref, Fw));
        o[6] = fl.x; o[7] = fl.y; o[8] = fl.z;
        o[9] = tl.x; o[10] = tl.y; o[11] = tl.z;
        o[1] = o[2] = o[3] = o[4] = o[5] = 0.0f;
        if (G.flags & MR_TASK_CONTACT_SUPPORT) {
            const float force = si * inv_h;
            const bool touching = force > P.support_force_threshold;
            const float3 koff = rotate(rr, make_float3(G.kinematic_reference[0], G.kinematic_reference[1], G.kinematic_reference[2]));
            const float3 kv = vr + cross3(wr, koff);
            const float air_prev = air[g];
            o[0] = force;
            o[1] = touching ? sqrtf(kv.x * kv.x + kv.y * kv.y) : 0.0f;
            o[2] = touching ? 0.0f : air_prev + P.dt;
            o[3] = ref.z - G.local_reference[3] - P.ground_height;
            if (si > 1.0e-6f) {
                const float3 cl = rotate_inverse(rr, Pa - si * ref);
                o[4] = cl.x / si;
                o[5] = cl.y / si;
            }
        } else if (G.flags & MR_TASK_CONTACT_FORBIDDEN) {
            o[0] = hg * inv_h > P.support_force_threshold ? 1.0f : 0.0f;
        } else {
            o[0] = 0.0f;
        }
    }
    __syncwarp();
    if (lane < P.ncontact_groups) air[lane] = out[lane * kTaskGroupMetrics + 2];
}

// desiredSupportContact (:1617-1630).
__device__ __forceinline__ bool desired_support(const MRTaskContactGroupC& G, float phase) {
    float x = fmodf(phase + G.gait_phase_offset, kTwoPi);
    if (x < 0.0f) x += kTwoPi;
    return x / kTwoPi < G.stance_fraction;
}

__global__ void __launch_bounds__(32 * kTaskWarps) task_observe_kernel(TaskParams p) {
    const int lane = threadIdx.x & 31;
    const int local = blockIdx.x * kTaskWarps + (threadIdx.x >> 5);
    if (local >= p.env_count) return;
    const TaskProgramDevice& P = p.prog;
    const unsigned env = static_cast<unsigned>(p.env_base + local);
    TaskEnvState st = p.state[local];
    const bool reset = st.initialized == 0u || st.pending_reset != 0u || (p.masks_in != nullptr && p.masks_in[local] != 0u);
    float* frame = p.frame + static_cast<size_t>(local) * P.frames * P.nobs;  // the env's history, oldest first
    if (reset) {
        const unsigned episode = st.episode + 1u;
        float* rq = p.reset_q + static_cast<size_t>(local) * P.nq;
        float* rv = p.reset_v + static_cast<size_t>(local) * P.nv;
        for (int i = lane; i < P.nq; i += 32) rq[i] = P.default_q[i];
        for (int i = lane; i < P.nv; i += 32) rv[i] = 0.0f;
        __syncwarp();
        st.action_delay = static_cast<unsigned>(P.delay);
        st.observation_delay = 0u;
        st.band = sample_band(P, env, episode);
        // Randomization operators in order (:2452-2770), channel 2048 + index.
        for (int k = 0; k < P.nrandom; ++k) {
            const MRTaskRandomizationOperatorC op = P.randomization[k];
            const unsigned channel = 2048u + static_cast<unsigned>(k);
            if (st.band < op.minimum_band) continue;
            switch (op.opcode) {
            case MR_TASK_RANDOMIZE_ROOT_POSITION:
                if (lane < 3) rq[lane] += op.parameters[lane] * signed_draw(P.seed, env, episode, 0u, channel + lane);
                break;
            case MR_TASK_RANDOMIZE_ROOT_YAW:
                if (lane == 0) {
                    const float yaw = range_draw(P.seed, env, episode, 0u, channel, op.parameters[0], op.parameters[1]);
                    const float half = 0.5f * yaw;
                    const float4 authored = make_float4(P.default_q[3], P.default_q[4], P.default_q[5], P.default_q[6]);
                    const float4 out = quat_product(make_float4(0.0f, 0.0f, sinf(half), cosf(half)), authored);
                    rq[3] = out.x;
                    rq[4] = out.y;
                    rq[5] = out.z;
                    rq[6] = out.w;
                }
                break;
            case MR_TASK_RANDOMIZE_ROOT_HEIGHT:
                if (lane == 0) rq[2] = range_draw(P.seed, env, episode, 0u, channel, op.parameters[0], op.parameters[1]);
                break;
            case MR_TASK_RANDOMIZE_JOINT_POSITION:
                if (lane == 0) rq[op.target] = range_draw(P.seed, env, episode, 0u, channel, op.parameters[0], op.parameters[1]);
                break;
            case MR_TASK_RANDOMIZE_ACTION_POSITION:
                for (int a = lane; a < P.na; a += 32) {
                    const MRTaskActionBindingC b = P.actions[a];
                    const float x = P.default_q[b.q_index] +
                                    range_draw(P.seed, env, episode, 0u, channel + a, op.parameters[0], op.parameters[1]);
                    rq[b.q_index] = fminf(fmaxf(x, b.lower_target), b.upper_target);
                }
                break;
            case MR_TASK_RANDOMIZE_VELOCITY:
                for (int i = lane; i < P.nv; i += 32)
                    rv[i] = range_draw(P.seed, env, episode, 0u, channel + i, op.parameters[0], op.parameters[1]);
                break;
            case MR_TASK_RANDOMIZE_ACTION_DELAY:
            case MR_TASK_RANDOMIZE_OBSERVATION_DELAY: {
                // An integer in [lower, upper] (:2738-2783), capped.
                const unsigned lo = static_cast<unsigned>(fmaxf(op.parameters[0], 0.0f));
                const unsigned hi = static_cast<unsigned>(fmaxf(op.parameters[1], op.parameters[0]));
                const unsigned d = lo + static_cast<unsigned>(floorf(static_cast<float>(hi - lo + 1u) *
                                                                     unit_draw(P.seed, env, episode, 0u, channel)));
                if (op.opcode == MR_TASK_RANDOMIZE_ACTION_DELAY)
                    st.action_delay = min(d, static_cast<unsigned>(P.history - 1));
                else
                    st.observation_delay = min(d, static_cast<unsigned>(P.max_observation_delay));
                break;
            }
            case MR_TASK_RANDOMIZE_ACTION_VELOCITY:
                for (int a = lane; a < P.na; a += 32)
                    rv[P.actions[a].v_index] = range_draw(P.seed, env, episode, 0u, channel + a, op.parameters[0], op.parameters[1]);
                break;
            default:
                break;
            }
            __syncwarp();
        }
        float* hist = p.action_history + static_cast<size_t>(local) * P.history * P.na;
        float* prev = p.previous_joint + static_cast<size_t>(local) * 2 * P.na;
        for (int i = lane; i < P.history * P.na; i += 32) hist[i] = 0.0f;
        if (lane < kTaskMaxGroups) p.air_time[static_cast<size_t>(local) * kTaskMaxGroups + lane] = 0.0f;
        for (int a = lane; a < P.na; a += 32) {
            prev[a] = 0.0f;
            prev[P.na + a] = rq[P.actions[a].q_index];
        }
        // A new episode (:2947-3010).
        st.episode_step = 0u;
        st.episode = episode;
        st.command_steps = duration_steps(P, env, episode, 0u, 32u);
        st.initialized = 1u;
        st.pending_reset = 0u;
        st.last_reason = MR_TASK_TERMINATION_CONTINUING;
        sample_command(P, env, episode, 0u, st.band, st.command);
        st.phase = 0.0f;
        st.previous_height = root_frame(P, rq, rv).position.z;
        st.episode_return = 0.0f;
        st.episode_tracking = 0.0f;
        __syncwarp();
        // Every delay-line slot is zero here; the newest raw slot stands for
        // all of them.
        write_frame(P, rq, rv, st, hist + (P.history - 2) * P.na, prev + P.na, nullptr, env, episode, 0u, frame, lane);
        if (P.ncritic > 0)
            write_critic(P, rq, rv, st, hist + (P.history - 2) * P.na, prev + P.na, nullptr,
                         p.critic_frame + static_cast<size_t>(local) * P.ncritic, lane);
        __syncwarp();
        for (int i = lane; i < (P.frames - 1) * P.nobs; i += 32) frame[P.nobs + i] = frame[i % P.nobs];  // every slot the reset frame
        if (lane == 0) p.state[local] = st;
    }
    if (lane == 0) p.masks_out[local] = reset ? 1u : 0u;
    __syncwarp();
    if (p.observations) {
        float* out = p.observations + static_cast<size_t>(local) * P.frames * P.nobs;
        for (int i = lane; i < P.frames * P.nobs; i += 32) out[i] = frame[i];
    }
}

// One thread per (environment, action) (:3520-3668).
__global__ void __launch_bounds__(kApplyThreads) task_apply_kernel(TaskParams p) {
    const TaskProgramDevice& P = p.prog;
    const long long idx = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (idx >= static_cast<long long>(p.env_count) * P.na) return;
    const int local = static_cast<int>(idx / P.na), a = static_cast<int>(idx - static_cast<long long>(local) * P.na);
    float* hist = p.action_history + static_cast<size_t>(local) * P.history * P.na;
    const int filter = P.history - 1, raw_last = filter - 1;
    for (int d = 0; d < raw_last; ++d) hist[d * P.na + a] = hist[(d + 1) * P.na + a];
    const float requested = p.actions[static_cast<size_t>(local) * P.na + a];
    const float previous = hist[filter * P.na + a];
    const MRTaskActionBindingC b = P.actions[a];
    const float response = b.response_time_seconds > 0.0f
                               ? fminf(fmaxf(1.0f - expf(-P.dt / b.response_time_seconds), 0.0f), 1.0f)
                               : 1.0f;
    hist[raw_last * P.na + a] = requested;
    const int selected = raw_last - min(static_cast<int>(p.state[local].action_delay), raw_last);
    const float filtered = mixf(previous, hist[selected * P.na + a], response);
    hist[filter * P.na + a] = filtered;
    const float target = P.default_q[b.q_index] + b.scale * filtered;
    p.targets[static_cast<size_t>(local) * P.na + a] = fminf(fmaxf(target, b.lower_target), b.upper_target);
}

__global__ void __launch_bounds__(32 * kTaskWarps) task_complete_kernel(TaskParams p) {
    const int lane = threadIdx.x & 31;
    const int local = blockIdx.x * kTaskWarps + (threadIdx.x >> 5);
    if (local >= p.env_count) return;
    const TaskProgramDevice& P = p.prog;
    const unsigned env = static_cast<unsigned>(p.env_base + local);
    TaskEnvState st = p.state[local];
    const float* q = p.q + static_cast<size_t>(local) * P.nq;
    const float* v = p.v + static_cast<size_t>(local) * P.nv;
    float* hist = p.action_history + static_cast<size_t>(local) * P.history * P.na;
    float* prev = p.previous_joint + static_cast<size_t>(local) * 2 * P.na;
    const bool physics_error = p.status[local] != MR_STEP_SUCCESS;

    // Reward inputs (:4376-4500).
    const Root r = root_frame(P, q, v);
    const float3 base_linear = rotate_inverse(r.orientation, r.linear);
    const float3 base_angular = rotate_inverse(r.orientation, r.angular);
    const float3 gravity = projected_gravity(r);
    const float height = r.position.z;
    const float tilt = atan2f(sqrtf(gravity.x * gravity.x + gravity.y * gravity.y), fmaxf(-gravity.z, 1.0e-6f));
    const float4 o = r.orientation;
    float yx = 1.0f - 2.0f * (o.y * o.y + o.z * o.z), yy = 2.0f * (o.w * o.z + o.x * o.y);
    const float ys = rsqrtf(fmaxf(yx * yx + yy * yy, 1.0e-12f));
    yx *= ys;
    yy *= ys;
    const float fx = yx * r.linear.x + yy * r.linear.y, fy = -yy * r.linear.x + yx * r.linear.y;
    const float tdx = fx - st.command[0], tdy = fy - st.command[1];
    const float tracking_error = tdx * tdx + tdy * tdy;
    const float yaw_delta = base_angular.z - st.command[2];
    const float yaw_error = yaw_delta * yaw_delta;

    const int raw_last = P.history - 2, raw_previous = raw_last - 1;
    float vel2 = 0.0f, acc2 = 0.0f, rate2 = 0.0f, lim2 = 0.0f;
    for (int a = lane; a < P.na; a += 32) {
        const MRTaskActionBindingC b = P.actions[a];
        const float delta = hist[raw_last * P.na + a] - hist[raw_previous * P.na + a];
        rate2 += delta * delta;
        const float position = q[b.q_index], velocity = v[b.v_index];
        const float acceleration = (velocity - prev[a]) / P.dt;
        const float lower = fmaxf(P.limit_lower[a] - position, 0.0f), upper = fmaxf(position - P.limit_upper[a], 0.0f);
        vel2 += velocity * velocity;
        acc2 += acceleration * acceleration;
        lim2 += lower * lower + upper * upper;
    }
    vel2 = warp_sum(vel2);
    acc2 = warp_sum(acc2);
    rate2 = warp_sum(rate2);
    lim2 = warp_sum(lim2);

    const float phase = fmodf(st.phase + kTwoPi * P.dt / P.gait_period, kTwoPi);
    const bool moving = sqrtf(st.command[0] * st.command[0] + st.command[1] * st.command[1] + st.command[2] * st.command[2]) > 0.1f;
    float gm[kTaskMaxGroups * kTaskGroupMetrics];
    BodyFrame frames;  // body `lane`'s world frame (contact groups only)
    if (P.ncontact_groups > 0) {
        frames = body_frames(*P.model, q, v, lane);
        contact_metrics(P, frames, p.manifolds + static_cast<size_t>(local) * P.model->np * kManifoldWords,
                        p.air_time + static_cast<size_t>(local) * kTaskMaxGroups, gm, lane);
    }

    float reward = 0.0f;
    float b0[4] = {0.0f, 0.0f, 0.0f, 0.0f}, b1[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    for (int k = 0; k < P.nrewards; ++k) {
        const MRTaskRewardOperatorC op = P.rewards[k];
        float value = 0.0f;
        switch (op.opcode) {
        case MR_TASK_REWARD_LINEAR_VELOCITY_TRACKING:
            value = expf(-tracking_error / fmaxf(op.parameters[0], 1.0e-8f));
            break;
        case MR_TASK_REWARD_YAW_VELOCITY_TRACKING:
            value = expf(-yaw_error / fmaxf(op.parameters[0], 1.0e-8f));
            break;
        case MR_TASK_REWARD_CONSTANT:
            value = 1.0f;
            break;
        case MR_TASK_REWARD_ROOT_VERTICAL_VELOCITY_SQUARED:
            value = base_linear.z * base_linear.z;
            break;
        case MR_TASK_REWARD_ROOT_ROLL_PITCH_VELOCITY_SQUARED:
            value = base_angular.x * base_angular.x + base_angular.y * base_angular.y;
            break;
        case MR_TASK_REWARD_TILT_SQUARED:
            value = tilt * tilt;
            break;
        case MR_TASK_REWARD_PROJECTED_GRAVITY_HORIZONTAL_SQUARED:
            value = gravity.x * gravity.x + gravity.y * gravity.y;
            break;
        case MR_TASK_REWARD_ROOT_HEIGHT_ERROR_SQUARED: {
            const float e = height - P.base_height;
            value = e * e;
            break;
        }
        case MR_TASK_REWARD_ROOT_HEIGHT_NORMALIZED:
            value = fminf(fmaxf(height / fmaxf(P.base_height, 1.0e-6f), 0.0f), 1.0f);
            break;
        case MR_TASK_REWARD_ROOT_HEIGHT_PROGRESS:
            value = fminf(fmaxf((height - st.previous_height) / P.dt, -2.0f), 2.0f);
            break;
        case MR_TASK_REWARD_UPRIGHTNESS: {
            const float up = fminf(fmaxf(-gravity.z, 0.0f), 1.0f);
            value = up * up;
            break;
        }
        case MR_TASK_REWARD_JOINT_VELOCITY_SQUARED:
            value = vel2;
            break;
        case MR_TASK_REWARD_JOINT_ACCELERATION_SQUARED:
            value = acc2;
            break;
        case MR_TASK_REWARD_ACTION_RATE_SQUARED:
            value = rate2;
            break;
        case MR_TASK_REWARD_JOINT_LIMIT_VIOLATION_SQUARED:
            value = lim2;
            break;
        case MR_TASK_REWARD_JOINT_LIMIT_VIOLATION_ABSOLUTE: {
            const float soft = fminf(fmaxf(op.parameters[0], 1.0e-6f), 1.0f);
            float sum = 0.0f;
            for (int a = lane; a < P.na; a += 32) {
                const float center = 0.5f * (P.limit_lower[a] + P.limit_upper[a]);
                const float half = 0.5f * (P.limit_upper[a] - P.limit_lower[a]) * soft;
                const float position = q[P.actions[a].q_index];
                sum += fmaxf(center - half - position, 0.0f) + fmaxf(position - center - half, 0.0f);
            }
            value = warp_sum(sum);
            break;
        }
        case MR_TASK_REWARD_JOINT_GROUP_POSTURE_SQUARED:
        case MR_TASK_REWARD_JOINT_GROUP_POSTURE_ABSOLUTE: {
            const MRTaskIndexGroupC g = P.groups[op.group];
            float sum = 0.0f;
            for (unsigned m = static_cast<unsigned>(lane); m < g.count; m += 32u) {
                const int qi = static_cast<int>(P.actions[P.members[g.first + m]].q_index);
                const float e = q[qi] - P.default_q[qi];
                sum += op.opcode == MR_TASK_REWARD_JOINT_GROUP_POSTURE_SQUARED ? e * e : fabsf(e);
            }
            sum = warp_sum(sum);
            value = op.opcode == MR_TASK_REWARD_JOINT_GROUP_POSTURE_SQUARED ? sum / fmaxf(static_cast<float>(g.count), 1.0f) : sum;
            break;
        }
        case MR_TASK_REWARD_GAIT_CONTACT_MATCH:
        case MR_TASK_REWARD_SWING_CLEARANCE:
        case MR_TASK_REWARD_FOOT_CLEARANCE:
        case MR_TASK_REWARD_SUPPORT_SLIP:
        case MR_TASK_REWARD_FORBIDDEN_CONTACT: {
            // The contact-group operators (:5405-5553); `group` selects one
            // group, MR_INVALID_INDEX every group.
            float acc = 0.0f, count = 0.0f;
            for (int g = 0; g < P.ncontact_groups; ++g) {
                if (op.group != MR_INVALID_INDEX && op.group != static_cast<unsigned>(g)) continue;
                const MRTaskContactGroupC G = P.contact_groups[g];
                const float* m = gm + g * kTaskGroupMetrics;
                const bool support = (G.flags & MR_TASK_CONTACT_SUPPORT) != 0u;
                if (op.opcode == MR_TASK_REWARD_GAIT_CONTACT_MATCH && support) {
                    acc += desired_support(G, phase) == (m[0] > P.support_force_threshold) ? 1.0f : 0.0f;
                } else if (op.opcode == MR_TASK_REWARD_SWING_CLEARANCE && support && !desired_support(G, phase)) {
                    const float e = m[3] - P.clearance_target;
                    acc += expf(-(e * e) / fmaxf(op.parameters[0], 1.0e-8f));
                    count += 1.0f;
                } else if (op.opcode == MR_TASK_REWARD_SUPPORT_SLIP && support) {
                    acc += m[1];
                } else if (op.opcode == MR_TASK_REWARD_FORBIDDEN_CONTACT && (G.flags & MR_TASK_CONTACT_FORBIDDEN)) {
                    acc = fmaxf(acc, m[0]);
                } else if (op.opcode == MR_TASK_REWARD_FOOT_CLEARANCE && support) {
                    // Height of the kinematic reference point, weighted by its planar speed.
                    const int rb = static_cast<int>(G.reference_body);
                    const float3 c = shfl3(frames.c, rb), vb = shfl3(frames.v, rb), wb = shfl3(frames.w, rb);
                    const float4 r = shfl4(frames.r, rb);
                    const float3 off = rotate(r, make_float3(G.kinematic_reference[0], G.kinematic_reference[1], G.kinematic_reference[2]));
                    const float3 vel = vb + cross3(wb, off);
                    const float e = c.z + off.z - P.clearance_target;
                    acc += e * e * tanhf(op.parameters[1] * sqrtf(vel.x * vel.x + vel.y * vel.y));
                }
            }
            if (op.opcode == MR_TASK_REWARD_FOOT_CLEARANCE) value = expf(-acc / fmaxf(op.parameters[0], 1.0e-8f));
            else if (op.opcode == MR_TASK_REWARD_SWING_CLEARANCE) value = moving ? acc / fmaxf(count, 1.0f) : 0.0f;
            else if (op.opcode == MR_TASK_REWARD_GAIT_CONTACT_MATCH) value = moving ? acc : 0.0f;
            else value = acc;
            break;
        }
        default:
            break;
        }
        const float contribution = op.weight * value;
        reward += contribution;
        // Reward breakdown lanes (:5985-6046).
        switch (op.opcode) {
        case MR_TASK_REWARD_LINEAR_VELOCITY_TRACKING:
        case MR_TASK_REWARD_YAW_VELOCITY_TRACKING:
        case MR_TASK_REWARD_CONSTANT:
        case MR_TASK_REWARD_GAIT_CONTACT_MATCH:
        case MR_TASK_REWARD_SWING_CLEARANCE:
        case MR_TASK_REWARD_FOOT_CLEARANCE:
            b0[0] += contribution;
            break;
        case MR_TASK_REWARD_SUPPORT_SLIP:
        case MR_TASK_REWARD_FORBIDDEN_CONTACT:
            b1[3] += contribution;
            break;
        case MR_TASK_REWARD_JOINT_VELOCITY_SQUARED:
            b0[2] += contribution;
            break;
        case MR_TASK_REWARD_JOINT_ACCELERATION_SQUARED:
            b0[3] += contribution;
            break;
        case MR_TASK_REWARD_ACTION_RATE_SQUARED:
            b1[0] += contribution;
            break;
        case MR_TASK_REWARD_JOINT_LIMIT_VIOLATION_SQUARED:
        case MR_TASK_REWARD_JOINT_LIMIT_VIOLATION_ABSOLUTE:
        case MR_TASK_REWARD_JOINT_GROUP_POSTURE_SQUARED:
        case MR_TASK_REWARD_JOINT_GROUP_POSTURE_ABSOLUTE:
            b1[1] += contribution;
            break;
        default:  // the base-state operators
            b0[1] += contribution;
            break;
        }
    }

    // Terminations (:6064-6160): the highest priority among the triggered.
    const unsigned episode_steps = st.episode_step + 1u;
    const bool timeout = episode_steps >= static_cast<unsigned>(P.max_episode_steps);
    bool done = false;
    unsigned reason = MR_TASK_TERMINATION_CONTINUING, priority = 0u;
    float penalty = 0.0f;
    for (int k = 0; k < P.nterminations; ++k) {
        const MRTaskTerminationOperatorC op = P.terminations[k];
        const unsigned top = op.maximum_band == MR_INVALID_INDEX ? static_cast<unsigned>(max(P.bands, 1) - 1) : op.maximum_band;
        if (st.band < op.minimum_band || st.band > top) continue;
        const bool triggered = op.opcode == MR_TASK_TERMINATE_MINIMUM_ROOT_HEIGHT ? height < op.threshold
                               : op.opcode == MR_TASK_TERMINATE_MAXIMUM_TILT        ? tilt > op.threshold
                               : op.opcode == MR_TASK_TERMINATE_CONTACT_GROUP
                                   ? gm[op.group * kTaskGroupMetrics] > op.threshold
                                   : false;
        if (triggered && (!done || op.priority >= priority)) {
            done = true;
            reason = op.reason;
            priority = op.priority;
            penalty = op.failure_penalty;
        }
    }
    if (timeout) {
        done = true;
        reason = MR_TASK_TERMINATION_TIMEOUT;
    }
    if (physics_error) {
        done = true;
        reason = MR_TASK_TERMINATION_PHYSICS_ERROR;
    }
    if (done && reason != MR_TASK_TERMINATION_TIMEOUT && reason != MR_TASK_TERMINATION_PHYSICS_ERROR) {
        reward += penalty;
        b0[1] += penalty;
    }
    reward *= P.dt;
    for (int i = 0; i < 4; ++i) {
        b0[i] *= P.dt;
        b1[i] *= P.dt;
    }
    const float tracking = expf(-tracking_error / 0.25f);
    const float yaw_tracking = expf(-yaw_error / 0.25f);
    const float episode_tracking = st.episode_tracking + tracking;
    const float episode_score = episode_tracking / fmaxf(static_cast<float>(episode_steps), 1.0f);
    const float episode_return = st.episode_return + reward;

    // Command schedule and state (:6388-6440).
    if (!done && st.command_steps <= 1u) {
        sample_command(P, env, st.episode, episode_steps, st.band, st.command);
        st.command_steps = duration_steps(P, env, st.episode, episode_steps, 64u);
    } else if (!done) {
        --st.command_steps;
    }
    st.episode_step = episode_steps;
    st.pending_reset = done ? 1u : 0u;
    st.last_reason = reason;
    st.phase = phase;
    st.previous_height = height;
    st.episode_return = done ? 0.0f : episode_return;
    st.episode_tracking = done ? 0.0f : episode_tracking;

    // The next decision's frame, then this step's joint history (:6478-6630).
    if (!done || (timeout && !physics_error)) {
        float* frame = p.frame + static_cast<size_t>(local) * P.frames * P.nobs;
        // Shift the history one frame older, then write the newest (:6478-6517).
        for (int h = 0; h + 1 < P.frames; ++h) {
            for (int i = lane; i < P.nobs; i += 32) frame[h * P.nobs + i] = frame[(h + 1) * P.nobs + i];
            __syncwarp();
        }
        write_frame(P, q, v, st, hist + raw_last * P.na, prev + P.na, gm, env, st.episode, episode_steps,
                    frame + (P.frames - 1) * P.nobs, lane);
        if (st.observation_delay != 0u && P.frames > 1) {  // the newest slot shows an older frame (:6549-6565)
            __syncwarp();
            const int src = P.frames - 1 - min(static_cast<int>(st.observation_delay), P.frames - 1);
            for (int i = lane; i < P.nobs; i += 32) frame[(P.frames - 1) * P.nobs + i] = frame[src * P.nobs + i];
        }
        if (P.ncritic > 0)
            write_critic(P, q, v, st, hist + raw_last * P.na, prev + P.na, gm, p.critic_frame + static_cast<size_t>(local) * P.ncritic,
                         lane);
        __syncwarp();
        for (int a = lane; a < P.na; a += 32) {
            const MRTaskActionBindingC b = P.actions[a];
            prev[a] = v[b.v_index];
            prev[P.na + a] = q[b.q_index];
        }
    }
    if (lane == 0) {
        p.state[local] = st;
        MRTaskTransitionC t{};
        t.reward = reward;
        t.tracking_score = 0.5f * (tracking + yaw_tracking);
        t.root_height = height;
        t.tilt = tilt;
        t.done = done ? 1u : 0u;
        t.timeout = timeout ? 1u : 0u;
        t.physics_error = physics_error ? 1u : 0u;
        t.termination_reason = reason;
        t.task_reward = b0[0];
        t.base_reward = b0[1];
        t.joint_velocity_reward = b0[2];
        t.joint_acceleration_reward = b0[3];
        t.control_reward = b1[0];
        t.posture_reward = b1[1];
        t.energy_reward = b1[2];
        t.contact_reward = b1[3];
        t.policy_revision = p.policy_revision;
        t.episode_tracking_score = done && !physics_error ? episode_score : 0.0f;
        t.difficulty_band = st.band;
        p.transitions[local] = t;
    }
}

}  // namespace

cudaError_t launch_task_observe(const TaskParams& p, cudaStream_t stream) {
    if (p.env_count <= 0) return cudaSuccess;
    const int blocks = (p.env_count + kTaskWarps - 1) / kTaskWarps;
    task_observe_kernel<<<blocks, 32 * kTaskWarps, 0, stream>>>(p);
    return cudaGetLastError();
}

cudaError_t launch_task_apply(const TaskParams& p, cudaStream_t stream) {
    const long long n = static_cast<long long>(p.env_count) * p.prog.na;
    if (n <= 0) return cudaSuccess;
    const int blocks = static_cast<int>((n + kApplyThreads - 1) / kApplyThreads);
    task_apply_kernel<<<blocks, kApplyThreads, 0, stream>>>(p);
    return cudaGetLastError();
}

cudaError_t launch_task_complete(const TaskParams& p, cudaStream_t stream) {
    if (p.env_count <= 0) return cudaSuccess;
    const int blocks = (p.env_count + kTaskWarps - 1) / kTaskWarps;
    task_complete_kernel<<<blocks, 32 * kTaskWarps, 0, stream>>>(p);
    return cudaGetLastError();
}

}  // namespace numi
