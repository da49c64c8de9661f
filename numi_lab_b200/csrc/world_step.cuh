// Batched articulated-physics control step for B200 (sm_100a): device code
// shared by the per-world kernel (world_step.cu) and the heterogeneous
// batch kernel (mix_step.cu).
//
// One warp owns one environment for a whole control step (all physics
// substeps).  Lane b owns body b of the tree (<= 32 bodies): its constants,
// articulated inertia, bias, joint subspace and factor live in registers
// through the tree sweeps, and only values a child or parent needs cross
// lanes, through shared memory.  Byte-sized topology tables sit in the CTA's
// shared memory.  HBM sees each control step's inputs (resident q, v,
// manifolds, actions, reset mask) once and its outputs (committed state,
// observation, status) once.
//
// Stage order per substep follows numi-lab's MetalWorld graph
// (src/metal/MetalWorld.mm:17075-17370 and encodeContactSubstep
// :12682-13260): drive refresh -> ABA -> [kinematics, collider projection,
// pair flags, narrowphase, persistent manifolds, ConstraintIR evaluation,
// contact responses, temporalCone solve, joint limits, integration] -> latch.
// The control step is one transaction: the first failing substep latches a
// status and the environment keeps its step-start checkpoint.
//
// Contact responses use the tree-sparse factor H = L^T L of the joint-space
// inertia (Featherstone, Rigid Body Dynamics Algorithms, sec. 6.5):
// Y = L^-T G^T is nonzero only on a contact body's ancestor DoFs, the
// temporalCone sweeps run on z = Y lambda (contact velocities
// u = u_free + Y^T z), and one substitution L x = z returns the velocity
// change x = H^-1 G^T lambda.  It is the reference's Jacobi block iteration
// in generalized velocities (MetalWorldContact.metal:6655-7000), evaluated
// without dense response columns.
#pragma once

#include "device_model.h"
#include "dmath.cuh"
#include "layout.h"
#include "audit.cuh"
#include "contact.cuh"
#include "quality.cuh"

#include <cfloat>
#include <cstdint>

namespace numi {
namespace {

constexpr float kFloatEps = 1.1920928955078125e-7f;
constexpr float kAbsolutePivotFloor = 1.0e-12f;
constexpr float kQueryPad = 0.00000762939453125f;  // MR_COLLISION_QUERY_RELATIVE_PAD
constexpr float kAabbPad = 0.00000762939453125f;   // MR_COLLISION_AABB_RELATIVE_PAD
constexpr unsigned char kNone = 255;
constexpr int kMaxRawPerPair = 8;
constexpr int kRootFactorWords = 24;  // rows 0-5 of the factor (21 words), padded
constexpr int kRegisterChain = 16;    // longest ancestor chain solved in registers
constexpr int kMaxCandidates = 4 + kMaxRawPerPair;  // manifold candidates of one pair
constexpr float kTieRelative = 1.0e-5f;  // manifold reduction ties
constexpr float kTieAbsolute = 1.0e-12f;

__device__ __forceinline__ int as_int(float f) { return __float_as_int(f); }
__device__ __forceinline__ float as_float(int i) { return __int_as_float(i); }

struct Warp {
    int lane;
    float* s;  // this warp's shared-memory base
    const WarpLayout* L;
    const DeviceModel* M;
    const DeviceTables* T;  // shared-memory copy
};

__device__ __forceinline__ void set_status(float* misc, unsigned code, unsigned index) {
    // Only the first failure of a control step is kept.
    if (as_int(misc[kMiscStatus]) == MR_STEP_SUCCESS) {
        misc[kMiscStatus] = as_float(static_cast<int>(code));
        misc[kMiscFailIndex] = as_float(static_cast<int>(index));
    }
}

__device__ __forceinline__ bool warp_ok(const float* misc) {
    __syncwarp();
    return as_int(misc[kMiscStatus]) == MR_STEP_SUCCESS;
}

// Per-lane body topology, loaded once per control step.  The body's float
// constants (joint frames, mass, inertia) are read from the model record at
// their point of use: every warp of an SM reads the same record, so those
// loads hit L1, and registers stay free for the FP64 articulated inertia.
struct BodyConst {
    int parent, dof, type, qidx;
};

__device__ void load_body(const DeviceModel& M, int b, BodyConst& c) {
    c.parent = M.parent[b];
    c.dof = M.body_dof[b];
    c.type = M.joint_type[b];
    c.qidx = c.dof >= 0 ? M.dof_q[c.dof] : -1;
}

// Per-lane dynamic body state of one substep.  R is the precision of the
// articulated inertia and its joint terms (U = I s, D, u): float (the
// reference's precision) or double (the FP64 articulated-inertia mode).
// Shifting a child's inertia to its parent's COM adds parallel-axis terms
// two to three orders of magnitude larger than the pivots D of light distal
// links, and FP32 rounding of those terms alone moves joint accelerations by
// ~3e-5 relative on a 7-link chain.
template <typename R>
struct BodyState {
    float3 c;       // COM position
    float4 qr;      // orientation
    float3 w, v;    // angular velocity, COM linear velocity
    float3 ba, bl;  // velocity-product bias accelerations
    float3 r;       // parent COM -> body COM
    float s[6];     // joint motion subspace about this body's COM
    R I[21];        // articulated inertia, packed symmetric
    float p[6];     // articulated bias force
    R U[6], D, u;
};

// ---------------------------------------------------------------------------
// Drives: implicit PD refresh or effort pass-through with the actuator
// envelope (MetalWorld.metal:113-370 with the default actuator profile of
// MetalWorld.mm:1376-1411, which reduces the envelope to min(limit, stall)).
// ---------------------------------------------------------------------------
__device__ void compute_drives(const Warp& w) {
    const DeviceModel& M = *w.M;
    const float* q = w.s + w.L->q;
    const float* v = w.s + w.L->v;
    const float* tgt = w.s + w.L->tgt;
    float* tau = w.s + w.L->tau;
    for (int d = w.lane; d < M.nv; d += 32) {
        const unsigned flags = M.dof_flags[d];
        const float vel = v[d];
        float command = tgt[d];
        if (M.implicit_drives) {
            command = 0.0f;
            if ((flags & MR_DOF_FLAG_DRIVE) != 0u && M.dof_q[d] >= 0) {
                float target = tgt[d];
                if ((flags & MR_DOF_FLAG_POSITION_LIMIT) != 0u) target = fminf(fmaxf(target, M.q_lower[d]), M.q_upper[d]);
                command = M.kp[d] * (target - q[M.dof_q[d]] - M.h * vel) - M.kd[d] * vel;
                const float dry = M.dry_friction[d];
                if (dry > 0.0f) {
                    if (fabsf(vel) > 1.0e-4f) command -= copysignf(dry, vel);
                    else command -= fminf(fmaxf(command, -dry), dry);
                }
                if ((flags & MR_DOF_FLAG_EFFORT_LIMIT) != 0u && M.effort_limit[d] > 0.0f)
                    command = fminf(fmaxf(command, -M.effort_limit[d]), M.effort_limit[d]);
            }
        }
        const float envelope = M.effort_envelope[d];
        tau[d] = fminf(fmaxf(command, -envelope), envelope);
    }
}

// Packed symmetric 6x6 spatial inertia shift X^T I X for a translation r
// from a child COM to its parent COM (ArticulatedABA.metal:1230-1262 with
// motionTransformElement :160-190, written out in 3x3 blocks):
// I = [[A, B], [B^T, D]], E = [r]x:  A' = A - B E + E B^T - E D E,
// B' = B + E D, D' = D.
template <typename R>
struct Vec3 {
    R x, y, z;
};
template <typename R>
__device__ __forceinline__ Vec3<R> vcross(Vec3<R> a, Vec3<R> b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

template <typename R>
__device__ __forceinline__ void shift_inertia(R* I, float3 rf) {
    // In place.  With E = [r]x: row i of B E is B_i x r, E D column j is
    // r x D_j, E B^T = -(B E)^T and row i of E D E is (E D)_i x r.
    const Vec3<R> r{rf.x, rf.y, rf.z};
    Vec3<R> EDc[3], BE[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        EDc[i] = vcross(r, Vec3<R>{I[sym6(3, 3 + i)], I[sym6(4, 3 + i)], I[sym6(5, 3 + i)]});
        BE[i] = vcross(Vec3<R>{I[sym6(3, i)], I[sym6(4, i)], I[sym6(5, i)]}, r);
    }
    const Vec3<R> E0 = vcross(Vec3<R>{EDc[0].x, EDc[1].x, EDc[2].x}, r);
    const Vec3<R> E1 = vcross(Vec3<R>{EDc[0].y, EDc[1].y, EDc[2].y}, r);
    const Vec3<R> E2 = vcross(Vec3<R>{EDc[0].z, EDc[1].z, EDc[2].z}, r);
    const R bex[3][3] = {{BE[0].x, BE[0].y, BE[0].z}, {BE[1].x, BE[1].y, BE[1].z}, {BE[2].x, BE[2].y, BE[2].z}};
    const R ede[3][3] = {{E0.x, E0.y, E0.z}, {E1.x, E1.y, E1.z}, {E2.x, E2.y, E2.z}};
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j <= i; ++j) I[sym6(i, j)] -= bex[i][j] + bex[j][i] + ede[i][j];
    const R edx[3][3] = {{EDc[0].x, EDc[1].x, EDc[2].x}, {EDc[0].y, EDc[1].y, EDc[2].y}, {EDc[0].z, EDc[1].z, EDc[2].z}};
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) I[sym6(3 + j, i)] += edx[i][j];
}

// Rigid spatial inertia about the COM in world axes: [[R Ib R^T, 0], [0, m 1]].
template <typename R>
__device__ __forceinline__ void body_inertia(const DeviceModel& M, int b, float4 qb, R* I6, float Iw[3][3]) {
    const float4 idiag = M.inertia_diag[b], ioff = M.inertia_off[b];
    const float mass = M.mass_damping[b].x;
    const float3 c0 = qrot(qb, f3(1.0f, 0.0f, 0.0f));
    const float3 c1 = qrot(qb, f3(0.0f, 1.0f, 0.0f));
    const float3 c2 = qrot(qb, f3(0.0f, 0.0f, 1.0f));
    const float Ib[3][3] = {{idiag.x, ioff.x, ioff.y}, {ioff.x, idiag.y, ioff.z}, {ioff.y, ioff.z, idiag.z}};
    const float Rot[3][3] = {{c0.x, c1.x, c2.x}, {c0.y, c1.y, c2.y}, {c0.z, c1.z, c2.z}};
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            float acc = 0.0f;
#pragma unroll
            for (int k = 0; k < 3; ++k)
#pragma unroll
                for (int l2 = 0; l2 < 3; ++l2) acc = fmaf(Rot[i][k] * Ib[k][l2], Rot[j][l2], acc);
            Iw[i][j] = acc;
        }
#pragma unroll
    for (int e = 0; e < 21; ++e) I6[e] = R(0);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
#pragma unroll
        for (int j = 0; j <= i; ++j) I6[sym6(i, j)] = Iw[i][j];
        I6[sym6(3 + i, 3 + i)] = mass;
    }
}

// ---------------------------------------------------------------------------
// Forward kinematics (ArticulatedABA.metal:735-905): lane b computes body b
// at its tree level from its parent's pose and twist, read from the parent
// lane's registers by warp shuffle.  Leaves the pose in shared memory (for
// collision) and the joint axis / origin of the body's DoF in the Jacobian
// table; bias accelerations, offset and subspace stay in registers.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float3 shfl3(float3 a, int src) {
    return f3(__shfl_sync(0xffffffffu, a.x, src), __shfl_sync(0xffffffffu, a.y, src), __shfl_sync(0xffffffffu, a.z, src));
}
__device__ __forceinline__ float4 shfl4(float4 a, int src) {
    return make_float4(__shfl_sync(0xffffffffu, a.x, src), __shfl_sync(0xffffffffu, a.y, src),
                       __shfl_sync(0xffffffffu, a.z, src), __shfl_sync(0xffffffffu, a.w, src));
}

__device__ __forceinline__ float3 shfl3g(float3 a, int src, unsigned mask) {
    return f3(__shfl_sync(mask, a.x, src, 16), __shfl_sync(mask, a.y, src, 16), __shfl_sync(mask, a.z, src, 16));
}

template <typename R>
__device__ void kinematics(const Warp& w, const BodyConst& bc, BodyState<R>& st) {
    const DeviceModel& M = *w.M;
    const DeviceTables& T = *w.T;
    const WarpLayout& L = *w.L;
    float* s = w.s;
    float* misc = s + L.misc;
    const float* q = s + L.q;
    const float* v = s + L.v;
    float* pose = s + L.body_pose;
    float* J = s + L.dof_J;
    const int b = w.lane;
    const bool mine = b < T.nb;
    const int my_depth = mine ? T.depth[b] : -1;
    const int par = (mine && b > 0) ? T.parent[b] : b;

    st.c = f3(0.0f, 0.0f, 0.0f);
    st.qr = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
    st.w = st.v = st.ba = st.bl = st.r = f3(0.0f, 0.0f, 0.0f);
#pragma unroll
    for (int i = 0; i < 6; ++i) st.s[i] = 0.0f;
    if (b == 0 && T.floating) {
        float4 rq;
        const float3 c0 = f3(q[0], q[1], q[2]);
        if (!finite3(c0) || !qnormalize(make_float4(q[3], q[4], q[5], q[6]), rq, true)) {
            set_status(misc, MR_STEP_NONFINITE_INPUT, 0u);
            rq = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
        }
        st.c = c0;
        st.qr = rq;
        st.w = f3(v[3], v[4], v[5]);
        st.v = f3(v[0], v[1], v[2]);
    }
    if (T.floating && b < 6) {
        // Root DoFs: translations along e_k, rotations about the root COM.
        float* Jd = J + b * kJStride;
        const int k = b < 3 ? b : b - 3;
        Jd[0] = k == 0 ? 1.0f : 0.0f;
        Jd[1] = k == 1 ? 1.0f : 0.0f;
        Jd[2] = k == 2 ? 1.0f : 0.0f;
        Jd[3] = q[0]; Jd[4] = q[1]; Jd[5] = q[2];
        Jd[6] = b < 3 ? 1.0f : 0.0f;
    }
    for (int l = 1; l <= T.n_levels; ++l) {
        const float3 cp = shfl3(st.c, par);
        const float4 qp = shfl4(st.qr, par);
        const float3 wp = shfl3(st.w, par);
        const float3 vp = shfl3(st.v, par);
        if (my_depth == l) {
            const float3 axis = xyz(M.axis[b]);
            const float4 pj = qmul(qp, M.parent_rotation[b]);
            float4 motion = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
            float qj = 0.0f, qdj = 0.0f;
            const bool has = bc.dof >= 0;
            const bool prismatic = bc.type == MR_JOINT_PRISMATIC;
            if (has) {
                qj = q[bc.qidx];
                qdj = v[bc.dof];
                if (!prismatic) {
                    float sh, ch;
                    sincosf(0.5f * qj, &sh, &ch);
                    motion = make_float4(axis.x * sh, axis.y * sh, axis.z * sh, ch);
                }
            }
            float4 qb;
            if (!qnormalize(qmul(qmul(pj, motion), M.child_rotation_conj[b]), qb, false)) {
                set_status(misc, MR_STEP_NONFINITE_RESULT, static_cast<unsigned>(b));
                qb = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
            }
            const float3 ja = qrot(pj, axis);
            float3 jp = cp + qrot(qp, xyz(M.parent_anchor[b]));
            if (prismatic) jp = jp + ja * qj;
            const float3 ca = qrot(qb, xyz(M.child_anchor[b]));
            const float3 cb = jp - ca;
            const float3 ptj = jp - cp;
            const float3 zero = f3(0.0f, 0.0f, 0.0f);
            const float3 wb = wp + ((has && !prismatic) ? ja * qdj : zero);
            const float3 vb = vp + cross3(wp, ptj) + (prismatic ? ja * qdj : zero) - cross3(wb, ca);
            const float3 ma = (has && !prismatic) ? ja : zero;
            const float3 ml = prismatic ? ja : (has ? -cross3(ja, ca) : zero);
            st.ba = (has && !prismatic) ? cross3(wp, ja) * qdj : zero;
            const float3 pc = prismatic ? cross3(wp, ja) * (2.0f * qdj) : zero;
            st.bl = cross3(wp, cross3(wp, ptj)) + pc - cross3(st.ba, ca) - cross3(wb, cross3(wb, ca));
            st.c = cb;
            st.qr = qb;
            st.w = wb;
            st.v = vb;
            st.r = cb - cp;
            st.s[0] = ma.x; st.s[1] = ma.y; st.s[2] = ma.z;
            st.s[3] = ml.x; st.s[4] = ml.y; st.s[5] = ml.z;
            if (has) {
                float* Jd = J + bc.dof * kJStride;
                Jd[0] = ja.x; Jd[1] = ja.y; Jd[2] = ja.z;
                Jd[3] = jp.x; Jd[4] = jp.y; Jd[5] = jp.z;
                Jd[6] = prismatic ? 1.0f : 0.0f;
            }
            if (!finite3(cb) || !finite3(wb) || !finite3(vb) || !finite3(st.bl))
                set_status(misc, MR_STEP_NONFINITE_RESULT, static_cast<unsigned>(b));
        }
    }
    if (mine) {
        float* pb = pose + b * kPoseStride;
        st3(pb, st.c);
        st4(pb + 3, st.qr);
    }
    __syncwarp();
}

// ---------------------------------------------------------------------------
// Articulated-body algorithm (ArticulatedABA.metal:905-1440): per-body COM
// frames in world axes, classical accelerations, 21-entry inertias.  Each
// body shifts its articulated inertia and bias into its parent's frame in
// its own registers; the parent pulls its children's contributions by warp
// shuffle in a fixed order, so the sums are deterministic without atomics.
// With `factor` non-null (contact worlds) the body lanes also write their
// rows of the joint-space factor H = L^T L (rows 0-5 of a floating root come
// from the root's 6x6 factorisation): eliminating a DoF's descendants
// leaves its body's articulated inertia, so L_kk = sqrt(D_k) and
// L_kj = U_k . S_j(c_b) / L_kk for the ancestor DoFs j, with S_j moved to
// body b's COM.
// ---------------------------------------------------------------------------
template <typename R>
__device__ bool aba(const Warp& w, const BodyConst& bc, BodyState<R>& st, float* factor) {
    const DeviceModel& M = *w.M;
    const DeviceTables& T = *w.T;
    const WarpLayout& L = *w.L;
    float* s = w.s;
    float* misc = s + L.misc;
    const float* q = s + L.q;
    const float* v = s + L.v;
    const float* tau = s + L.tau;
    float* qdd = s + L.qdd;
    const float* J = s + L.dof_J;
    const int b = w.lane;
    const bool mine = b < T.nb;

    for (int i = b; i < M.nq; i += 32)
        if (!isfinite(q[i])) set_status(misc, MR_STEP_NONFINITE_INPUT, static_cast<unsigned>(i));
    for (int i = b; i < M.nv; i += 32)
        if (!isfinite(v[i]) || !isfinite(tau[i])) set_status(misc, MR_STEP_NONFINITE_INPUT, static_cast<unsigned>(i));
    if (!warp_ok(misc)) return false;

    kinematics(w, bc, st);
    if (!warp_ok(misc)) return false;

    // Rigid inertia and velocity-dependent bias about the COM.
#pragma unroll
    for (int e = 0; e < 21; ++e) st.I[e] = R(0);
#pragma unroll
    for (int e = 0; e < 6; ++e) st.p[e] = 0.0f;
    if (mine) {
        float Iw[3][3];
        body_inertia(M, b, st.qr, st.I, Iw);
        const float3 om = st.w;
        const float3 Iom = f3(Iw[0][0] * om.x + Iw[0][1] * om.y + Iw[0][2] * om.z,
                              Iw[1][0] * om.x + Iw[1][1] * om.y + Iw[1][2] * om.z,
                              Iw[2][0] * om.x + Iw[2][1] * om.y + Iw[2][2] * om.z);
        float3 bt = cross3(om, Iom);
        const float4 md = M.mass_damping[b];
        float3 bf = -(md.x * f3(M.gravity[0], M.gravity[1], M.gravity[2]));
        if (M.apply_damping) {
            bt = bt + md.z * om;
            bf = bf + md.y * st.v;
        }
        st.p[0] = bt.x; st.p[1] = bt.y; st.p[2] = bt.z; st.p[3] = bf.x; st.p[4] = bf.y; st.p[5] = bf.z;
        if (b == 0 && T.floating) {
            for (int k = 0; k < 3; ++k) {
                st.I[sym6(3 + k, 3 + k)] += M.armature_eff[k];
                st.I[sym6(k, k)] += M.armature_eff[3 + k];
                st.p[k] -= tau[3 + k];
                st.p[3 + k] -= tau[k];
            }
        }
    }
    // Backward sweep, deepest level first; the root (level 0) last.  After
    // its level, a body's I and p hold its contribution in its parent's frame.
    const int my_depth = mine ? T.depth[b] : -1;
    const int first_child = mine ? T.child_offsets[b] : 0;
    const int n_children = mine ? T.child_offsets[b + 1] - first_child : 0;
    float3 acc_ang = f3(0.0f, 0.0f, 0.0f), acc_lin = f3(0.0f, 0.0f, 0.0f);
    for (int l = T.n_levels; l >= 0; --l) {
        const bool active = my_depth == l;
        for (int k = 0; k < T.level_children[l]; ++k) {
            const bool take = active && k < n_children;
            const int src = take ? T.children[first_child + k] : b;
#pragma unroll
            for (int e = 0; e < 21; ++e) {
                const R x = __shfl_sync(0xffffffffu, st.I[e], src);
                if (take) st.I[e] += x;
            }
#pragma unroll
            for (int e = 0; e < 6; ++e) {
                const float x = __shfl_sync(0xffffffffu, st.p[e], src);
                if (take) st.p[e] += x;
            }
        }
        if (!active) continue;
        if (l > 0) {
            R prop[6];
            const float cv[6] = {st.ba.x, st.ba.y, st.ba.z, st.bl.x, st.bl.y, st.bl.z};
            sym6_mul(st.I, cv, prop);
#pragma unroll
            for (int e = 0; e < 6; ++e) prop[e] += st.p[e];
            st.D = R(1);
            st.u = R(0);
#pragma unroll
            for (int e = 0; e < 6; ++e) st.U[e] = R(0);
            if (bc.dof >= 0) {
                sym6_mul(st.I, st.s, st.U);
                R D = M.armature_eff[bc.dof];
#pragma unroll
                for (int e = 0; e < 6; ++e) D = fma(static_cast<R>(st.s[e]), st.U[e], D);
                R maxI = R(0);
#pragma unroll
                for (int e = 0; e < 21; ++e) maxI = fmax(maxI, fabs(st.I[e]));
                const R floor = fmax(static_cast<R>(kAbsolutePivotFloor), maxI * R(6) * static_cast<R>(kFloatEps));
                if (!(D > floor) || !isfinite(D)) {
                    set_status(misc, MR_STEP_FACTORIZATION_FAILED, static_cast<unsigned>(bc.dof));
                } else {
                    st.D = D;
                    R u = tau[bc.dof];
#pragma unroll
                    for (int e = 0; e < 6; ++e) u = fma(-static_cast<R>(st.s[e]), prop[e], u);
                    st.u = u;
                    const R invD = R(1) / D;
#pragma unroll
                    for (int e = 0; e < 6; ++e) prop[e] += st.U[e] * (u * invD);
#pragma unroll
                    for (int i = 0; i < 6; ++i)
#pragma unroll
                        for (int j = 0; j <= i; ++j) st.I[sym6(i, j)] -= st.U[i] * st.U[j] * invD;
                }
            }
            shift_inertia(st.I, st.r);
            const float3 pf = f3(static_cast<float>(prop[3]), static_cast<float>(prop[4]), static_cast<float>(prop[5]));
            const float3 pt = f3(static_cast<float>(prop[0]), static_cast<float>(prop[1]), static_cast<float>(prop[2])) +
                              cross3(st.r, pf);
            st.p[0] = pt.x; st.p[1] = pt.y; st.p[2] = pt.z; st.p[3] = pf.x; st.p[4] = pf.y; st.p[5] = pf.z;
        } else if (T.floating) {
            // Root articulated inertia in DoF order (linear x, y, z, then
            // angular x, y, z), factored leaves-first in FP64 in place as
            // H0 = L0^T L0; solves H0 a0 = -pA for the root acceleration.
            R maxI = R(0);
#pragma unroll
            for (int e = 0; e < 21; ++e) maxI = fmax(maxI, fabs(st.I[e]));
            const R floor = fmax(static_cast<R>(kAbsolutePivotFloor), maxI * R(6) * static_cast<R>(kFloatEps));
#define NUMI_ROOT(k, j) st.I[sym6((k) < 3 ? (k) + 3 : (k) - 3, (j) < 3 ? (j) + 3 : (j) - 3)]
            R x[6];
#pragma unroll
            for (int k = 0; k < 6; ++k) x[k] = -static_cast<R>(st.p[k < 3 ? k + 3 : k - 3]);
            bool ok = true;
#pragma unroll
            for (int k = 5; k >= 0; --k) {
                R d = NUMI_ROOT(k, k);
                if (!(d > floor) || !isfinite(d)) {
                    ok = false;
                    d = R(1);
                }
                const R lkk = sqrt(d);
                NUMI_ROOT(k, k) = lkk;
                const R inv = R(1) / lkk;
#pragma unroll
                for (int j = 0; j < k; ++j) NUMI_ROOT(k, j) *= inv;
#pragma unroll
                for (int i = 0; i < k; ++i)
#pragma unroll
                    for (int j = 0; j <= i; ++j) NUMI_ROOT(i, j) -= NUMI_ROOT(k, i) * NUMI_ROOT(k, j);
            }
            // L0^T y = r (descending), then L0 x = y (ascending), in place.
#pragma unroll
            for (int k = 5; k >= 0; --k) {
                R val = x[k];
#pragma unroll
                for (int i = k + 1; i < 6; ++i) val -= NUMI_ROOT(i, k) * x[i];
                x[k] = val / NUMI_ROOT(k, k);
            }
#pragma unroll
            for (int k = 0; k < 6; ++k) {
                R val = x[k];
#pragma unroll
                for (int j = 0; j < k; ++j) val -= NUMI_ROOT(k, j) * x[j];
                x[k] = val / NUMI_ROOT(k, k);
            }
            if (!ok) set_status(misc, MR_STEP_FACTORIZATION_FAILED, 0u);
            if (factor != nullptr) {
#pragma unroll
                for (int k = 0; k < 6; ++k)
#pragma unroll
                    for (int j = 0; j <= k; ++j) factor[sym6(k, j)] = static_cast<float>(NUMI_ROOT(k, j));
            }
#undef NUMI_ROOT
#pragma unroll
            for (int k = 0; k < 6; ++k) qdd[k] = static_cast<float>(x[k]);
            acc_ang = f3(static_cast<float>(x[3]), static_cast<float>(x[4]), static_cast<float>(x[5]));
            acc_lin = f3(static_cast<float>(x[0]), static_cast<float>(x[1]), static_cast<float>(x[2]));
        }
    }
    if (!warp_ok(misc)) return false;

    // Joint rows of the factor.
    if (factor != nullptr && mine && b > 0 && bc.dof >= 0) {
        const int k = bc.dof;
        float* rowk = factor + k * (k + 1) / 2;
        const R lkk = sqrt(st.D);
        const R inv = R(1) / lkk;
        rowk[k] = static_cast<float>(lkk);
        const int na = T.dof_depth[k];
        for (int t = 0; t < na; ++t) {
            const int j = T.anc[b][t];
            const float* jd = J + j * kJStride;
            const float3 ax = f3(jd[0], jd[1], jd[2]);
            R val;
            if (jd[6] != 0.0f) {
                val = st.U[3] * ax.x + st.U[4] * ax.y + st.U[5] * ax.z;
            } else {
                const float3 lin = cross3(ax, st.c - f3(jd[3], jd[4], jd[5]));
                val = st.U[0] * ax.x + st.U[1] * ax.y + st.U[2] * ax.z + st.U[3] * lin.x + st.U[4] * lin.y + st.U[5] * lin.z;
            }
            rowk[j] = static_cast<float>(val * inv);
        }
    }

    // Forward acceleration sweep: the parent's acceleration by shuffle.
    const int par = (mine && b > 0) ? T.parent[b] : b;
    for (int l = 1; l <= T.n_levels; ++l) {
        const float3 pa = shfl3(acc_ang, par);
        const float3 plin = shfl3(acc_lin, par);
        if (my_depth == l) {
            const float3 pl = plin + cross3(pa, st.r);
            float3 ang = pa + st.ba;
            float3 lin = pl + st.bl;
            if (bc.dof >= 0) {
                const R proj = st.U[0] * pa.x + st.U[1] * pa.y + st.U[2] * pa.z + st.U[3] * pl.x + st.U[4] * pl.y + st.U[5] * pl.z;
                const float acc = static_cast<float>((st.u - proj) / st.D);
                qdd[bc.dof] = acc;
                ang = ang + f3(st.s[0], st.s[1], st.s[2]) * acc;
                lin = lin + f3(st.s[3], st.s[4], st.s[5]) * acc;
            }
            acc_ang = ang;
            acc_lin = lin;
        }
    }
    __syncwarp();
    // v_free = v + h qdd.
    float* vf = s + L.vf;
    for (int d = b; d < M.nv; d += 32) {
        const float a = qdd[d];
        const float nvv = v[d] + M.h * a;
        if (!isfinite(a) || !isfinite(nvv)) set_status(misc, MR_STEP_NONFINITE_RESULT, static_cast<unsigned>(d));
        vf[d] = nvv;
    }
    return warp_ok(misc);
}

// Free-motion commit of the ABA candidate (ArticulatedABA.metal:1466-1540):
// v' = v_free, joints q' = q + h v', root exponential map with the angle
// reduced modulo 2 pi.  kComp: joint and root positions as compensated sums.
template <bool kComp>
__device__ bool integrate_free(const Warp& w) {
    const DeviceModel& M = *w.M;
    const WarpLayout& L = *w.L;
    float* s = w.s;
    float* misc = s + L.misc;
    float* q = s + L.q;
    float* v = s + L.v;
    float* qc = s + L.qcomp;
    const float* vf = s + L.vf;
    for (int d = w.lane; d < M.nv; d += 32) {
        v[d] = vf[d];
        const int qi = M.dof_q[d];
        if (qi >= 0 && !(M.floating && d < 6)) {
            const float nq = kComp ? kahan_madd(q[qi], M.h, vf[d], qc[qi]) : q[qi] + M.h * vf[d];
            if (!isfinite(nq)) set_status(misc, MR_STEP_NONFINITE_RESULT, static_cast<unsigned>(qi));
            q[qi] = nq;
        }
    }
    if (M.floating && w.lane == 0) {
        if (kComp) {
            for (int i = 0; i < 3; ++i) q[i] = kahan_madd(q[i], M.h, vf[i], qc[i]);
        } else {
            q[0] += M.h * vf[0];
            q[1] += M.h * vf[1];
            q[2] += M.h * vf[2];
        }
        const float4 inc = so3_increment(M.h * f3(vf[3], vf[4], vf[5]), true);
        float4 out;
        if (!qnormalize(qmul(inc, make_float4(q[3], q[4], q[5], q[6])), out, false)) {
            set_status(misc, MR_STEP_NONFINITE_RESULT, 3u);
        } else {
            q[3] = out.x; q[4] = out.y; q[5] = out.z; q[6] = out.w;
        }
        if (!isfinite(q[0]) || !isfinite(q[1]) || !isfinite(q[2])) set_status(misc, MR_STEP_NONFINITE_RESULT, 0u);
    }
    return warp_ok(misc);
}

// ---------------------------------------------------------------------------
// Collision: collider projection, plane pair flag, analytic plane witnesses
// and persistent manifolds (Collision.metal:380-1000, 4379-4830, 5115-5560,
// 5712-6030, 9557-9830).  One lane owns one compiled pair.
// ---------------------------------------------------------------------------
struct ShapeWorld {
    int type;
    float3 center;
    float4 rot;
    float3 body_pos;
    float4 body_rot;      // normalised body quaternion
    float3 lower, upper;  // swept, inflated bounds (finite shapes)
    float3 half;          // box half extents
    float radius, half_length;
    float3 ep0, ep1;
    float offset;         // contact offset including the speculative margin
    float3 normal;        // plane normal
};

__device__ void make_shape(const DeviceModel& M, const float* pose, int sh, float margin, ShapeWorld& o) {
    o.type = M.shape_type[sh];
    const int b = M.shape_body[sh];
    const float4 lp = M.shape_position[sh];
    const float4 lr = M.shape_rotation[sh];
    if (b >= 0) {
        o.body_pos = ld3(pose + b * kPoseStride);
        o.body_rot = ld4(pose + b * kPoseStride + 3);
        o.center = o.body_pos + qrot(o.body_rot, xyz(lp));
        o.rot = qmul(o.body_rot, lr);
    } else {
        o.body_pos = xyz(M.static_body_position[sh]);
        o.body_rot = M.static_body_rotation[sh];
        o.center = xyz(lp);
        o.rot = lr;
    }
    const float4 dims = M.shape_dims[sh];
    const float base_offset = M.shape_offsets[sh].x;
    o.offset = base_offset + margin;
    o.half = f3(0.0f, 0.0f, 0.0f);
    o.radius = 0.0f;
    o.half_length = 0.0f;
    o.ep0 = o.ep1 = f3(0.0f, 0.0f, 0.0f);
    o.lower = o.upper = f3(0.0f, 0.0f, 0.0f);
    o.normal = f3(0.0f, 0.0f, 0.0f);
    if (o.type == MR_SHAPE_PLANE) {
        const float3 n = qrot(o.rot, f3(0.0f, 1.0f, 0.0f));
        o.normal = n * rsqrtf(dot3(n, n));
        return;
    }
    float3 ext;
    if (o.type == MR_SHAPE_SPHERE) {
        o.radius = dims.x;
        const float e = o.radius + base_offset;
        ext = f3(e, e, e);
        o.lower = o.center - ext;
        o.upper = o.center + ext;
    } else if (o.type == MR_SHAPE_CAPSULE) {
        o.radius = dims.x;
        o.half_length = dims.y;
        const float3 ax = qrot(o.rot, f3(0.0f, dims.y, 0.0f));
        o.ep0 = o.center - ax;
        o.ep1 = o.center + ax;
        const float e = o.radius + base_offset;
        o.lower = f3(fminf(o.ep0.x, o.ep1.x), fminf(o.ep0.y, o.ep1.y), fminf(o.ep0.z, o.ep1.z)) - f3(e, e, e);
        o.upper = f3(fmaxf(o.ep0.x, o.ep1.x), fmaxf(o.ep0.y, o.ep1.y), fmaxf(o.ep0.z, o.ep1.z)) + f3(e, e, e);
    } else {  // box
        o.half = xyz(dims);
        const float3 bx = qrot(o.rot, f3(1.0f, 0.0f, 0.0f));
        const float3 by = qrot(o.rot, f3(0.0f, 1.0f, 0.0f));
        const float3 bz = qrot(o.rot, f3(0.0f, 0.0f, 1.0f));
        ext = f3(fabsf(bx.x), fabsf(bx.y), fabsf(bx.z)) * o.half.x + f3(fabsf(by.x), fabsf(by.y), fabsf(by.z)) * o.half.y +
              f3(fabsf(bz.x), fabsf(bz.y), fabsf(bz.z)) * o.half.z + f3(base_offset, base_offset, base_offset);
        o.lower = o.center - ext;
        o.upper = o.center + ext;
    }
    // Conservative inflation (inflateFiniteBounds), then the speculative sweep.
    const float3 sc = f3(fmaxf(fabsf(o.lower.x), fabsf(o.upper.x)) + 1.0f, fmaxf(fabsf(o.lower.y), fabsf(o.upper.y)) + 1.0f,
                         fmaxf(fabsf(o.lower.z), fabsf(o.upper.z)) + 1.0f);
    o.lower = o.lower - sc * kAabbPad - f3(margin, margin, margin);
    o.upper = o.upper + sc * kAabbPad + f3(margin, margin, margin);
}

__device__ __forceinline__ float shape_scale(const ShapeWorld& s) {
    return fmaxf(fmaxf(fmaxf(maxabs3(s.center), maxabs3(s.half)), fmaxf(maxabs3(s.ep0), maxabs3(s.ep1))),
                 fmaxf(fmaxf(fabsf(s.radius), fabsf(s.half_length)),
                       fmaxf(fabsf(s.offset), fmaxf(maxabs3(s.lower), maxabs3(s.upper)))));
}

// Narrowphase candidate record in shared-memory scratch (16 words): local
// anchors on A and B, feature ids, world midpoint, separation, lifetime and
// accumulated impulse.  Records 0-3 are the kept points of the old manifold,
// records 4.. the raw contacts of this substep.
enum CandidateWord : int {
    kCdLa = 0, kCdLb = 3, kCdFa = 6, kCdFb = 7, kCdWp = 8, kCdSep = 11, kCdLife = 12, kCdImp = 13
};
// A candidate is one byte: low nibble = record that holds its geometry,
// high nibble = old record it inherits lifetime and impulse from (15: new).
constexpr unsigned kFresh = 15u;

__device__ __forceinline__ unsigned long long record_key(const float* rec) {
    return (static_cast<unsigned long long>(static_cast<unsigned>(as_int(rec[kCdFa]))) << 32) |
           static_cast<unsigned>(as_int(rec[kCdFb]));
}

// Builds the new persistent manifold of one pair into `slot` (in/out), using
// `scratch` (pair_scratch_words of the pair class) for its candidates.
// Returns the number of points, or -1 on a non-finite / overflow failure.
// Plane pair classes only: every raw contact shares the plane normal.
__device__ int pair_manifold(const DeviceModel& M, const float* pose, const float* margins, int pair, float* slot,
                             float* scratch, int& raw_count_out, bool& candidate_out) {
    raw_count_out = 0;
    candidate_out = false;
    const int sa = M.pair_a[pair];
    const int sb = M.pair_b[pair];
    ShapeWorld A, B;
    make_shape(M, pose, sa, margins[sa], A);
    make_shape(M, pose, sb, margins[sb], B);
    const bool a_plane = A.type == MR_SHAPE_PLANE;
    const ShapeWorld& plane = a_plane ? A : B;
    const ShapeWorld& fin = a_plane ? B : A;
    // Pair flag (projectedPairMayOverlap, plane branch).
    {
        const float3 center = 0.5f * (fin.lower + fin.upper);
        const float3 halfx = 0.5f * (fin.upper - fin.lower);
        const float scale = fmaxf(fmaxf(maxabs3(plane.center), maxabs3(fin.lower)),
                                  fmaxf(maxabs3(fin.upper), fmaxf(fabsf(plane.offset), fabsf(fin.offset))));
        const float qpad = (scale + 1.0f) * kQueryPad;
        const float3 an = f3(fabsf(plane.normal.x), fabsf(plane.normal.y), fabsf(plane.normal.z));
        const float msd = dot3(plane.normal, center - plane.center) - dot3(an, halfx);
        if (!(msd <= plane.offset + qpad)) {
            slot[7] = as_float(0);
            return 0;
        }
    }
    candidate_out = true;
    const float accepted = A.offset + B.offset + (fmaxf(shape_scale(A), shape_scale(B)) + 1.0f) * kQueryPad;
    const float3 posA = A.body_pos, posB = B.body_pos;
    const float4 rotA = A.body_rot, rotB = B.body_rot;
    const unsigned plane_feature = feature_key(MR_SHAPE_PLANE, 0u);
    const float3 raw_normal = a_plane ? plane.normal : -plane.normal;
    float* raw = scratch + 4 * kCandidateWords;
    int nraw = 0;
    bool finite = true;
    // Raw contact: surface point of the finite shape, its projection on the
    // plane, normal A -> B (Collision.metal:4379-4830, plane witnesses).
    auto append = [&](float3 surface, float sep, unsigned ffeat) {
        const float3 pp = surface - plane.normal * sep;
        const float3 pa = a_plane ? pp : surface;
        const float3 pb = a_plane ? surface : pp;
        float* rec = raw + nraw * kCandidateWords;
        const float3 la = qrotinv(rotA, pa - posA);
        const float3 lb = qrotinv(rotB, pb - posB);
        st3(rec + kCdLa, la);
        st3(rec + kCdLb, lb);
        rec[kCdFa] = as_float(static_cast<int>(a_plane ? plane_feature : ffeat));
        rec[kCdFb] = as_float(static_cast<int>(a_plane ? ffeat : plane_feature));
        st3(rec + kCdWp, 0.5f * (pa + pb));
        rec[kCdSep] = sep;
        finite = finite && isfinite(sep) && finite3(pa) && finite3(pb);
        ++nraw;
    };
    const int cls = M.pair_class[pair];
    if (cls == MR_COLLISION_PAIR_SPHERE_PLANE) {
        const float3 surface = fin.center - plane.normal * fin.radius;
        const float sep = dot3(plane.normal, surface - plane.center);
        if (sep <= accepted) append(surface, sep, feature_key(MR_SHAPE_SPHERE, 0u));
    } else if (cls == MR_COLLISION_PAIR_CAPSULE_PLANE) {
        for (int e = 0; e < 2; ++e) {
            const float3 surface = (e == 0 ? fin.ep0 : fin.ep1) - plane.normal * fin.radius;
            const float sep = dot3(plane.normal, surface - plane.center);
            if (sep <= accepted) append(surface, sep, feature_key(MR_SHAPE_CAPSULE, static_cast<unsigned>(e)));
        }
    } else if (cls == MR_COLLISION_PAIR_BOX_PLANE) {
        for (unsigned vtx = 0; vtx < 8u; ++vtx) {
            const float3 local = f3((vtx & 1u) ? fin.half.x : -fin.half.x, (vtx & 2u) ? fin.half.y : -fin.half.y,
                                    (vtx & 4u) ? fin.half.z : -fin.half.z);
            const float3 wpt = fin.center + qrot(fin.rot, local);
            const float sep = dot3(plane.normal, wpt - plane.center);
            if (sep <= accepted) append(wpt, sep, feature_key(MR_SHAPE_BOX, vtx));
        }
    }
    raw_count_out = nraw;
    if (nraw == 0) {
        slot[7] = as_float(0);
        return 0;
    }
    if (!finite || !finite3(raw_normal)) return -1;

    // buildPersistentWorldManifold (Collision.metal:5290-5560,
    // Collision.cpp:2546-2760).
    float3 nw = raw_normal * (1.0f / len3(raw_normal));
    if (!finite3(nw) || dot3(nw, nw) < 0.9999f) return -1;
    const float4 thr = make_float4(M.manifold_thresholds[0], M.manifold_thresholds[1], M.manifold_thresholds[2],
                                   M.manifold_thresholds[3]);
    unsigned char* ids = reinterpret_cast<unsigned char*>(scratch + (4 + pair_max_raw(cls)) * kCandidateWords);
    int nc = 0;
    bool old_ok = false;
    float3 transported = f3(0.0f, 0.0f, 0.0f);
    float old_age = 0.0f;
    const int old_count = as_int(slot[7]);
    if (old_count > 0 && old_count <= kManifoldPoints) {
        float3 on = qrot(rotA, ld3(slot));
        on = on * (1.0f / len3(on));
        old_ok = finite3(on) && dot3(on, nw) >= thr.w;
        if (old_ok) {
            const float3 ot = qrot(rotA, ld3(slot + 4));
            transported = ot - nw * dot3(ot, nw);
            old_age = slot[3];
            for (int i = 0; i < old_count; ++i) {
                const float* op = slot + 8 + i * 12;
                const float3 pa = posA + qrot(rotA, ld3(op));
                const float3 pb = posB + qrot(rotB, ld3(op + 3));
                const float3 delta = pb - pa;
                const float sep = dot3(delta, nw);
                const float3 tan = delta - nw * sep;
                if (sep > thr.x || len3(tan) > thr.y) continue;
                float* rec = scratch + i * kCandidateWords;
#pragma unroll
                for (int k = 0; k < 8; ++k) rec[k] = op[k];  // anchors and feature ids
                const unsigned life = static_cast<unsigned>(as_int(op[8]));
                rec[kCdLife] = as_float(static_cast<int>(life == 0xffffffffu ? 0xffffffffu : life + 1u));
                rec[kCdImp + 0] = op[9];
                rec[kCdImp + 1] = op[10];
                rec[kCdImp + 2] = op[11];
                st3(rec + kCdWp, 0.5f * (pa + pb));
                rec[kCdSep] = sep;
                ids[nc++] = static_cast<unsigned char>((i << 4) | i);
            }
        }
    }
    // Raw contacts refresh a candidate with the same features, else one
    // within the merge distance, else join as new points.
    const float merge2 = thr.z * thr.z;
    for (int r = 0; r < nraw; ++r) {
        const float* rr = raw + r * kCandidateWords;
        const float3 la = ld3(rr + kCdLa), lb = ld3(rr + kCdLb);
        const int fa = as_int(rr[kCdFa]), fb = as_int(rr[kCdFb]);
        int match = -1;
        for (int k = 0; k < nc; ++k) {
            const float* g = scratch + (ids[k] & 15u) * kCandidateWords;
            if (as_int(g[kCdFa]) == fa && as_int(g[kCdFb]) == fb) { match = k; break; }
        }
        if (match < 0) {
            for (int k = 0; k < nc; ++k) {
                const float* g = scratch + (ids[k] & 15u) * kCandidateWords;
                const float3 da = ld3(g + kCdLa) - la;
                const float3 db = ld3(g + kCdLb) - lb;
                if (dot3(da, da) + dot3(db, db) <= 2.0f * merge2) { match = k; break; }
            }
        }
        if (match < 0) {
            if (nc >= 4 + kMaxRawPerPair) return -1;
            ids[nc++] = static_cast<unsigned char>((kFresh << 4) | (4u + r));
        } else {
            ids[match] = static_cast<unsigned char>((ids[match] & 0xf0u) | (4u + r));
        }
    }
    // reduceCandidates.  With at most four candidates the separation order
    // cannot change the result (the final order is canonical by feature), so
    // the separation sort and the reduction run only for larger sets.
    if (nc > kManifoldPoints) {
        for (int i = 1; i < nc; ++i) {
            const unsigned char val = ids[i];
            const float* gv = scratch + (val & 15u) * kCandidateWords;
            const float sv = gv[kCdSep];
            const unsigned long long kv = record_key(gv);
            int d = i;
            while (d > 0) {
                const float* gp = scratch + (ids[d - 1] & 15u) * kCandidateWords;
                const float sp = gp[kCdSep];
                if (!(sv < sp || (sv == sp && kv < record_key(gp)))) break;
                ids[d] = ids[d - 1];
                --d;
            }
            ids[d] = val;
        }
        // Greedy selection: deepest, farthest in the tangent plane, largest
        // area, then largest minimum distance.  Box faces make exact ties
        // structural (parallel edges give equal distances and areas), so
        // scores within a relative 1e-5 count as tied and go to the smaller
        // feature key: the choice no longer depends on FP32 rounding.  The
        // reference compares with absolute tolerances below the rounding of
        // these scores (Collision.metal:5247, Collision.cpp:2531-2544).
        unsigned selected = 1u;
        unsigned chosen = 0u;  // candidate indices, one byte each
        int chosen_count = 1;
        const float3 w0 = ld3(scratch + (ids[0] & 15u) * kCandidateWords + kCdWp);
        float3 w1 = w0;
        for (int stage = 1; stage < kManifoldPoints; ++stage) {
            int best = -1;
            float best_score = -1.0f;
            unsigned long long best_feature = ~0ull;
            for (int i = 0; i < nc; ++i) {
                if (selected & (1u << i)) continue;
                const float* gi = scratch + (ids[i] & 15u) * kCandidateWords;
                const float3 wi = ld3(gi + kCdWp);
                float score;
                if (stage == 1) {
                    const float3 dl = wi - w0;
                    const float3 t = dl - nw * dot3(dl, nw);
                    score = dot3(t, t);
                } else if (stage == 2) {
                    score = fabsf(dot3(cross3(w1 - w0, wi - w0), nw));
                } else {
                    score = INFINITY;
                    for (int k = 0; k < chosen_count; ++k) {
                        const int ck = static_cast<int>((chosen >> (8 * k)) & 0xffu);
                        const float3 dl = wi - ld3(scratch + (ids[ck] & 15u) * kCandidateWords + kCdWp);
                        const float3 t = dl - nw * dot3(dl, nw);
                        score = fminf(score, dot3(t, t));
                    }
                }
                const unsigned long long f = record_key(gi);
                const float tol = fmaxf(kTieAbsolute, kTieRelative * fmaxf(fabsf(score), fabsf(best_score)));
                if (score > best_score + tol || (fabsf(score - best_score) <= tol && f < best_feature)) {
                    best = i;
                    best_score = score;
                    best_feature = f;
                }
            }
            if (best >= 0) {
                chosen |= static_cast<unsigned>(best) << (8 * chosen_count);
                ++chosen_count;
                selected |= 1u << best;
                if (stage == 1) w1 = ld3(scratch + (ids[best] & 15u) * kCandidateWords + kCdWp);
            }
        }
        unsigned packed = 0u;
        for (int k = 0; k < chosen_count; ++k) packed |= static_cast<unsigned>(ids[(chosen >> (8 * k)) & 0xffu]) << (8 * k);
        for (int k = 0; k < chosen_count; ++k) ids[k] = static_cast<unsigned char>((packed >> (8 * k)) & 0xffu);
        nc = chosen_count;
    }
    // Canonical order by feature pair.
    for (int i = 1; i < nc; ++i) {
        const unsigned char val = ids[i];
        const unsigned long long f = record_key(scratch + (val & 15u) * kCandidateWords);
        int d = i;
        while (d > 0 && f < record_key(scratch + (ids[d - 1] & 15u) * kCandidateWords)) {
            ids[d] = ids[d - 1];
            --d;
        }
        ids[d] = val;
    }
    float3 tw = transported;
    if (!old_ok || !finite3(tw) || dot3(tw, tw) <= 1.0e-12f) tw = stable_tangent(nw);
    else tw = tw * (1.0f / len3(tw));
    st3(slot, qrotinv(rotA, nw));
    slot[3] = old_ok ? fminf(old_age + 1.0f, 65535.0f) : 0.0f;
    st3(slot + 4, qrotinv(rotA, tw));
    slot[7] = as_float(nc);
    for (int i = 0; i < kManifoldPoints; ++i) {
        float* op = slot + 8 + i * 12;
        if (i < nc) {
            const unsigned id = ids[i];
            const float* g = scratch + (id & 15u) * kCandidateWords;
#pragma unroll
            for (int k = 0; k < 8; ++k) op[k] = g[k];
            if ((id >> 4) == kFresh) {
                op[8] = as_float(0);
                op[9] = op[10] = op[11] = 0.0f;
            } else {
                const float* hrec = scratch + (id >> 4) * kCandidateWords;
                op[8] = hrec[kCdLife];
                op[9] = hrec[kCdImp + 0];
                op[10] = hrec[kCdImp + 1];
                op[11] = hrec[kCdImp + 2];
            }
        } else {
#pragma unroll
            for (int k = 0; k < 12; ++k) op[k] = 0.0f;
        }
    }
    return nc;
}

// Heavy pair classes (more than two raw contacts: box vs plane) are built by
// a 16-lane group: lanes compute the raw witnesses (one feature each), the
// kept old points, the match tests and the reduction scores in parallel,
// and every sequential decision of the reference algorithm (match order,
// greedy reduction scan, canonical order) is taken uniformly by the group
// from shuffled values, so the result equals the one-lane build
// (pair_manifold) decision for decision.  `sl` is the lane in the group,
// `gbase` the group's first lane in the warp.
__device__ __forceinline__ unsigned group_ballot(unsigned gmask, int gbase, bool pred) {
    return (__ballot_sync(gmask, pred) >> gbase) & 0xffffu;
}

__device__ void group_manifold(const DeviceModel& M, const float* pose, const float* margins, int pair, float* slot,
                               float* scratch, int sl, int gbase, unsigned gmask, int& npoints_out, int& nraw_out,
                               bool& cand_out, bool& fail_out) {
    npoints_out = 0;
    nraw_out = 0;
    cand_out = false;
    fail_out = false;
    const int sa = M.pair_a[pair];
    const int sb = M.pair_b[pair];
    ShapeWorld A, B;
    make_shape(M, pose, sa, margins[sa], A);
    make_shape(M, pose, sb, margins[sb], B);
    const bool a_plane = A.type == MR_SHAPE_PLANE;
    const ShapeWorld& plane = a_plane ? A : B;
    const ShapeWorld& fin = a_plane ? B : A;
    {
        const float3 center = 0.5f * (fin.lower + fin.upper);
        const float3 halfx = 0.5f * (fin.upper - fin.lower);
        const float scale = fmaxf(fmaxf(maxabs3(plane.center), maxabs3(fin.lower)),
                                  fmaxf(maxabs3(fin.upper), fmaxf(fabsf(plane.offset), fabsf(fin.offset))));
        const float qpad = (scale + 1.0f) * kQueryPad;
        const float3 an = f3(fabsf(plane.normal.x), fabsf(plane.normal.y), fabsf(plane.normal.z));
        const float msd = dot3(plane.normal, center - plane.center) - dot3(an, halfx);
        if (!(msd <= plane.offset + qpad)) {
            if (sl == 0) slot[7] = as_float(0);
            __syncwarp(gmask);
            return;
        }
    }
    cand_out = true;
    const float accepted = A.offset + B.offset + (fmaxf(shape_scale(A), shape_scale(B)) + 1.0f) * kQueryPad;
    const float3 posA = A.body_pos, posB = B.body_pos;
    const float4 rotA = A.body_rot, rotB = B.body_rot;
    const unsigned plane_feature = feature_key(MR_SHAPE_PLANE, 0u);
    const float3 raw_normal = a_plane ? plane.normal : -plane.normal;
    float* raw = scratch + 4 * kCandidateWords;
    const int cls = M.pair_class[pair];

    // Raw witnesses, one feature per lane; record r holds feature r.
    bool racc = false, rbad = false;
    if (sl < pair_max_raw(cls)) {
        float3 surface = f3(0.0f, 0.0f, 0.0f);
        unsigned ffeat = 0u;
        if (cls == MR_COLLISION_PAIR_BOX_PLANE) {
            const unsigned vtx = static_cast<unsigned>(sl);
            const float3 local = f3((vtx & 1u) ? fin.half.x : -fin.half.x, (vtx & 2u) ? fin.half.y : -fin.half.y,
                                    (vtx & 4u) ? fin.half.z : -fin.half.z);
            surface = fin.center + qrot(fin.rot, local);
            ffeat = feature_key(MR_SHAPE_BOX, vtx);
        } else if (cls == MR_COLLISION_PAIR_CAPSULE_PLANE) {
            surface = (sl == 0 ? fin.ep0 : fin.ep1) - plane.normal * fin.radius;
            ffeat = feature_key(MR_SHAPE_CAPSULE, static_cast<unsigned>(sl));
        } else {
            surface = fin.center - plane.normal * fin.radius;
            ffeat = feature_key(MR_SHAPE_SPHERE, 0u);
        }
        const float sep = dot3(plane.normal, surface - plane.center);
        racc = sep <= accepted;
        if (racc) {
            const float3 pp = surface - plane.normal * sep;
            const float3 pa = a_plane ? pp : surface;
            const float3 pb = a_plane ? surface : pp;
            float* rec = raw + sl * kCandidateWords;
            st3(rec + kCdLa, qrotinv(rotA, pa - posA));
            st3(rec + kCdLb, qrotinv(rotB, pb - posB));
            rec[kCdFa] = as_float(static_cast<int>(a_plane ? plane_feature : ffeat));
            rec[kCdFb] = as_float(static_cast<int>(a_plane ? ffeat : plane_feature));
            st3(rec + kCdWp, 0.5f * (pa + pb));
            rec[kCdSep] = sep;
            rbad = !(isfinite(sep) && finite3(pa) && finite3(pb));
        }
    }
    const unsigned raw_mask = group_ballot(gmask, gbase, racc);
    const bool any_bad = group_ballot(gmask, gbase, rbad) != 0u;
    nraw_out = __popc(raw_mask);
    if (raw_mask == 0u) {
        if (sl == 0) slot[7] = as_float(0);
        __syncwarp(gmask);
        return;
    }
    if (any_bad || !finite3(raw_normal)) {
        fail_out = true;
        return;
    }
    const float3 nw = raw_normal * (1.0f / len3(raw_normal));
    if (!finite3(nw) || dot3(nw, nw) < 0.9999f) {
        fail_out = true;
        return;
    }
    const float4 thr = make_float4(M.manifold_thresholds[0], M.manifold_thresholds[1], M.manifold_thresholds[2],
                                   M.manifold_thresholds[3]);
    // Old manifold: lanes 8-11 test and copy the old points.
    bool old_ok = false;
    float3 transported = f3(0.0f, 0.0f, 0.0f);
    float old_age = 0.0f;
    const int old_count = as_int(slot[7]);
    if (old_count > 0 && old_count <= kManifoldPoints) {
        float3 on = qrot(rotA, ld3(slot));
        on = on * (1.0f / len3(on));
        old_ok = finite3(on) && dot3(on, nw) >= thr.w;
        if (old_ok) {
            const float3 ot = qrot(rotA, ld3(slot + 4));
            transported = ot - nw * dot3(ot, nw);
            old_age = slot[3];
        }
    }
    bool keep = false;
    const int oi = sl - 8;
    if (old_ok && oi >= 0 && oi < old_count) {
        const float* op = slot + 8 + oi * 12;
        const float3 pa = posA + qrot(rotA, ld3(op));
        const float3 pb = posB + qrot(rotB, ld3(op + 3));
        const float3 delta = pb - pa;
        const float sep = dot3(delta, nw);
        const float3 tan = delta - nw * sep;
        keep = !(sep > thr.x || len3(tan) > thr.y);
        if (keep) {
            float* rec = scratch + oi * kCandidateWords;
#pragma unroll
            for (int k = 0; k < 8; ++k) rec[k] = op[k];
            const unsigned life = static_cast<unsigned>(as_int(op[8]));
            rec[kCdLife] = as_float(static_cast<int>(life == 0xffffffffu ? 0xffffffffu : life + 1u));
            rec[kCdImp + 0] = op[9];
            rec[kCdImp + 1] = op[10];
            rec[kCdImp + 2] = op[11];
            st3(rec + kCdWp, 0.5f * (pa + pb));
            rec[kCdSep] = sep;
        }
    }
    const unsigned kept_mask = (group_ballot(gmask, gbase, keep) >> 8) & 0xfu;
    __syncwarp(gmask);

    // Candidate list: lane k holds candidate k's id (geometry record in the
    // low nibble, inherited old record in the high nibble).
    int nc = __popc(kept_mask);
    unsigned my_id = 0xffu;
    {
        unsigned m = kept_mask;
        for (int k = 0; k < sl && m != 0u; ++k) m &= m - 1u;
        if (sl < nc) {
            const unsigned i = static_cast<unsigned>(__ffs(m) - 1);
            my_id = (i << 4) | i;
        }
    }
    // Raw contacts in feature order refresh the first candidate with the
    // same features, else the first within the merge distance, else join.
    const float merge2 = thr.z * thr.z;
    for (unsigned m = raw_mask; m != 0u; m &= m - 1u) {
        const int r = __ffs(m) - 1;
        const float* rr = raw + r * kCandidateWords;
        const float3 la = ld3(rr + kCdLa), lb = ld3(rr + kCdLb);
        const int fa = as_int(rr[kCdFa]), fb = as_int(rr[kCdFb]);
        bool feat = false, prox = false;
        if (sl < nc) {
            const float* g = scratch + (my_id & 15u) * kCandidateWords;
            feat = as_int(g[kCdFa]) == fa && as_int(g[kCdFb]) == fb;
            const float3 da = ld3(g + kCdLa) - la;
            const float3 db = ld3(g + kCdLb) - lb;
            prox = dot3(da, da) + dot3(db, db) <= 2.0f * merge2;
        }
        const unsigned fm = group_ballot(gmask, gbase, feat);
        const unsigned pm = group_ballot(gmask, gbase, prox);
        const int match = fm != 0u ? __ffs(fm) - 1 : (pm != 0u ? __ffs(pm) - 1 : -1);
        if (match < 0) {
            if (sl == nc) my_id = (kFresh << 4) | (4u + static_cast<unsigned>(r));
            ++nc;
        } else if (sl == match) {
            my_id = (my_id & 0xf0u) | (4u + static_cast<unsigned>(r));
        }
    }
    // Per-candidate geometry for the ordering and the scores.
    float my_sep = 0.0f;
    unsigned my_fa = 0xffffffffu, my_fb = 0xffffffffu;
    float3 my_wp = f3(0.0f, 0.0f, 0.0f);
    if (sl < nc) {
        const float* g = scratch + (my_id & 15u) * kCandidateWords;
        my_sep = g[kCdSep];
        my_fa = static_cast<unsigned>(as_int(g[kCdFa]));
        my_fb = static_cast<unsigned>(as_int(g[kCdFb]));
        my_wp = ld3(g + kCdWp);
    }
    // Final candidate lanes in canonical (feature) order, 4 bits each.
    unsigned long long final_order = 0ull;
    int nfinal = 0;
    if (nc > kManifoldPoints) {
        // reduceCandidates: order by (separation, features), then greedy
        // selection with the precision-independent tie rule of pair_manifold.
        int rank = 0;
#pragma unroll
        for (int j = 0; j < kMaxCandidates; ++j) {
            const float sj = __shfl_sync(gmask, my_sep, j, 16);
            const unsigned fj = __shfl_sync(gmask, my_fa, j, 16);
            const unsigned gj = __shfl_sync(gmask, my_fb, j, 16);
            if (j < nc && sl < nc && j != sl) {
                const bool less = sj < my_sep || (sj == my_sep && (fj < my_fa || (fj == my_fa && gj < my_fb)));
                rank += less ? 1 : 0;
            }
        }
        unsigned long long order = 0ull;  // candidate lane of each rank
#pragma unroll
        for (int i = 0; i < kMaxCandidates; ++i) {
            const unsigned who = group_ballot(gmask, gbase, sl < nc && rank == i);
            if (i < nc) order |= static_cast<unsigned long long>(__ffs(who) - 1) << (4 * i);
        }
        const int c0 = static_cast<int>(order & 0xfull);
        unsigned selected = 1u << c0;
        unsigned long long chosen = static_cast<unsigned long long>(c0);
        int chosen_count = 1;
        const float3 w0 = shfl3g(my_wp, c0, gmask);
        float3 w1 = w0, w2 = w0;
        for (int stage = 1; stage < kManifoldPoints; ++stage) {
            float score;
            if (stage == 1) {
                const float3 dl = my_wp - w0;
                const float3 t = dl - nw * dot3(dl, nw);
                score = dot3(t, t);
            } else if (stage == 2) {
                score = fabsf(dot3(cross3(w1 - w0, my_wp - w0), nw));
            } else {
                score = INFINITY;
                const float3 ws[3] = {w0, w1, w2};
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const float3 dl = my_wp - ws[k];
                    const float3 t = dl - nw * dot3(dl, nw);
                    score = fminf(score, dot3(t, t));
                }
            }
            int best = -1;
            float best_score = -1.0f;
            unsigned long long best_feature = ~0ull;
#pragma unroll
            for (int i = 0; i < kMaxCandidates; ++i) {
                const int k = static_cast<int>((order >> (4 * i)) & 0xfull);
                const float sc = __shfl_sync(gmask, score, k, 16);
                const unsigned fk = __shfl_sync(gmask, my_fa, k, 16);
                const unsigned gk = __shfl_sync(gmask, my_fb, k, 16);
                if (i >= nc || (selected & (1u << k))) continue;
                const unsigned long long f = (static_cast<unsigned long long>(fk) << 32) | gk;
                const float tol = fmaxf(kTieAbsolute, kTieRelative * fmaxf(fabsf(sc), fabsf(best_score)));
                if (sc > best_score + tol || (fabsf(sc - best_score) <= tol && f < best_feature)) {
                    best = k;
                    best_score = sc;
                    best_feature = f;
                }
            }
            if (best >= 0) {
                selected |= 1u << best;
                chosen |= static_cast<unsigned long long>(best) << (4 * chosen_count);
                ++chosen_count;
                if (stage == 1) w1 = shfl3g(my_wp, best, gmask);
                if (stage == 2) w2 = shfl3g(my_wp, best, gmask);
            }
        }
        // Chosen candidates in feature order.
        unsigned long long keys[kManifoldPoints];
        int lanes[kManifoldPoints];
#pragma unroll
        for (int i = 0; i < kManifoldPoints; ++i) {
            const int k = static_cast<int>((chosen >> (4 * i)) & 0xfull);
            const unsigned fk = __shfl_sync(gmask, my_fa, k, 16);
            const unsigned gk = __shfl_sync(gmask, my_fb, k, 16);
            keys[i] = i < chosen_count ? ((static_cast<unsigned long long>(fk) << 32) | gk) : ~0ull;
            lanes[i] = k;
        }
#pragma unroll
        for (int i = 1; i < kManifoldPoints; ++i)
#pragma unroll
            for (int j = i; j > 0; --j)
                if (keys[j] < keys[j - 1]) {
                    const unsigned long long tk = keys[j]; keys[j] = keys[j - 1]; keys[j - 1] = tk;
                    const int tl = lanes[j]; lanes[j] = lanes[j - 1]; lanes[j - 1] = tl;
                }
#pragma unroll
        for (int i = 0; i < kManifoldPoints; ++i) final_order |= static_cast<unsigned long long>(lanes[i]) << (4 * i);
        nfinal = chosen_count;
    } else {
        // Canonical order of all candidates by feature key.
        int rank = 0;
#pragma unroll
        for (int j = 0; j < kManifoldPoints; ++j) {
            const unsigned fj = __shfl_sync(gmask, my_fa, j, 16);
            const unsigned gj = __shfl_sync(gmask, my_fb, j, 16);
            if (j < nc && sl < nc && j != sl && (fj < my_fa || (fj == my_fa && gj < my_fb))) ++rank;
        }
#pragma unroll
        for (int i = 0; i < kManifoldPoints; ++i) {
            const unsigned who = group_ballot(gmask, gbase, sl < nc && rank == i);
            if (i < nc) final_order |= static_cast<unsigned long long>(__ffs(who) - 1) << (4 * i);
        }
        nfinal = nc;
    }
    // Write the slot: lane i < 4 writes point i, lane 0 the header.
    const int src = sl < nfinal ? static_cast<int>((final_order >> (4 * (sl & 3))) & 0xfull) : 0;
    const unsigned id = __shfl_sync(gmask, my_id, src, 16);
    __syncwarp(gmask);
    if (sl < kManifoldPoints) {
        float* op = slot + 8 + sl * 12;
        if (sl < nfinal) {
            const float* g = scratch + (id & 15u) * kCandidateWords;
#pragma unroll
            for (int k = 0; k < 8; ++k) op[k] = g[k];
            if ((id >> 4) == kFresh) {
                op[8] = as_float(0);
                op[9] = op[10] = op[11] = 0.0f;
            } else {
                const float* hrec = scratch + (id >> 4) * kCandidateWords;
                op[8] = hrec[kCdLife];
                op[9] = hrec[kCdImp + 0];
                op[10] = hrec[kCdImp + 1];
                op[11] = hrec[kCdImp + 2];
            }
        } else {
#pragma unroll
            for (int k = 0; k < 12; ++k) op[k] = 0.0f;
        }
    }
    if (sl == 0) {
        float3 tw = transported;
        if (!old_ok || !finite3(tw) || dot3(tw, tw) <= 1.0e-12f) tw = stable_tangent(nw);
        else tw = tw * (1.0f / len3(tw));
        st3(slot, qrotinv(rotA, nw));
        slot[3] = old_ok ? fminf(old_age + 1.0f, 65535.0f) : 0.0f;
        st3(slot + 4, qrotinv(rotA, tw));
        slot[7] = as_float(nfinal);
    }
    __syncwarp(gmask);
    npoints_out = nfinal;
}

// ---------------------------------------------------------------------------
// Rows of Y = L^-T G^T over each contact body's ancestor DoFs, as the
// quality solver reads them (quality.cuh).
struct TreeRows {
    const DeviceTables* T;
    const float* Y;
    const float* C;
    int ma;
    __device__ __forceinline__ int body(int c) const { return as_int(C[c * kContactWords + kCwBody]); }
    __device__ __forceinline__ int count(int c) const { return T->anc_count[body(c)]; }
    __device__ __forceinline__ int dof(int c, int k) const { return T->anc[body(c)][k]; }
    __device__ __forceinline__ int pos(int c, int d) const {
        const int t = T->pos[body(c)][d];
        return t == kNone ? -1 : t;
    }
    __device__ __forceinline__ double y(int c, int r, int k) const { return static_cast<double>(Y[(c * 3 + r) * ma + k]); }
};

// Converged contact solve (qualityNewton) of the `total` evaluated contacts
// in place of the temporalCone sweeps: the regularisation floor, the warm
// impulses of the manifold points, the FP64 Newton solve, then z = Y lambda
// and the impulses back into the contact records.  A solve that does not
// converge latches MR_STEP_DID_NOT_CONVERGE (the step keeps its checkpoint).
__device__ bool quality_contacts(const Warp& w, int total, int ma, const QualityConfig& cfg) {
    const WarpLayout& L = *w.L;
    float* s = w.s;
    float* misc = s + L.misc;
    float* C = s + L.contacts;
    float* z = s + L.z;
    const int nv = w.M->nv, lane = w.lane;
    double* ws = reinterpret_cast<double*>(s + L.quality);
    double* K = ws + quality_contact_offset(nv);
    if (lane < total) {
        const float* c = C + lane * kContactWords;
        double* k = K + lane * kQuWords;
        for (int r = 0; r < 3; ++r) {
            k[kQuFree + r] = c[kCwUfree + r];
            k[kQuTarget + r] = c[kCwTarget + r];
            k[kQuReg + r] = fmax(static_cast<double>(c[kCwReg + r]), cfg.regularization_floor);
        }
        k[kQuMu] = c[kCwMuU];
        const float3 warm = project_cone(ld3(c + kCwLambda), c[kCwMuU], c[kCwMuV]);
        k[kQuLambda + 0] = warm.x;
        k[kQuLambda + 1] = warm.y;
        k[kQuLambda + 2] = warm.z;
    }
    __syncwarp();
    const TreeRows rows{w.T, s + L.G, C, ma};
    const QualityOutcome o = quality_solve(rows, nv, total, ws, cfg, lane);
    for (int d = lane; d < nv; d += 32) z[d] = static_cast<float>(quality_y_lambda(rows, total, K, d));
    if (lane < total) {
        const double* k = K + lane * kQuWords + kQuLambda;
        st3(C + lane * kContactWords + kCwLambda, f3(static_cast<float>(k[0]), static_cast<float>(k[1]), static_cast<float>(k[2])));
    }
    if (lane == 0) {
        misc[kMiscQualityNewton] = as_float(max(as_int(misc[kMiscQualityNewton]), o.newton));
        misc[kMiscQualityLineSearch] = as_float(as_int(misc[kMiscQualityLineSearch]) + o.line_search);
        misc[kMiscQualityResidual] = fmaxf(misc[kMiscQualityResidual], static_cast<float>(o.residual));
        misc[kMiscQualityCone] = fmaxf(misc[kMiscQualityCone], static_cast<float>(o.cone));
        misc[kMiscQualityComplementarity] = fmaxf(misc[kMiscQualityComplementarity], static_cast<float>(o.complementarity));
        if (o.status != kQualityConverged)
            set_status(misc,
                       o.status == kQualityFactorization ? MR_STEP_FACTORIZATION_FAILED
                                                         : (o.status == kQualityNonfinite ? MR_STEP_NONFINITE_RESULT : MR_STEP_DID_NOT_CONVERGE),
                       static_cast<unsigned>(o.newton));
    }
    __syncwarp();
    return warp_ok(misc);
}

// Contact substep after the ABA: collision, ConstraintIR evaluation, joint
// inertia factor, temporalCone (or quality) solve, joint limits, integration.
// ---------------------------------------------------------------------------
template <bool kComp, bool kQuality, typename R>
__device__ bool contact_substep(const Warp& w, const BodyConst& bc, BodyState<R>& st, bool final_substep,
                                int velocity_iterations, int final_iterations, float friction_scale,
                                const QualityConfig& quality) {
    const DeviceModel& M = *w.M;
    const DeviceTables& T = *w.T;
    const WarpLayout& L = *w.L;
    float* s = w.s;
    float* misc = s + L.misc;
    const int lane = w.lane;
    const int nv = M.nv;
    const float h = M.h;
    const float* pose = s + L.body_pose;
    float* q = s + L.q;
    float* v = s + L.v;
    const float* vf = s + L.vf;
    const float* Jax = s + L.dof_J;
    float* slots = s + L.manifolds;
    float* C = s + L.contacts;
    float* Y = s + L.G;     // G rows, factored in place into Y = L^-T G^T
    float* Lm = s + L.L;    // packed lower factor rows
    float* z = s + L.z;     // L-space image of the accumulated impulses
    const int ma = T.max_anc | 1;  // odd row stride of Y: lane-per-row access is conflict free

    // Speculative margins of articulated colliders (Collision.metal:5882-5915):
    // h * sum|v_free| * max(sweep radius, 0.25), capped by h * speed envelope.
    float gs = 0.0f;
    for (int d = lane; d < nv; d += 32) gs += fabsf(vf[d]);
    gs = warp_sum(gs);
    float* margins = s + L.margins;
    if (lane < M.ns) {
        float m = 0.0f;
        if (M.shape_body[lane] >= 0 && M.shape_type[lane] != MR_SHAPE_PLANE)
            m = M.speculative_scale * fminf(h * gs * fmaxf(M.shape_offsets[lane].z, 0.25f), h * M.speed_envelope);
        margins[lane] = m;
    }
    __syncwarp();

    // Narrowphase + manifolds: lane per pair.
    int npoints = 0, nraw = 0;
    bool cand = false;
    bool pair_fail = false;
    // Scratch of each pair: exclusive prefix of the per-class sizes.
    const int my_words = lane < M.np ? pair_scratch_words(pair_max_raw(M.pair_class[lane])) : 0;
    int scratch_end = my_words;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, scratch_end, o);
        if (lane >= o) scratch_end += t;
    }
    // Light pair classes (at most two raw contacts): one lane per pair.
    const bool heavy = lane < M.np && pair_max_raw(M.pair_class[lane]) > 2;
    const unsigned heavy_mask = __ballot_sync(0xffffffffu, heavy);
    if (lane < M.np && !heavy) {
        npoints = pair_manifold(M, pose, margins, lane, slots + lane * kSlotStride, s + L.narrow + scratch_end - my_words,
                                nraw, cand);
        if (npoints < 0) { pair_fail = true; npoints = 0; }
    }
    // Heavy pair classes: a 16-lane group per pair, two pairs at a time.
    if (heavy_mask != 0u) {
        float* pstats = s + L.pair_stats;
        const int g = lane >> 4, sl = lane & 15, gbase = lane & 16;
        const unsigned gmask = g ? 0xffff0000u : 0x0000ffffu;
        const int nheavy = __popc(heavy_mask);
        for (int first = 0; first < nheavy; first += 2) {
            unsigned m = heavy_mask;
            for (int k = 0; k < first + g && m != 0u; ++k) m &= m - 1u;
            const int pair = m != 0u ? __ffs(m) - 1 : -1;
            const int off = __shfl_sync(0xffffffffu, scratch_end - my_words, pair >= 0 ? pair : 0);
            if (pair >= 0) {
                int gp = 0, gr = 0;
                bool gc = false, gf = false;
                group_manifold(M, pose, margins, pair, slots + pair * kSlotStride, s + L.narrow + off, sl, gbase, gmask, gp,
                               gr, gc, gf);
                if (sl == 0) pstats[pair] = as_float(gp | (gr << 8) | (gc ? 1 << 16 : 0) | (gf ? 1 << 17 : 0));
            }
        }
        __syncwarp();
        if (heavy) {
            const int packed = as_int(pstats[lane]);
            npoints = packed & 0xff;
            nraw = (packed >> 8) & 0xff;
            cand = (packed >> 16) & 1;
            pair_fail = (packed >> 17) & 1;
        }
    }
    const unsigned fail_mask = __ballot_sync(0xffffffffu, pair_fail);
    if (fail_mask != 0u) {
        if (lane == 0) set_status(misc, MR_STEP_NONFINITE_RESULT, static_cast<unsigned>(__ffs(fail_mask) - 1));
        __syncwarp();
        return false;
    }
    // Stable exclusive prefix over pairs (contacts ordered by pair, then point).
    int incl = npoints;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    const int base = incl - npoints;
    {
        const unsigned mcount = __popc(__ballot_sync(0xffffffffu, npoints > 0));
        int raw_total = nraw;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) raw_total += __shfl_xor_sync(0xffffffffu, raw_total, o);
        const unsigned cand_count = __popc(__ballot_sync(0xffffffffu, cand));
        if (lane == 0) {
            misc[kMiscContactCount] = as_float(total);
            misc[kMiscManifoldCount] = as_float(max(as_int(misc[kMiscManifoldCount]), static_cast<int>(mcount)));
            misc[kMiscRawCount] = as_float(max(as_int(misc[kMiscRawCount]), raw_total));
            misc[kMiscCandidatePairs] = as_float(max(as_int(misc[kMiscCandidatePairs]), static_cast<int>(cand_count)));
        }
    }
    if (total > M.contact_capacity) {
        if (lane == 0) set_status(misc, MR_STEP_CONTACT_CAPACITY_OVERFLOW, static_cast<unsigned>(total));
        __syncwarp();
        return false;
    }

    // Contact records (mr_world_scatter_manifold_ir): the pair lane emits
    // its points in manifold order.
    if (lane < M.np && npoints > 0) {
        const int pair = lane;
        const float* slot = slots + pair * kSlotStride;
        const int sa = M.pair_a[pair], sb = M.pair_b[pair];
        const int ba = M.shape_body[sa], bb = M.shape_body[sb];
        float3 posA, posB;
        float4 rotA, rotB;
        if (ba >= 0) { posA = ld3(pose + ba * kPoseStride); rotA = ld4(pose + ba * kPoseStride + 3); }
        else { posA = xyz(M.static_body_position[sa]); rotA = M.static_body_rotation[sa]; }
        if (bb >= 0) { posB = ld3(pose + bb * kPoseStride); rotB = ld4(pose + bb * kPoseStride + 3); }
        else { posB = xyz(M.static_body_position[sb]); rotB = M.static_body_rotation[sb]; }
        float3 nw = qrot(rotA, ld3(slot));
        nw = nw * (1.0f / len3(nw));
        float3 tw = qrot(rotA, ld3(slot + 4));
        tw = tw - nw * dot3(tw, nw);
        tw = dot3(tw, tw) > 1.0e-12f ? tw * (1.0f / len3(tw)) : stable_tangent(nw);
        const float3 bw = cross3(nw, tw);
        const float4 fa = M.material_friction[M.shape_material[sa]];
        const float4 fb = M.material_friction[M.shape_material[sb]];
        const float mu_s = sqrtf(fmaxf(0.0f, fa.x * fb.x)) * friction_scale;
        const float mu_d = sqrtf(fmaxf(0.0f, fa.y * fb.y)) * friction_scale;
        const float4 ra = M.material_response[M.shape_material[sa]];
        const float4 rb = M.material_response[M.shape_material[sb]];
        const float restitution = fminf(fmaxf(fmaxf(ra.x, rb.x), 0.0f), 1.0f);
        const float rthreshold = fmaxf(ra.y, rb.y);
        const float compliance = ra.z + rb.z;
        const float dissipation = ra.w + rb.w;
        const float rest = M.shape_offsets[sa].y + M.shape_offsets[sb].y;
        for (int i = 0; i < npoints; ++i) {
            const float* op = slot + 8 + i * 12;
            float* c = C + (base + i) * kContactWords;
            const float3 pa = posA + qrot(rotA, ld3(op));
            const float3 pb = posB + qrot(rotB, ld3(op + 3));
            const float3 pw = 0.5f * (pa + pb);
            const float sep = dot3(pb - pa, nw) - rest;
            st3(c + kCwPoint, pw);
            c[kCwSeparation] = sep;
            st3(c + kCwNormal, nw);
            st3(c + kCwTangent, tw);
            st3(c + kCwBitangent, bw);
            const unsigned life = static_cast<unsigned>(as_int(op[8]));
            const bool new_impact = life == 0u;
            const bool b_side = ba < 0;
            c[kCwBody] = as_float(b_side ? bb : ba);
            c[kCwFlags] = as_float((new_impact ? 1 : 0) | (b_side ? 256 : 0));
            c[kCwSlot] = as_float(pair * 4 + i);
            c[kCwLambda + 0] = op[9];
            c[kCwLambda + 1] = op[10];
            c[kCwLambda + 2] = op[11];
            c[kCwTarget + 0] = sep > 0.0f ? -sep / h : 0.0f;
            c[kCwTarget + 1] = 0.0f;
            c[kCwTarget + 2] = 0.0f;
            c[kCwReg + 0] = fmaxf(compliance / (h * h) + dissipation / h, 0.0f);
            c[kCwReg + 1] = 0.0f;
            c[kCwReg + 2] = 0.0f;
            c[kCwMuU] = mu_s;
            c[kCwMuV] = mu_d;
            c[kCwRelax] = restitution;
            c[kCwDelta + 0] = rthreshold;
        }
    }
    __syncwarp();

    // Jacobian rows G over the body's ancestor DoFs (positions in anc[b])
    // and evaluation of the ConstraintIR rows at v_free
    // (MetalWorldContact.metal:3580-3990).
    if (lane < total) {
        float* c = C + lane * kContactWords;
        const int b = as_int(c[kCwBody]);
        const int flags = as_int(c[kCwFlags]);
        const float sign = (flags & 256) ? 1.0f : -1.0f;
        const float3 x = ld3(c + kCwPoint);
        const float3 dirs[3] = {ld3(c + kCwNormal), ld3(c + kCwTangent), ld3(c + kCwBitangent)};
        const int na = T.anc_count[b];
        float* g = Y + lane * 3 * ma;
        float rel[3] = {0.0f, 0.0f, 0.0f};
        for (int k = 0; k < na; ++k) {
            const int d = T.anc[b][k];
            // Point-Jacobian column: a x (x - o) for rotations, a for translations.
            const float* jd = Jax + d * kJStride;
            const float3 ax = f3(jd[0], jd[1], jd[2]);
            const float3 jc = jd[6] != 0.0f ? ax : cross3(ax, x - f3(jd[3], jd[4], jd[5]));
            const float vk = vf[d];
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                const float gv = sign * dot3(dirs[r], jc);
                g[r * ma + k] = gv;
                rel[r] = fmaf(gv, vk, rel[r]);
            }
        }
        for (int r = 0; r < 3; ++r) c[kCwUfree + r] = rel[r];
        // Normal row: critically damped stabilisation clamped to the maximum
        // depenetration speed, plus restitution on a new impact.
        const float sep = c[kCwSeparation];
        const float tau_c = 2.0f * h;
        const float err = fminf(sep + M.slop, 0.0f);
        const float ratio = h / tau_c;
        const float den = 1.0f + 2.0f * 1.0f * ratio + ratio * ratio;
        float stab = -h * err / (tau_c * tau_c * den);
        stab = fminf(fmaxf(stab, 0.0f), M.max_depenetration);
        const float restitution = c[kCwRelax];
        const float rthreshold = c[kCwDelta + 0];
        if (flags & 1) {
            const float incoming = rel[0] - c[kCwTarget + 0];
            if (incoming < -rthreshold) stab = fmaxf(stab, -restitution * incoming);
        }
        c[kCwTarget + 0] += stab;
        const float slip = sqrtf(rel[1] * rel[1] + rel[2] * rel[2]);
        const float mu = slip <= 1.0e-3f ? c[kCwMuU] : c[kCwMuV];
        c[kCwMuU] = mu;
        c[kCwMuV] = mu;
        if (!isfinite(c[kCwTarget + 0]) || !isfinite(c[kCwReg + 0])) set_status(misc, MR_STEP_NONFINITE_RESULT, static_cast<unsigned>(lane));
    }
    if (!warp_ok(misc)) return false;

    for (int d = lane; d < nv; d += 32) v[d] = vf[d];
    if (total > 0) {
        if (lane == 0) misc[kMiscIslands] = as_float(max(as_int(misc[kMiscIslands]), 1));
        // Y = L^-T G^T per contact row, in place over the ancestor positions.
        const int nrows = 3 * total;
        for (int row = lane; row < nrows; row += 32) {
            const int c = row / 3, r = row - 3 * (row / 3);
            const int b = as_int(C[c * kContactWords + kCwBody]);
            const int na = T.anc_count[b];
            float* y = Y + c * 3 * ma + r * ma;
            if (na <= kRegisterChain) {
                // Register-resident back substitution for chains of up to 16
                // ancestor DoFs (fully unrolled, predicated on the length).
                float yr[kRegisterChain];
                int off[kRegisterChain];
#pragma unroll
                for (int t = 0; t < kRegisterChain; ++t) {
                    const int k = t < na ? T.anc[b][t] : 0;
                    off[t] = k * (k + 1) / 2;
                    yr[t] = t < na ? y[t] : 0.0f;
                }
#pragma unroll
                for (int t = kRegisterChain - 1; t >= 0; --t) {
                    if (t < na) {
                        const float* rowk = Lm + off[t];
                        const float yt = yr[t] / rowk[T.anc[b][t]];
                        yr[t] = yt;
#pragma unroll
                        for (int u = 0; u < t; ++u) yr[u] -= rowk[T.anc[b][u]] * yt;
                    }
                }
#pragma unroll
                for (int t = 0; t < kRegisterChain; ++t)
                    if (t < na) y[t] = yr[t];
            } else {
                for (int t = na - 1; t >= 0; --t) {
                    const int k = T.anc[b][t];
                    const float* rowk = Lm + k * (k + 1) / 2;
                    const float yt = y[t] / rowk[k];
                    y[t] = yt;
                    for (int u = 0; u < t; ++u) y[u] -= rowk[T.anc[b][u]] * yt;
                }
            }
        }
        __syncwarp();
        if constexpr (kQuality) {
            if (!quality_contacts(w, total, ma, quality)) return false;
        } else {
        // Per-DoF lists of the contact rows that reach it, as (position in
        // the contact's ancestor list << 5 | contact), so a sweep's z update
        // visits only those.  The lists reuse the factor rows past the root
        // block: once Y exists the sweeps read no joint row of L.
        std::uint16_t* dlist = reinterpret_cast<std::uint16_t*>(Lm + kRootFactorWords);
        const int ncap = M.contact_capacity;
        int dcount[2] = {0, 0};
#pragma unroll
        for (int pass = 0; pass < 2; ++pass) {
            const int d = lane + 32 * pass;
            if (d < nv) {
                z[d] = 0.0f;
                int cnt = 0;
                for (int j = 0; j < total; ++j) {
                    const int t = T.pos[as_int(C[j * kContactWords + kCwBody])][d];
                    if (t != kNone) dlist[d * ncap + cnt++] = static_cast<std::uint16_t>((t << 5) | j);
                }
                dcount[pass] = cnt;
            }
        }
        __syncwarp();
        // Preconditioners, relaxation and warm start (lane per contact):
        // W_cc = Y_c^T Y_c + R, normal row sums over the common ancestor prefix.
        if (lane < total) {
            float* c = C + lane * kContactWords;
            const int b = as_int(c[kCwBody]);
            const int na = T.anc_count[b];
            const float* yc = Y + lane * 3 * ma;
            float Wm[3][3];
            for (int r = 0; r < 3; ++r)
                for (int cc = 0; cc <= r; ++cc) {
                    float acc = 0.0f;
                    for (int t = 0; t < na; ++t) acc = fmaf(yc[r * ma + t], yc[cc * ma + t], acc);
                    Wm[r][cc] = acc;
                    Wm[cc][r] = acc;
                }
            float rowsum = 0.0f;
            for (int j = 0; j < total; ++j) {
                const int bj = as_int(C[j * kContactWords + kCwBody]);
                const int n = T.lcp[b][bj];
                const float* yj = Y + j * 3 * ma;
                float acc = 0.0f;
                for (int t = 0; t < n; ++t) acc = fmaf(yc[t], yj[t], acc);
                rowsum += fabsf(acc);
            }
            const float diag = fabsf(Wm[0][0]) + c[kCwReg + 0];
            for (int r = 0; r < 3; ++r) Wm[r][r] += c[kCwReg + r];
            float inv[3][3];
            if (!invert3x3_reg(Wm, inv)) {
                set_status(misc, MR_STEP_FACTORIZATION_FAILED, static_cast<unsigned>(lane));
            } else {
                for (int r = 0; r < 3; ++r)
                    for (int cc = 0; cc < 3; ++cc) c[kCwPre + r * 3 + cc] = inv[r][cc];
            }
            c[kCwRelax] = rowsum > fmaxf(diag, kMatrixFloor) ? fminf(fmaxf(diag / rowsum, 1.0f / 32.0f), 1.0f) : 1.0f;
            const float3 warm = project_cone(ld3(c + kCwLambda), c[kCwMuU], c[kCwMuV]);
            st3(c + kCwLambda, warm);
            st3(c + kCwDelta, warm);
        }
        if (!warp_ok(misc)) return false;
        // Jacobi sweeps: lane per contact proposes from u = u_free + Y^T z,
        // lane per DoF accumulates z += Y delta.  Sweep -1 applies the warm start.
        const int iters = velocity_iterations + (final_substep ? final_iterations : 0);
        float zcomp[2] = {0.0f, 0.0f};  // kComp: compensation of the z sums
        for (int it = -1; it < iters; ++it) {
            if (it >= 0 && lane < total) {
                float* c = C + lane * kContactWords;
                const int b = as_int(c[kCwBody]);
                const int na = T.anc_count[b];
                const float* yc = Y + lane * 3 * ma;
                float u0 = c[kCwUfree + 0], u1 = c[kCwUfree + 1], u2 = c[kCwUfree + 2];
                for (int t = 0; t < na; ++t) {
                    const float zk = z[T.anc[b][t]];
                    u0 = fmaf(yc[t], zk, u0);
                    u1 = fmaf(yc[ma + t], zk, u1);
                    u2 = fmaf(yc[2 * ma + t], zk, u2);
                }
                const float3 prev = ld3(c + kCwLambda);
                const float r0 = c[kCwTarget + 0] - u0 - c[kCwReg + 0] * prev.x;
                const float r1 = c[kCwTarget + 1] - u1 - c[kCwReg + 1] * prev.y;
                const float r2 = c[kCwTarget + 2] - u2 - c[kCwReg + 2] * prev.z;
                const float* P = c + kCwPre;
                float3 prop = f3(prev.x + P[0] * r0 + P[1] * r1 + P[2] * r2, prev.y + P[3] * r0 + P[4] * r1 + P[5] * r2,
                                 prev.z + P[6] * r0 + P[7] * r1 + P[8] * r2);
                prop = project_cone(prop, c[kCwMuU], c[kCwMuV]);
                const float relax = c[kCwRelax];
                const float3 delta = relax * (prop - prev);
                const float3 next = prev + delta;
                if (!finite3(next) || !finite3(delta)) {
                    set_status(misc, MR_STEP_NONFINITE_RESULT, static_cast<unsigned>(lane));
                    st3(c + kCwDelta, f3(0.0f, 0.0f, 0.0f));
                } else {
                    st3(c + kCwLambda, next);
                    st3(c + kCwDelta, delta);
                }
            }
            __syncwarp();
#pragma unroll
            for (int pass = 0; pass < 2; ++pass) {
                const int d = lane + 32 * pass;
                if (d < nv) {
                    float acc = 0.0f;
                    const std::uint16_t* list = dlist + d * ncap;
#pragma unroll 4
                    for (int k = 0; k < dcount[pass]; ++k) {
                        const int e = list[k];
                        const int j = e & 31;
                        const float* cj = C + j * kContactWords;
                        const float* yj = Y + j * 3 * ma + (e >> 5);
                        acc = fmaf(yj[0], cj[kCwDelta + 0], acc);
                        acc = fmaf(yj[ma], cj[kCwDelta + 1], acc);
                        acc = fmaf(yj[2 * ma], cj[kCwDelta + 2], acc);
                    }
                    if (kComp) z[d] = kahan_madd(z[d], 1.0f, acc, zcomp[pass]);
                    else z[d] += acc;
                }
            }
            __syncwarp();
        }
        if (!warp_ok(misc)) return false;
        }  // temporalCone
        // Velocity change x = L^-1 z as one forward tree sweep: with
        // L_kj = U_k . S_j(c_k) / L_kk, sum_j L_kj x_j is U_k applied to the
        // parent's twist change moved to body k's COM, so each body needs
        // only its parent's twist change (by shuffle), not its ancestors' x.
        {
            const bool mine = lane < T.nb;
            const int my_depth = mine ? T.depth[lane] : -1;
            const int par = (mine && lane > 0) ? T.parent[lane] : lane;
            float3 dw = f3(0.0f, 0.0f, 0.0f), dv = f3(0.0f, 0.0f, 0.0f);
            if (lane == 0 && T.floating) {
                float xr[6];
#pragma unroll
                for (int k = 0; k < 6; ++k) {
                    const float* rowk = Lm + k * (k + 1) / 2;
                    float acc = z[k];
#pragma unroll
                    for (int j = 0; j < k; ++j) acc -= rowk[j] * xr[j];
                    xr[k] = acc / rowk[k];
                    v[k] += xr[k];
                }
                dv = f3(xr[0], xr[1], xr[2]);
                dw = f3(xr[3], xr[4], xr[5]);
            }
            for (int l = 1; l <= T.n_levels; ++l) {
                const float3 pw = shfl3(dw, par);
                const float3 pv = shfl3(dv, par);
                if (my_depth == l) {
                    dw = pw;
                    dv = pv + cross3(pw, st.r);
                    if (bc.dof >= 0) {
                        const int k = bc.dof;
                        const float lkk = static_cast<float>(sqrt(st.D));  // = L_kk as written by the ABA
                        const float sum = static_cast<float>(st.U[0] * dw.x + st.U[1] * dw.y + st.U[2] * dw.z +
                                                             st.U[3] * dv.x + st.U[4] * dv.y + st.U[5] * dv.z);
                        const float xk = (z[k] - sum / lkk) / lkk;
                        v[k] += xk;
                        dw = dw + f3(st.s[0], st.s[1], st.s[2]) * xk;
                        dv = dv + f3(st.s[3], st.s[4], st.s[5]) * xk;
                    }
                }
            }
        }
        __syncwarp();
        // Impulses back into the manifold points (warm start of the next substep).
        if (lane < total) {
            const float* c = C + lane * kContactWords;
            const int slot = as_int(c[kCwSlot]);
            float* op = slots + (slot >> 2) * kSlotStride + 8 + (slot & 3) * 12;
            op[9] = c[kCwLambda + 0];
            op[10] = c[kCwLambda + 1];
            op[11] = c[kCwLambda + 2];
        }
    }
    __syncwarp();

    // Joint limits on the post-solve velocity (mr_world_project_joint_limits).
    for (int d = lane; d < nv; d += 32) {
        const unsigned flags = M.dof_flags[d];
        float vel = v[d];
        if (flags & MR_DOF_FLAG_VELOCITY_LIMIT) vel = fminf(fmaxf(vel, -M.v_max[d]), M.v_max[d]);
        const int qi = M.dof_q[d];
        if ((flags & MR_DOF_FLAG_POSITION_LIMIT) && qi >= 0) {
            const float pos = q[qi];
            vel = fminf(fmaxf(vel, (M.q_lower[d] - pos) / h), (M.q_upper[d] - pos) / h);
        }
        if (!isfinite(vel)) set_status(misc, MR_STEP_NONFINITE_RESULT, static_cast<unsigned>(d));
        v[d] = vel;
    }
    __syncwarp();
    // Integration from the substep-start configuration
    // (mr_world_integrate_contact_state; no angle reduction).
    float* qc = s + L.qcomp;
    for (int d = lane; d < nv; d += 32) {
        const int qi = M.dof_q[d];
        if (qi >= 0 && !(M.floating && d < 6)) q[qi] = kComp ? kahan_madd(q[qi], h, v[d], qc[qi]) : q[qi] + h * v[d];
    }
    if (M.floating && lane == 0) {
        if (kComp) {
            for (int i = 0; i < 3; ++i) q[i] = kahan_madd(q[i], h, v[i], qc[i]);
        } else {
            q[0] += h * v[0];
            q[1] += h * v[1];
            q[2] += h * v[2];
        }
        const float4 inc = so3_increment(h * f3(v[3], v[4], v[5]), false);
        const float4 prod = qmul(inc, make_float4(q[3], q[4], q[5], q[6]));
        if (!finite4(prod) || !(qdot(prod, prod) > 1.0e-12f)) {
            set_status(misc, MR_STEP_NONFINITE_RESULT, 3u);
        } else {
            const float4 out = qscale(prod, rsqrtf(qdot(prod, prod)));
            q[3] = out.x; q[4] = out.y; q[5] = out.z; q[6] = out.w;
        }
    }
    __syncwarp();
    for (int i = lane; i < M.nq; i += 32)
        if (!isfinite(q[i])) set_status(misc, MR_STEP_NONFINITE_RESULT, static_cast<unsigned>(i));
    return warp_ok(misc);
}

// FP64 audit of one environment's state (audit.cuh): forward kinematics of
// the q and v in the warp's layout, then each lane's body.  Run by its own
// kernel after the control step, so the step kernel carries none of it.
template <typename R>
__device__ void audit_articulated(const Warp& w, const BodyConst& bc, double* rec, bool reset) {
    const DeviceModel& M = *w.M;
    BodyState<R> st;
    kinematics(w, bc, st);
    __syncwarp();
    AuditSum a{};
    const int b = w.lane;
    if (b < M.nb)
        audit_body(a, M.mass_damping[b].x, st.c, st.qr, st.v, st.w, xyz(M.inertia_diag[b]), xyz(M.inertia_off[b]), M.gravity);
    audit_commit(a, rec, reset, w.lane);
}

// kComp (compensated precision): q's running sums carry compensation terms
// in the layout's qcomp section, loaded from and committed to p.q_comp.
//
// One warp advances work item `item` (the compact index of the launch's
// outputs: observations, status codes, contact counts) of environment slot
// `env` by one control step.  `tables` is the model's topology table (a
// shared-memory copy or the model record itself), `warp_smem` the warp's
// layout.total floats of shared memory.  Only warp-level synchronisation is
// used, so warps of one CTA may run different items, or different worlds.
template <bool kContact, typename R, bool kComp, bool kQuality = false>
__device__ __forceinline__ void control_step_item(const StepParams& p, const WarpLayout& layout, const DeviceTables* tables,
                                                  float* warp_smem, int item, int env) {
    const int lane = threadIdx.x & 31;
    const DeviceModel& M = *p.model;
    Warp w;
    w.lane = lane;
    w.T = tables;
    w.s = warp_smem;
    w.L = &layout;
    w.M = p.model;
    float* s = w.s;
    float* misc = s + layout.misc;
    const int nq = M.nq, nv = M.nv;

    // Prepare: reset, checkpoint, actions (mr_metal_world_prepare).
    const bool reset = p.reset_masks != nullptr && p.reset_masks[item] != 0u;
    const float* srcq = (reset ? p.reset_q : p.q) + static_cast<size_t>(env) * nq;
    const float* srcv = (reset ? p.reset_v : p.v) + static_cast<size_t>(env) * nv;
    for (int i = lane; i < nq; i += 32) {
        const float x = srcq[i];
        s[layout.q + i] = x;
        s[layout.qc + i] = x;
    }
    for (int i = lane; i < nv; i += 32) {
        const float x = srcv[i];
        s[layout.v + i] = x;
        s[layout.vc + i] = x;
        s[layout.tgt + i] = 0.0f;
    }
    if (kComp) {
        const float* srcc = p.q_comp + static_cast<size_t>(env) * nq;
        for (int i = lane; i < nq; i += 32) s[layout.qcomp + i] = reset ? 0.0f : srcc[i];
    }
    misc[lane] = 0.0f;
    __syncwarp();
    for (int a = lane; a < M.action_count; a += 32)
        s[layout.tgt + M.action_dof[a]] =
            p.action_rows != nullptr ? p.action_rows[item][a] : p.actions[static_cast<size_t>(item) * M.action_count + a];
    if (kContact) {
        // Slots sit at an odd stride in shared memory (lane-per-pair access
        // is conflict free) and packed in HBM.
        float* slots = s + layout.manifolds;
        const int words = M.np * kManifoldWords;
        const float* src = p.manifolds + static_cast<size_t>(env) * words;
        for (int i = lane; i < words; i += 32) {
            const int pair = i / kManifoldWords;
            slots[pair * kSlotStride + (i - pair * kManifoldWords)] = reset ? 0.0f : src[i];
        }
    }
    const float friction_scale = kContact ? p.friction_scale[env] : 1.0f;
    BodyConst bc;
    if (lane < M.nb) load_body(M, lane, bc);
    BodyState<R> st;
    __syncwarp();

    for (int sub = 0; sub < p.substeps; ++sub) {
        compute_drives(w);
        __syncwarp();
        bool ok = aba(w, bc, st, kContact ? s + layout.L : nullptr);
        if (ok) {
            if (kContact)
                ok = contact_substep<kComp, kQuality>(w, bc, st, sub + 1 == p.substeps, p.velocity_iterations,
                                                      p.final_velocity_iterations, friction_scale, p.quality);
            else
                ok = integrate_free<kComp>(w);
        }
        if (!ok) break;
    }
    const unsigned code = static_cast<unsigned>(as_int(misc[kMiscStatus]));
    const bool success = code == MR_STEP_SUCCESS;
    // Capture + commit: a failed step publishes (and keeps) its checkpoint.
    float* qd = p.q + static_cast<size_t>(env) * nq;
    float* vd = p.v + static_cast<size_t>(env) * nv;
    const float* qsrc = s + (success ? layout.q : layout.qc);
    const float* vsrc = s + (success ? layout.v : layout.vc);
    float* obs = p.observations ? p.observations + static_cast<size_t>(item) * (nq + nv) : nullptr;
    for (int i = lane; i < nq; i += 32) {
        const float x = qsrc[i];
        qd[i] = x;
        if (obs) obs[i] = x;
    }
    for (int i = lane; i < nv; i += 32) {
        const float x = vsrc[i];
        vd[i] = x;
        if (obs) obs[nq + i] = x;
    }
    if (kComp && (success || reset)) {
        // A failed step keeps the step-start terms (a failed reset, zeros).
        float* cd = p.q_comp + static_cast<size_t>(env) * nq;
        for (int i = lane; i < nq; i += 32) cd[i] = success ? s[layout.qcomp + i] : 0.0f;
    }
    if (kContact && (success || reset)) {
        const int words = M.np * kManifoldWords;
        float* dst = p.manifolds + static_cast<size_t>(env) * words;
        const float* slots = s + layout.manifolds;
        for (int i = lane; i < words; i += 32) {
            const int pair = i / kManifoldWords;
            dst[i] = success ? slots[pair * kSlotStride + (i - pair * kManifoldWords)] : 0.0f;
        }
    }
    if (lane == 0) {
        const unsigned contacts = kContact ? static_cast<unsigned>(as_int(misc[kMiscContactCount])) : 0u;
        if (p.status_codes) p.status_codes[item] = code;
        if (p.active_contacts) p.active_contacts[item] = success ? contacts : 0u;
        if (!success) {
            atomicAdd(p.stats + kStatFailedEnvs, 1u);
            atomicMin(p.stats + kStatFirstFailEnv, static_cast<unsigned>(env + p.env_base));
        }
        if (reset) atomicAdd(p.stats + kStatResets, 1u);
        if (kContact) {
            atomicMax(p.stats + kStatMaxContacts, contacts);
            atomicMax(p.stats + kStatMaxManifolds, static_cast<unsigned>(as_int(misc[kMiscManifoldCount])));
            atomicMax(p.stats + kStatMaxRawContacts, static_cast<unsigned>(as_int(misc[kMiscRawCount])));
            atomicMax(p.stats + kStatMaxCandidatePairs, static_cast<unsigned>(as_int(misc[kMiscCandidatePairs])));
            atomicMax(p.stats + kStatMaxIslands, static_cast<unsigned>(as_int(misc[kMiscIslands])));
        }
        if (kQuality) {
            atomicMax(p.stats + kStatQualityNewton, static_cast<unsigned>(as_int(misc[kMiscQualityNewton])));
            atomicAdd(p.stats + kStatQualityLineSearch, static_cast<unsigned>(as_int(misc[kMiscQualityLineSearch])));
            atomicMax(p.stats + kStatQualityResidual, static_cast<unsigned>(as_int(misc[kMiscQualityResidual])));
            atomicMax(p.stats + kStatQualityCone, static_cast<unsigned>(as_int(misc[kMiscQualityCone])));
            atomicMax(p.stats + kStatQualityComplementarity, static_cast<unsigned>(as_int(misc[kMiscQualityComplementarity])));
        }
    }
}

}  // namespace
}  // namespace numi
