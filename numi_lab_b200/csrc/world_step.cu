// Batched articulated-physics control step for B200 (sm_100a).
//
// One warp owns one environment for a whole control step (all physics
// substeps).  The environment's state, manifolds, articulated inertias,
// contact Jacobians and response columns stay in shared memory; HBM sees the
// step's inputs (resident q, v, manifolds, actions, reset mask) once and its
// outputs (committed state, observation, status) once.
//
// Stage order per substep follows numi-lab's MetalWorld graph
// (src/metal/MetalWorld.mm:17075-17370 and encodeContactSubstep
// :12682-13260): drive refresh -> ABA -> [kinematics, collider projection,
// pair flags, narrowphase, persistent manifolds, ConstraintIR evaluation,
// response columns, temporalCone solve, joint limits, integration] ->
// latch.  The control step is one transaction: the first failing substep
// latches a status and the environment keeps its step-start checkpoint.
//
// Spatial algebra uses (angular, linear) vectors about one reference point
// per environment (the floating root's COM at substep start, or the world
// origin for a fixed root), so no per-body shift transforms are needed in
// the tree sweeps.
#include "device_model.h"
#include "dmath.cuh"
#include "layout.h"

#include <cfloat>
#include <cstdint>

namespace numi {
namespace {

constexpr float kFloatEps = 1.1920928955078125e-7f;
constexpr float kAbsolutePivotFloor = 1.0e-12f;
constexpr float kMatrixFloor = 1.0e-10f;
constexpr float kContactCfm = 1.0e-2f;          // MetalWorldContact.metal:18
constexpr float kQueryPad = 0.00000762939453125f;  // MR_COLLISION_QUERY_RELATIVE_PAD
constexpr float kAabbPad = 0.00000762939453125f;   // MR_COLLISION_AABB_RELATIVE_PAD

__device__ __forceinline__ int as_int(float f) { return __float_as_int(f); }
__device__ __forceinline__ float as_float(int i) { return __int_as_float(i); }

struct Warp {
    int lane;
    float* s;          // this warp's shared-memory base
    const WarpLayout* L;
    const DeviceModel* M;
};

__device__ __forceinline__ void set_status(float* misc, unsigned code, unsigned index) {
    // Only the first failure of a control step is kept.
    if (as_int(misc[kMiscStatus]) == MR_STEP_SUCCESS) {
        misc[kMiscStatus] = as_float(static_cast<int>(code));
        misc[kMiscFailIndex] = as_float(static_cast<int>(index));
    }
}

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
__device__ void shift_inertia(const float* I, float3 r, float* out) {
    float A[3][3], B[3][3], D[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            A[i][j] = I[sym6(i, j)];
            B[i][j] = I[sym6(3 + j, i)];
            D[i][j] = I[sym6(3 + i, 3 + j)];
        }
    const float E[3][3] = {{0.0f, -r.z, r.y}, {r.z, 0.0f, -r.x}, {-r.y, r.x, 0.0f}};
    float ED[3][3], BE[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            float ed = 0.0f, be = 0.0f;
            for (int k = 0; k < 3; ++k) {
                ed = fmaf(E[i][k], D[k][j], ed);
                be = fmaf(B[i][k], E[k][j], be);
            }
            ED[i][j] = ed;
            BE[i][j] = be;
        }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j <= i; ++j) {
            float ede = 0.0f;
            for (int k = 0; k < 3; ++k) ede = fmaf(ED[i][k], E[k][j], ede);
            // E B^T (i, j) = sum_k E[i][k] B[j][k] = -(B E)^T... written directly:
            float ebt = 0.0f;
            for (int k = 0; k < 3; ++k) ebt = fmaf(E[i][k], B[j][k], ebt);
            out[sym6(i, j)] = A[i][j] - BE[i][j] + ebt - ede;
        }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) out[sym6(3 + j, i)] = B[i][j] + ED[i][j];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j <= i; ++j) out[sym6(3 + i, 3 + j)] = D[i][j];
}

// Body spatial inertia about its own COM in world axes: [[R Ib R^T, 0], [0, m 1]].
__device__ void body_inertia(const DeviceModel& M, int b, float4 qb, float* I6, float Iw[3][3]) {
    const float m = M.mass_damping[b].x;
    const float4 di = M.inertia_diag[b];
    const float4 of = M.inertia_off[b];
    const float3 c0 = qrot(qb, f3(1.0f, 0.0f, 0.0f));
    const float3 c1 = qrot(qb, f3(0.0f, 1.0f, 0.0f));
    const float3 c2 = qrot(qb, f3(0.0f, 0.0f, 1.0f));
    const float Ib[3][3] = {{di.x, of.x, of.y}, {of.x, di.y, of.z}, {of.y, of.z, di.z}};
    const float R[3][3] = {{c0.x, c1.x, c2.x}, {c0.y, c1.y, c2.y}, {c0.z, c1.z, c2.z}};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            float acc = 0.0f;
            for (int k = 0; k < 3; ++k)
                for (int l2 = 0; l2 < 3; ++l2) acc = fmaf(R[i][k] * Ib[k][l2], R[j][l2], acc);
            Iw[i][j] = acc;
        }
    for (int e = 0; e < 21; ++e) I6[e] = 0.0f;
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j <= i; ++j) I6[sym6(i, j)] = Iw[i][j];
        I6[sym6(3 + i, 3 + i)] = m;
    }
}

// ---------------------------------------------------------------------------
// Articulated-body algorithm (ArticulatedABA.metal:352-1578): per-body COM
// frames in world axes, classical accelerations, 21-entry inertias; tree
// levels run lane-parallel.  Each body shifts its articulated inertia and
// bias into its parent's frame; parents pull their children's shifted
// contributions in a fixed order, so sums are deterministic without atomics.
// ---------------------------------------------------------------------------
__device__ bool aba(const Warp& w) {
    const DeviceModel& M = *w.M;
    const WarpLayout& L = *w.L;
    float* s = w.s;
    float* misc = s + L.misc;
    const float* q = s + L.q;
    const float* v = s + L.v;
    const float* tau = s + L.tau;
    float* qdd = s + L.qdd;
    float* pose = s + L.body_pose;
    float* V = s + L.body_V;     // (omega, v_com)
    float* CV = s + L.body_CV;   // bias accelerations (angular, linear)
    float* IA = s + L.body_IA;
    float* PA = s + L.body_PA;
    float* U = s + L.body_U;
    float* Du = s + L.body_Du;
    float* A = s + L.body_A;
    float* R = s + L.body_r;     // parent COM -> body COM
    float* S = s + L.dof_S;      // motion subspace about the moving body's COM
    float* J = s + L.dof_J;      // joint axis (3), origin (3), prismatic flag
    const int lane = w.lane;

    // Non-finite inputs fail the step before any use
    // (ArticulatedABA.metal:640-662).
    for (int i = lane; i < M.nq; i += 32)
        if (!isfinite(q[i])) set_status(misc, MR_STEP_NONFINITE_INPUT, static_cast<unsigned>(i));
    for (int i = lane; i < M.nv; i += 32)
        if (!isfinite(v[i]) || !isfinite(tau[i])) set_status(misc, MR_STEP_NONFINITE_INPUT, static_cast<unsigned>(i));
    __syncwarp();
    if (as_int(misc[kMiscStatus]) != MR_STEP_SUCCESS) return false;

    // Root pose and velocity; root-DoF subspaces and Jacobian axes.
    if (lane == 0) {
        if (M.floating) {
            float4 rq;
            const float3 c0 = f3(q[0], q[1], q[2]);
            if (!finite3(c0) || !qnormalize(make_float4(q[3], q[4], q[5], q[6]), rq, true)) {
                set_status(misc, MR_STEP_NONFINITE_INPUT, 0u);
            } else {
                st3(pose, c0);
                st4(pose + 4, rq);
                V[0] = v[3]; V[1] = v[4]; V[2] = v[5];
                V[3] = v[0]; V[4] = v[1]; V[5] = v[2];
            }
        } else {
            st3(pose, f3(0.0f, 0.0f, 0.0f));
            st4(pose + 4, make_float4(0.0f, 0.0f, 0.0f, 1.0f));
            for (int i = 0; i < 6; ++i) V[i] = 0.0f;
        }
        pose[3] = 0.0f;
        for (int i = 0; i < 6; ++i) CV[i] = 0.0f;
        R[0] = R[1] = R[2] = 0.0f;
    }
    __syncwarp();
    if (as_int(misc[kMiscStatus]) != MR_STEP_SUCCESS) return false;
    if (M.floating && lane < 6) {
        float* Sd = S + lane * 6;
        float* Jd = J + lane * 8;
        for (int i = 0; i < 6; ++i) Sd[i] = 0.0f;
        // lin DoF k -> (0, e_k); ang DoF k -> (e_k, 0) about the root COM.
        if (lane < 3) Sd[3 + lane] = 1.0f;
        else Sd[lane - 3] = 1.0f;
        const int k = lane < 3 ? lane : lane - 3;
        Jd[0] = k == 0 ? 1.0f : 0.0f;
        Jd[1] = k == 1 ? 1.0f : 0.0f;
        Jd[2] = k == 2 ? 1.0f : 0.0f;
        Jd[3] = pose[0]; Jd[4] = pose[1]; Jd[5] = pose[2];
        Jd[6] = lane < 3 ? 1.0f : 0.0f;  // translational root DoFs act like prismatic axes
        Jd[7] = 0.0f;
    }

    // Forward kinematics: poses, twists, subspaces, bias accelerations.
    for (int l = 0; l < M.n_levels; ++l) {
        const int off = M.level_offsets[l];
        const int cnt = M.level_offsets[l + 1] - off;
        if (lane < cnt) {
            const int b = M.level_bodies[off + lane];
            const int p = M.parent[b];
            const int d = M.body_dof[b];
            const int type = M.joint_type[b];
            const float3 cp = ld3(pose + p * 8);
            const float4 qp = ld4(pose + p * 8 + 4);
            const float4 pj = qmul(qp, M.parent_rotation[b]);
            const float3 axis = xyz(M.axis[b]);
            float4 motion = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
            float qj = 0.0f, qdj = 0.0f;
            if (d >= 0) {
                qj = q[M.dof_q[d]];
                qdj = v[d];
                if (type == MR_JOINT_REVOLUTE || type == MR_JOINT_CONTINUOUS) {
                    const float half = 0.5f * qj;
                    const float sh = sinf(half);
                    motion = make_float4(axis.x * sh, axis.y * sh, axis.z * sh, cosf(half));
                }
            }
            float4 qb;
            if (!qnormalize(qmul(qmul(pj, motion), M.child_rotation_conj[b]), qb, false)) {
                set_status(misc, MR_STEP_NONFINITE_RESULT, static_cast<unsigned>(b));
                qb = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
            }
            const float3 ja = qrot(pj, axis);
            const bool prismatic = type == MR_JOINT_PRISMATIC;
            const bool has = d >= 0;
            float3 jp = cp + qrot(qp, xyz(M.parent_anchor[b]));
            if (prismatic) jp = jp + ja * qj;
            const float3 ca = qrot(qb, xyz(M.child_anchor[b]));
            const float3 cb = jp - ca;
            const float3 ptj = jp - cp;
            st3(pose + b * 8, cb);
            pose[b * 8 + 3] = 0.0f;
            st4(pose + b * 8 + 4, qb);
            st3(R + b * 4, cb - cp);
            const float3 wp = f3(V[p * 6 + 0], V[p * 6 + 1], V[p * 6 + 2]);
            const float3 vp = f3(V[p * 6 + 3], V[p * 6 + 4], V[p * 6 + 5]);
            const float3 wb = wp + ((has && !prismatic) ? ja * qdj : f3(0.0f, 0.0f, 0.0f));
            const float3 vb = vp + cross3(wp, ptj) + (prismatic ? ja * qdj : f3(0.0f, 0.0f, 0.0f)) - cross3(wb, ca);
            const float3 ma = (has && !prismatic) ? ja : f3(0.0f, 0.0f, 0.0f);
            const float3 ml = prismatic ? ja : (has ? -cross3(ja, ca) : f3(0.0f, 0.0f, 0.0f));
            const float3 ba = (has && !prismatic) ? cross3(wp, ja) * qdj : f3(0.0f, 0.0f, 0.0f);
            const float3 pc = prismatic ? cross3(wp, ja) * (2.0f * qdj) : f3(0.0f, 0.0f, 0.0f);
            const float3 bl = cross3(wp, cross3(wp, ptj)) + pc - cross3(ba, ca) - cross3(wb, cross3(wb, ca));
            V[b * 6 + 0] = wb.x; V[b * 6 + 1] = wb.y; V[b * 6 + 2] = wb.z;
            V[b * 6 + 3] = vb.x; V[b * 6 + 4] = vb.y; V[b * 6 + 5] = vb.z;
            CV[b * 6 + 0] = ba.x; CV[b * 6 + 1] = ba.y; CV[b * 6 + 2] = ba.z;
            CV[b * 6 + 3] = bl.x; CV[b * 6 + 4] = bl.y; CV[b * 6 + 5] = bl.z;
            if (has) {
                float* Sd = S + d * 6;
                Sd[0] = ma.x; Sd[1] = ma.y; Sd[2] = ma.z;
                Sd[3] = ml.x; Sd[4] = ml.y; Sd[5] = ml.z;
                float* Jd = J + d * 8;
                Jd[0] = ja.x; Jd[1] = ja.y; Jd[2] = ja.z;
                Jd[3] = jp.x; Jd[4] = jp.y; Jd[5] = jp.z;
                Jd[6] = prismatic ? 1.0f : 0.0f;
                Jd[7] = 0.0f;
            }
            if (!finite3(cb) || !finite3(wb) || !finite3(vb) || !finite3(bl))
                set_status(misc, MR_STEP_NONFINITE_RESULT, static_cast<unsigned>(b));
        }
        __syncwarp();
    }
    if (as_int(misc[kMiscStatus]) != MR_STEP_SUCCESS) return false;

    // Rigid inertia and velocity-dependent bias of every body about its COM.
    if (lane < M.nb) {
        const int b = lane;
        const float4 qb = ld4(pose + b * 8 + 4);
        const float4 md = M.mass_damping[b];
        float Iw[3][3];
        float* I6 = IA + b * 21;
        body_inertia(M, b, qb, I6, Iw);
        const float3 om = f3(V[b * 6 + 0], V[b * 6 + 1], V[b * 6 + 2]);
        const float3 vc = f3(V[b * 6 + 3], V[b * 6 + 4], V[b * 6 + 5]);
        const float3 Iom = f3(Iw[0][0] * om.x + Iw[0][1] * om.y + Iw[0][2] * om.z,
                              Iw[1][0] * om.x + Iw[1][1] * om.y + Iw[1][2] * om.z,
                              Iw[2][0] * om.x + Iw[2][1] * om.y + Iw[2][2] * om.z);
        float3 bt = cross3(om, Iom);
        float3 bf = -(md.x * f3(M.gravity[0], M.gravity[1], M.gravity[2]));
        if (M.apply_damping) {
            bt = bt + md.z * om;
            bf = bf + md.y * vc;
        }
        float* pa = PA + b * 6;
        pa[0] = bt.x; pa[1] = bt.y; pa[2] = bt.z; pa[3] = bf.x; pa[4] = bf.y; pa[5] = bf.z;
        if (b == 0 && M.floating) {
            for (int k = 0; k < 3; ++k) {
                I6[sym6(3 + k, 3 + k)] += M.armature_eff[k];
                I6[sym6(k, k)] += M.armature_eff[3 + k];
                pa[k] -= tau[3 + k];
                pa[3 + k] -= tau[k];
            }
        }
    }
    __syncwarp();

    // Backward sweep.
    for (int l = M.n_levels - 1; l >= 0; --l) {
        const int off = M.level_offsets[l];
        const int cnt = M.level_offsets[l + 1] - off;
        if (lane < cnt) {
            const int b = M.level_bodies[off + lane];
            float* I6 = IA + b * 21;
            float* pa = PA + b * 6;
            for (int k = M.child_offsets[b]; k < M.child_offsets[b + 1]; ++k) {
                const int c = M.children[k];
                for (int e = 0; e < 21; ++e) I6[e] += IA[c * 21 + e];
                for (int e = 0; e < 6; ++e) pa[e] += PA[c * 6 + e];
            }
            const int d = M.body_dof[b];
            float prop[6], ic[6];
            sym6_mul(I6, CV + b * 6, ic);
            for (int e = 0; e < 6; ++e) prop[e] = pa[e] + ic[e];
            if (d >= 0) {
                const float* sd = S + d * 6;
                float u6[6];
                sym6_mul(I6, sd, u6);
                const float D = dot6(sd, u6) + M.armature_eff[d];
                float maxI = 0.0f;
                for (int e = 0; e < 21; ++e) maxI = fmaxf(maxI, fabsf(I6[e]));
                const float floor = fmaxf(kAbsolutePivotFloor, maxI * 6.0f * kFloatEps);
                if (!(D > floor) || !isfinite(D)) {
                    set_status(misc, MR_STEP_FACTORIZATION_FAILED, static_cast<unsigned>(d));
                } else {
                    const float u = tau[d] - dot6(sd, prop);
                    const float invD = 1.0f / D;
                    for (int e = 0; e < 6; ++e) U[b * 6 + e] = u6[e];
                    Du[b * 2 + 0] = D;
                    Du[b * 2 + 1] = u;
                    for (int e = 0; e < 6; ++e) prop[e] += u6[e] * (u * invD);
                    for (int i = 0; i < 6; ++i)
                        for (int j = 0; j <= i; ++j) I6[sym6(i, j)] -= u6[i] * u6[j] * invD;
                }
            }
            // Contribution in the parent's frame, left in this body's slots.
            const float3 r = ld3(R + b * 4);
            float shifted[21];
            shift_inertia(I6, r, shifted);
            for (int e = 0; e < 21; ++e) I6[e] = shifted[e];
            const float3 pf = f3(prop[3], prop[4], prop[5]);
            const float3 pt = f3(prop[0], prop[1], prop[2]) + cross3(r, pf);
            pa[0] = pt.x; pa[1] = pt.y; pa[2] = pt.z; pa[3] = pf.x; pa[4] = pf.y; pa[5] = pf.z;
        }
        __syncwarp();
    }
    // Root: pull children (lane per entry), then solve the floating root.
    if (lane < 27) {
        float* dst = lane < 21 ? IA + lane : PA + (lane - 21);
        const int stride = lane < 21 ? 21 : 6;
        const float* src = lane < 21 ? IA : PA;
        const int e = lane < 21 ? lane : lane - 21;
        float acc = *dst;
        for (int k = M.child_offsets[0]; k < M.child_offsets[1]; ++k) acc += src[M.children[k] * stride + e];
        *dst = acc;
    }
    __syncwarp();
    if (lane == 0) {
        if (M.floating) {
            // 6x6 Cholesky of the root articulated inertia; a0 = -IA^-1 pA.
            float Lf[36];
            float maxI = 0.0f;
            for (int e = 0; e < 21; ++e) maxI = fmaxf(maxI, fabsf(IA[e]));
            const float floor = fmaxf(kAbsolutePivotFloor, maxI * 6.0f * kFloatEps);
            bool ok = true;
            for (int i = 0; i < 6 && ok; ++i) {
                for (int j = 0; j <= i; ++j) {
                    float val = IA[sym6(i, j)];
                    for (int k = 0; k < j; ++k) val -= Lf[i * 6 + k] * Lf[j * 6 + k];
                    if (i == j) {
                        if (!(val > floor) || !isfinite(val)) { ok = false; set_status(misc, MR_STEP_FACTORIZATION_FAILED, static_cast<unsigned>(i)); break; }
                        Lf[i * 6 + i] = sqrtf(val);
                    } else {
                        Lf[i * 6 + j] = val / Lf[j * 6 + j];
                    }
                }
            }
            if (ok) {
                float y[6], x[6];
                for (int i = 0; i < 6; ++i) {
                    float val = -PA[i];
                    for (int k = 0; k < i; ++k) val -= Lf[i * 6 + k] * y[k];
                    y[i] = val / Lf[i * 6 + i];
                }
                for (int i = 5; i >= 0; --i) {
                    float val = y[i];
                    for (int k = i + 1; k < 6; ++k) val -= Lf[k * 6 + i] * x[k];
                    x[i] = val / Lf[i * 6 + i];
                }
                for (int i = 0; i < 6; ++i) A[i] = x[i];
                qdd[0] = x[3]; qdd[1] = x[4]; qdd[2] = x[5];
                qdd[3] = x[0]; qdd[4] = x[1]; qdd[5] = x[2];
            }
        } else {
            for (int i = 0; i < 6; ++i) A[i] = 0.0f;
        }
    }
    __syncwarp();
    if (as_int(misc[kMiscStatus]) != MR_STEP_SUCCESS) return false;

    // Forward acceleration sweep.
    for (int l = 0; l < M.n_levels; ++l) {
        const int off = M.level_offsets[l];
        const int cnt = M.level_offsets[l + 1] - off;
        if (lane < cnt) {
            const int b = M.level_bodies[off + lane];
            const int p = M.parent[b];
            const int d = M.body_dof[b];
            const float3 r = ld3(R + b * 4);
            const float3 pa_ = f3(A[p * 6 + 0], A[p * 6 + 1], A[p * 6 + 2]);
            const float3 pl = f3(A[p * 6 + 3], A[p * 6 + 4], A[p * 6 + 5]) + cross3(pa_, r);
            float3 ang = pa_ + f3(CV[b * 6 + 0], CV[b * 6 + 1], CV[b * 6 + 2]);
            float3 lin = pl + f3(CV[b * 6 + 3], CV[b * 6 + 4], CV[b * 6 + 5]);
            if (d >= 0) {
                const float* Ub = U + b * 6;
                const float proj = Ub[0] * pa_.x + Ub[1] * pa_.y + Ub[2] * pa_.z + Ub[3] * pl.x + Ub[4] * pl.y + Ub[5] * pl.z;
                const float acc = (Du[b * 2 + 1] - proj) / Du[b * 2 + 0];
                qdd[d] = acc;
                const float* sd = S + d * 6;
                ang = ang + f3(sd[0], sd[1], sd[2]) * acc;
                lin = lin + f3(sd[3], sd[4], sd[5]) * acc;
            }
            A[b * 6 + 0] = ang.x; A[b * 6 + 1] = ang.y; A[b * 6 + 2] = ang.z;
            A[b * 6 + 3] = lin.x; A[b * 6 + 4] = lin.y; A[b * 6 + 5] = lin.z;
        }
        __syncwarp();
    }
    // v_free = v + h qdd.
    float* vf = s + L.vf;
    for (int d = lane; d < M.nv; d += 32) {
        const float a = qdd[d];
        const float nvv = v[d] + M.h * a;
        if (!isfinite(a) || !isfinite(nvv)) set_status(misc, MR_STEP_NONFINITE_RESULT, static_cast<unsigned>(d));
        vf[d] = nvv;
    }
    __syncwarp();
    return as_int(misc[kMiscStatus]) == MR_STEP_SUCCESS;
}

// Free-motion commit of the ABA candidate (ArticulatedABA.metal:1466-1540):
// v' = v_free, joints q' = q + h v', root exponential map with the angle
// reduced modulo 2 pi.
__device__ bool integrate_free(const Warp& w) {
    const DeviceModel& M = *w.M;
    const WarpLayout& L = *w.L;
    float* s = w.s;
    float* misc = s + L.misc;
    float* q = s + L.q;
    float* v = s + L.v;
    const float* vf = s + L.vf;
    for (int d = w.lane; d < M.nv; d += 32) {
        v[d] = vf[d];
        const int qi = M.dof_q[d];
        if (qi >= 0 && !(M.floating && d < 6)) {
            const float nq = q[qi] + M.h * vf[d];
            if (!isfinite(nq)) set_status(misc, MR_STEP_NONFINITE_RESULT, static_cast<unsigned>(qi));
            q[qi] = nq;
        }
    }
    if (M.floating && w.lane == 0) {
        q[0] += M.h * vf[0];
        q[1] += M.h * vf[1];
        q[2] += M.h * vf[2];
        const float4 inc = so3_increment(M.h * f3(vf[3], vf[4], vf[5]), true);
        float4 out;
        if (!qnormalize(qmul(inc, make_float4(q[3], q[4], q[5], q[6])), out, false)) {
            set_status(misc, MR_STEP_NONFINITE_RESULT, 3u);
        } else {
            q[3] = out.x; q[4] = out.y; q[5] = out.z; q[6] = out.w;
        }
        if (!isfinite(q[0]) || !isfinite(q[1]) || !isfinite(q[2])) set_status(misc, MR_STEP_NONFINITE_RESULT, 0u);
    }
    __syncwarp();
    return as_int(misc[kMiscStatus]) == MR_STEP_SUCCESS;
}

// ---------------------------------------------------------------------------
// Collision: collider projection, plane pair flag, analytic plane witnesses
// and persistent manifolds (Collision.metal:380-1000, 4379-4830, 5115-5560,
// 5712-6030, 9557-9830).  One lane owns one compiled pair.
// ---------------------------------------------------------------------------
struct RawContact {
    float3 normal;
    float sep;
    float3 pa, pb;
    unsigned fa, fb;
};

struct Candidate {
    float la[3], lb[3];
    unsigned fa, fb, life;
    float imp[3];
    float3 wp;
    float sep, drift;
};

__device__ __forceinline__ unsigned feature_key(unsigned type, unsigned local) {
    return ((type & 0x0fu) << 28u) | (local & 0x0fffffffu);
}
__device__ __forceinline__ unsigned long long cand_key(const Candidate& c) {
    return (static_cast<unsigned long long>(c.fa) << 32) | c.fb;
}
__device__ __forceinline__ bool cand_less(const Candidate& a, const Candidate& b) {
    if (a.sep != b.sep) return a.sep < b.sep;
    return cand_key(a) < cand_key(b);
}

__device__ __forceinline__ float3 stable_tangent(float3 n) {
    const float3 an = f3(fabsf(n.x), fabsf(n.y), fabsf(n.z));
    float3 ref;
    if (an.x <= an.y && an.x <= an.z) ref = f3(1.0f, 0.0f, 0.0f);
    else if (an.y <= an.z) ref = f3(0.0f, 1.0f, 0.0f);
    else ref = f3(0.0f, 0.0f, 1.0f);
    const float3 t = cross3(ref, n);
    return t * (1.0f / len3(t));
}

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
        o.body_pos = ld3(pose + b * 8);
        o.body_rot = ld4(pose + b * 8 + 4);
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

// Builds the new persistent manifold of one pair into `slot` (in/out).
// Returns the number of points, or -1 on a non-finite / overflow failure.
__device__ int pair_manifold(const DeviceModel& M, const float* pose, const float* margins, int pair, float* slot,
                             int& raw_count_out, bool& candidate_out) {
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
    RawContact raw[8];
    int nraw = 0;
    auto append = [&](float3 surface, float sep, unsigned ffeat) {
        const float3 pp = surface - plane.normal * sep;
        RawContact r;
        r.normal = -plane.normal;
        r.sep = sep;
        r.pa = surface;
        r.pb = pp;
        r.fa = ffeat;
        r.fb = feature_key(MR_SHAPE_PLANE, 0u);
        if (a_plane) {  // swapped orientation: A is the plane
            r.normal = plane.normal;
            r.pa = pp;
            r.pb = surface;
            r.fa = feature_key(MR_SHAPE_PLANE, 0u);
            r.fb = ffeat;
        }
        raw[nraw++] = r;
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
    for (int i = 0; i < nraw; ++i)
        if (!finite3(raw[i].normal) || !isfinite(raw[i].sep) || !finite3(raw[i].pa) || !finite3(raw[i].pb)) return -1;

    // buildPersistentWorldManifold.
    int deepest = 0;
    for (int i = 1; i < nraw; ++i) {
        const RawContact& l = raw[i];
        const RawContact& r = raw[deepest];
        if (l.sep < r.sep || (l.sep == r.sep && (l.fa < r.fa || (l.fa == r.fa && l.fb < r.fb)))) deepest = i;
    }
    float3 nw = raw[deepest].normal;
    nw = nw * (1.0f / len3(nw));
    if (!finite3(nw) || dot3(nw, nw) < 0.9999f) return -1;
    const float3 posA = A.body_pos, posB = B.body_pos;
    const float4 rotA = A.body_rot, rotB = B.body_rot;
    const float4 thr = make_float4(M.manifold_thresholds[0], M.manifold_thresholds[1], M.manifold_thresholds[2],
                                   M.manifold_thresholds[3]);
    Candidate cands[12];
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
                const float drift = len3(tan);
                if (sep > thr.x || drift > thr.y) continue;
                Candidate& c = cands[nc++];
                for (int k = 0; k < 3; ++k) { c.la[k] = op[k]; c.lb[k] = op[3 + k]; c.imp[k] = op[9 + k]; }
                c.fa = static_cast<unsigned>(as_int(op[6]));
                c.fb = static_cast<unsigned>(as_int(op[7]));
                const unsigned life = static_cast<unsigned>(as_int(op[8]));
                c.life = life == 0xffffffffu ? 0xffffffffu : life + 1u;
                c.wp = 0.5f * (pa + pb);
                c.sep = sep;
                c.drift = drift;
            }
        }
    }
    const float merge2 = thr.z * thr.z;
    for (int i = 0; i < nraw; ++i) {
        const RawContact& r = raw[i];
        const float3 la = qrotinv(rotA, r.pa - posA);
        const float3 lb = qrotinv(rotB, r.pb - posB);
        int match = -1;
        for (int k = 0; k < nc; ++k)
            if (cands[k].fa == r.fa && cands[k].fb == r.fb) { match = k; break; }
        if (match < 0) {
            for (int k = 0; k < nc; ++k) {
                const float3 da = f3(cands[k].la[0], cands[k].la[1], cands[k].la[2]) - la;
                const float3 db = f3(cands[k].lb[0], cands[k].lb[1], cands[k].lb[2]) - lb;
                if (dot3(da, da) + dot3(db, db) <= 2.0f * merge2) { match = k; break; }
            }
        }
        if (match < 0) {
            if (nc >= 12) return -1;
            match = nc++;
            Candidate& c = cands[match];
            c.life = 0u;
            c.imp[0] = c.imp[1] = c.imp[2] = 0.0f;
        }
        Candidate& c = cands[match];
        c.la[0] = la.x; c.la[1] = la.y; c.la[2] = la.z;
        c.lb[0] = lb.x; c.lb[1] = lb.y; c.lb[2] = lb.z;
        c.fa = r.fa;
        c.fb = r.fb;
        c.wp = 0.5f * (r.pa + r.pb);
        c.sep = r.sep;
        c.drift = 0.0f;
    }
    if (nc == 0) return -1;
    // reduceCandidates: sort by (separation, feature), pick 4 spread points,
    // then canonical feature order.
    for (int i = 1; i < nc; ++i) {
        Candidate val = cands[i];
        int d = i;
        while (d > 0 && cand_less(val, cands[d - 1])) { cands[d] = cands[d - 1]; --d; }
        cands[d] = val;
    }
    if (nc > kManifoldPoints) {
        bool selected[12];
        for (int i = 0; i < 12; ++i) selected[i] = false;
        int chosen[kManifoldPoints];
        chosen[0] = 0;
        selected[0] = true;
        int chosen_count = 1;
        for (int stage = 1; stage < kManifoldPoints; ++stage) {
            int best = -1;
            float best_score = -1.0f;
            unsigned long long best_feature = ~0ull;
            for (int i = 0; i < nc; ++i) {
                if (selected[i]) continue;
                float score;
                if (stage == 1) {
                    const float3 dl = cands[i].wp - cands[chosen[0]].wp;
                    const float3 t = dl - nw * dot3(dl, nw);
                    score = dot3(t, t);
                } else if (stage == 2) {
                    const float3 a = cands[chosen[1]].wp - cands[chosen[0]].wp;
                    const float3 bb = cands[i].wp - cands[chosen[0]].wp;
                    score = fabsf(dot3(cross3(a, bb), nw));
                } else {
                    score = INFINITY;
                    for (int k = 0; k < chosen_count; ++k) {
                        const float3 dl = cands[i].wp - cands[chosen[k]].wp;
                        const float3 t = dl - nw * dot3(dl, nw);
                        score = fminf(score, dot3(t, t));
                    }
                }
                const unsigned long long f = cand_key(cands[i]);
                if (score > best_score + 1.0e-12f || (fabsf(score - best_score) <= 1.0e-12f && f < best_feature)) {
                    best = i;
                    best_score = score;
                    best_feature = f;
                }
            }
            if (best >= 0) {
                chosen[chosen_count++] = best;
                selected[best] = true;
            }
        }
        Candidate reduced[kManifoldPoints];
        for (int i = 0; i < chosen_count; ++i) reduced[i] = cands[chosen[i]];
        nc = chosen_count;
        for (int i = 0; i < nc; ++i) cands[i] = reduced[i];
    }
    for (int i = 1; i < nc; ++i) {
        Candidate val = cands[i];
        const unsigned long long f = cand_key(val);
        int d = i;
        while (d > 0 && f < cand_key(cands[d - 1])) { cands[d] = cands[d - 1]; --d; }
        cands[d] = val;
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
            const Candidate& c = cands[i];
            for (int k = 0; k < 3; ++k) { op[k] = c.la[k]; op[3 + k] = c.lb[k]; op[9 + k] = c.imp[k]; }
            op[6] = as_float(static_cast<int>(c.fa));
            op[7] = as_float(static_cast<int>(c.fb));
            op[8] = as_float(static_cast<int>(c.life));
        } else {
            for (int k = 0; k < 12; ++k) op[k] = 0.0f;
        }
    }
    return nc;
}

__device__ __forceinline__ float3 project_cone(float3 imp, float mu_u, float mu_v) {
    float3 p = imp;
    p.x = fmaxf(p.x, 0.0f);
    const float lu = mu_u * p.x;
    const float lv = mu_v * p.x;
    if (!(lu > 0.0f) || !(lv > 0.0f)) {
        p.y = 0.0f;
        p.z = 0.0f;
        return p;
    }
    const float ns = (p.y * p.y) / (lu * lu) + (p.z * p.z) / (lv * lv);
    if (ns > 1.0f) {
        const float sc = rsqrtf(ns);
        p.y *= sc;
        p.z *= sc;
    }
    return p;
}

// Regularised inverse of the coupled 3x3 contact block (invert3x3,
// MetalWorldContact.metal:540-623): symmetrise, scale-normalise, add a 1 %
// CFM floor, invert by cofactors.
__device__ bool invert3x3_reg(const float m[3][3], float inv[3][3]) {
    float scale = 0.0f;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            if (!isfinite(m[i][j])) return false;
            scale = fmaxf(scale, fabsf(m[i][j]));
        }
    if (!(scale > kMatrixFloor)) return false;
    float r[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r[i][j] = 0.5f * (m[i][j] + m[j][i]) / scale + (i == j ? kContactCfm : 0.0f);
    const float c00 = r[1][1] * r[2][2] - r[1][2] * r[2][1];
    const float c01 = r[1][2] * r[2][0] - r[1][0] * r[2][2];
    const float c02 = r[1][0] * r[2][1] - r[1][1] * r[2][0];
    const float det = r[0][0] * c00 + r[0][1] * c01 + r[0][2] * c02;
    if (!(det > kMatrixFloor) || !isfinite(det)) return false;
    const float rc = 1.0f / (det * scale);
    inv[0][0] = c00 * rc;
    inv[0][1] = (r[0][2] * r[2][1] - r[0][1] * r[2][2]) * rc;
    inv[0][2] = (r[0][1] * r[1][2] - r[0][2] * r[1][1]) * rc;
    inv[1][0] = c01 * rc;
    inv[1][1] = (r[0][0] * r[2][2] - r[0][2] * r[2][0]) * rc;
    inv[1][2] = (r[0][2] * r[1][0] - r[0][0] * r[1][2]) * rc;
    inv[2][0] = c02 * rc;
    inv[2][1] = (r[0][1] * r[2][0] - r[0][0] * r[2][1]) * rc;
    inv[2][2] = (r[0][0] * r[1][1] - r[0][1] * r[1][0]) * rc;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            if (!isfinite(inv[i][j])) return false;
    return true;
}

// ---------------------------------------------------------------------------
// Contact substep after the ABA: collision, ConstraintIR evaluation, mass
// factor and response columns, temporalCone solve, joint limits, integration.
// ---------------------------------------------------------------------------
__device__ bool contact_substep(const Warp& w, bool final_substep, int velocity_iterations, int final_iterations,
                                float friction_scale) {
    const DeviceModel& M = *w.M;
    const WarpLayout& L = *w.L;
    float* s = w.s;
    float* misc = s + L.misc;
    const int lane = w.lane;
    const int nv = M.nv;
    const float h = M.h;
    float* pose = s + L.body_pose;
    float* q = s + L.q;
    float* v = s + L.v;
    const float* vf = s + L.vf;
    float* S = s + L.dof_S;
    float* slots = s + L.manifolds;
    float* C = s + L.contacts;
    float* G = s + L.G;
    float* R = s + L.R;
    float* Lm = s + L.L;
    const int rs = L.rstride;
    const int ma = M.max_anc;
    const float* Jax = s + L.dof_J;

    // Speculative margins of articulated colliders (Collision.metal:5882-5915):
    // h * sum|v_free| * max(sweep radius, 0.25), capped by h * speed envelope.
    float gs = 0.0f;
    for (int d = lane; d < nv; d += 32) gs += fabsf(vf[d]);
    gs = warp_sum(gs);
    // Per-shape margins live in the tau array's tail? Use registers: lane s holds margin of shape s.
    float my_margin = 0.0f;
    if (lane < M.ns && M.shape_body[lane] >= 0 && M.shape_type[lane] != MR_SHAPE_PLANE) {
        const float env = fminf(h * gs * fmaxf(M.shape_offsets[lane].z, 0.25f), h * M.speed_envelope);
        my_margin = M.speculative_scale * env;
    }
    // Stage margins in shared memory (R area is free at this point).
    float* margins = R;
    if (lane < M.ns) margins[lane] = my_margin;
    __syncwarp();

    // Narrowphase + manifolds: lane per pair.
    int npoints = 0, nraw = 0;
    bool cand = false;
    bool pair_fail = false;
    if (lane < M.np) {
        npoints = pair_manifold(M, pose, margins, lane, slots + lane * kManifoldWords, nraw, cand);
        if (npoints < 0) { pair_fail = true; npoints = 0; }
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
        const int raw_total = static_cast<int>(warp_sum(static_cast<float>(nraw)));
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

    // Contact records (mr_world_scatter_manifold_ir): one lane per pair
    // emits its points.
    if (lane < M.np && npoints > 0) {
        const int pair = lane;
        const float* slot = slots + pair * kManifoldWords;
        const int sa = M.pair_a[pair], sb = M.pair_b[pair];
        const int ba = M.shape_body[sa], bb = M.shape_body[sb];
        float3 posA, posB;
        float4 rotA, rotB;
        if (ba >= 0) { posA = ld3(pose + ba * 8); rotA = ld4(pose + ba * 8 + 4); }
        else { posA = xyz(M.static_body_position[sa]); rotA = M.static_body_rotation[sa]; }
        if (bb >= 0) { posB = ld3(pose + bb * 8); rotB = ld4(pose + bb * 8 + 4); }
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
            // Rows: target velocity (speculative gap), regularisation.
            c[kCwTarget + 0] = sep > 0.0f ? -sep / h : 0.0f;
            c[kCwTarget + 1] = 0.0f;
            c[kCwTarget + 2] = 0.0f;
            c[kCwReg + 0] = fmaxf(compliance / (h * h) + dissipation / h, 0.0f);
            c[kCwReg + 1] = 0.0f;
            c[kCwReg + 2] = 0.0f;
            c[kCwMuU] = mu_s;   // static coefficient; replaced by the slip test below
            c[kCwMuV] = mu_d;   // dynamic coefficient (temporarily)
            c[kCwRelax] = restitution;
            c[kCwDelta + 0] = rthreshold;
        }
    }
    __syncwarp();

    // Jacobian rows G (sparse over the body's ancestor DoFs) and evaluation
    // of the ConstraintIR rows at v_free (MetalWorldContact.metal:3580-3990).
    if (lane < total) {
        float* c = C + lane * kContactWords;
        const int b = as_int(c[kCwBody]);
        const int flags = as_int(c[kCwFlags]);
        const float sign = (flags & 256) ? 1.0f : -1.0f;
        const float3 x = ld3(c + kCwPoint);
        const float3 dirs[3] = {ld3(c + kCwNormal), ld3(c + kCwTangent), ld3(c + kCwBitangent)};
        const int na = M.anc_count[b];
        float* g = G + lane * 3 * ma;
        float rel[3] = {0.0f, 0.0f, 0.0f};
        for (int k = 0; k < na; ++k) {
            const int d = M.anc_dofs[b * kMaxDofs + k];
            // Point-Jacobian column: a x (x - o) for rotations, a for translations.
            const float* jd = Jax + d * 8;
            const float3 ax = f3(jd[0], jd[1], jd[2]);
            const float3 jc = jd[6] != 0.0f ? ax : cross3(ax, x - f3(jd[3], jd[4], jd[5]));
            for (int r = 0; r < 3; ++r) {
                const float gv = sign * dot3(dirs[r], jc);
                g[r * ma + k] = gv;
                rel[r] = fmaf(gv, vf[d], rel[r]);
            }
        }
        for (int k = na; k < ma; ++k)
            for (int r = 0; r < 3; ++r) g[r * ma + k] = 0.0f;
        // Normal row: critically damped stabilisation clamped to the maximum
        // depenetration speed, plus restitution on a new impact.
        const float sep = c[kCwSeparation];
        const float tau_c = 2.0f * h;
        const float err = fminf(sep + M.slop, 0.0f);
        const float ratio = h / tau_c;
        const float den = 1.0f + 2.0f * 1.0f * ratio + ratio * ratio;
        float stab = -h * err / (tau_c * tau_c * den);
        stab = fminf(fmaxf(fmaxf(stab, 0.0f), 0.0f), M.max_depenetration);
        const float restitution = c[kCwRelax];
        const float rthreshold = c[kCwDelta + 0];
        if (flags & 1) {
            const float incoming = rel[0] - c[kCwTarget + 0];
            if (incoming < -rthreshold) stab = fmaxf(stab, -restitution * incoming);
        }
        c[kCwTarget + 0] += stab;
        const float slip = sqrtf(rel[1] * rel[1] + rel[2] * rel[2]);
        const bool stat = slip <= fmaxf(1.0e-3f, 1.0e-3f);
        const float mu = stat ? c[kCwMuU] : c[kCwMuV];
        c[kCwMuU] = mu;
        c[kCwMuV] = mu;
        if (!isfinite(c[kCwTarget + 0]) || !isfinite(c[kCwReg + 0])) set_status(misc, MR_STEP_NONFINITE_RESULT, static_cast<unsigned>(lane));
    }
    __syncwarp();
    if (as_int(misc[kMiscStatus]) != MR_STEP_SUCCESS) return false;

    float* vv = v;  // solver velocity
    for (int d = lane; d < nv; d += 32) vv[d] = vf[d];
    if (total > 0) {
        if (lane == 0) misc[kMiscIslands] = as_float(max(as_int(misc[kMiscIslands]), 1));
        // Composite rigid-body inertias, each about its own body's COM:
        // rebuilt into the ABA inertia area, then children shifted into
        // their parent's frame and pulled level by level (deterministic).
        float* IC = s + L.body_IA;
        const float* Rr = s + L.body_r;
        if (lane < M.nb) {
            float Iw[3][3];
            body_inertia(M, lane, ld4(pose + lane * 8 + 4), IC + lane * 21, Iw);
        }
        __syncwarp();
        for (int l = M.n_levels - 1; l >= -1; --l) {
            const int off = l >= 0 ? M.level_offsets[l] : 0;
            const int cnt = l >= 0 ? M.level_offsets[l + 1] - off : 1;
            if (lane < cnt) {
                const int b = l >= 0 ? M.level_bodies[off + lane] : 0;
                float* I6 = IC + b * 21;
                for (int k = M.child_offsets[b]; k < M.child_offsets[b + 1]; ++k) {
                    const int c = M.children[k];
                    float shifted[21];
                    shift_inertia(IC + c * 21, ld3(Rr + c * 4), shifted);
                    for (int e = 0; e < 21; ++e) I6[e] += shifted[e];
                }
            }
            __syncwarp();
        }
        // Mass matrix (packed lower, tree DoF order): F = IC_body(i) S_i in
        // body(i)'s frame, moved to each ancestor DoF's body frame,
        // M_ij = S_j . F.  Entries of unrelated DoFs stay zero.
        for (int i = lane; i < nv; i += 32) {
            float* row = Lm + i * (i + 1) / 2;
            for (int j = 0; j <= i; ++j) row[j] = 0.0f;
            float F[6];
            const int bi = M.dof_body[i];
            sym6_mul(IC + bi * 21, S + i * 6, F);
            const float3 ci = ld3(pose + bi * 8);
            const float3 fl = f3(F[3], F[4], F[5]);
            const float3 fa = f3(F[0], F[1], F[2]);
            for (int j = i; j >= 0; j = M.dof_parent[j]) {
                const float3 cj = ld3(pose + M.dof_body[j] * 8);
                const float3 n = fa + cross3(ci - cj, fl);
                const float* sj = S + j * 6;
                row[j] = sj[0] * n.x + sj[1] * n.y + sj[2] * n.z + sj[3] * fl.x + sj[4] * fl.y + sj[5] * fl.z;
            }
            row[i] += M.armature_eff[i];
        }
        __syncwarp();
        // LTL factorisation H = L^T L exploiting the tree sparsity
        // (Featherstone, Rigid Body Dynamics Algorithms, sec. 6.5).
        for (int k = nv - 1; k >= 0; --k) {
            float* rowk = Lm + k * (k + 1) / 2;
            if (lane == 0) {
                const float dkk = rowk[k];
                if (!(dkk > kAbsolutePivotFloor) || !isfinite(dkk)) set_status(misc, MR_STEP_FACTORIZATION_FAILED, static_cast<unsigned>(k));
                rowk[k] = sqrtf(fmaxf(dkk, kAbsolutePivotFloor));
            }
            __syncwarp();
            const float lkk = rowk[k];
            const int* ancs = M.anc_dofs + M.dof_body[k] * kMaxDofs;
            const int nanc = M.dof_anc_count[k];
            for (int t = lane; t < nanc; t += 32) rowk[ancs[t]] /= lkk;
            __syncwarp();
            for (int t = lane; t < nanc; t += 32) {
                const int i = ancs[t];
                const float lki = rowk[i];
                float* rowi = Lm + i * (i + 1) / 2;
                for (int u = 0; u <= t; ++u) rowi[ancs[u]] -= lki * rowk[ancs[u]];
            }
            __syncwarp();
        }
        if (as_int(misc[kMiscStatus]) != MR_STEP_SUCCESS) return false;
        // Response columns R = H^-1 G^T: one lane per column.
        const int ncol = 3 * total;
        for (int col = lane; col < ncol; col += 32) {
            const int c = col / 3, r = col % 3;
            float* x = R + col * rs;
            for (int d = 0; d < nv; ++d) x[d] = 0.0f;
            const int b = as_int(C[c * kContactWords + kCwBody]);
            const int na = M.anc_count[b];
            const float* g = G + c * 3 * ma + r * ma;
            for (int k = 0; k < na; ++k) x[M.anc_dofs[b * kMaxDofs + k]] = g[k];
            // L^T y = b
            for (int k = nv - 1; k >= 0; --k) {
                const float* rowk = Lm + k * (k + 1) / 2;
                const float yk = x[k] / rowk[k];
                x[k] = yk;
                for (int i = M.dof_parent[k]; i >= 0; i = M.dof_parent[i]) x[i] -= rowk[i] * yk;
            }
            // L x = y
            for (int k = 0; k < nv; ++k) {
                const float* rowk = Lm + k * (k + 1) / 2;
                float acc = x[k];
                for (int i = M.dof_parent[k]; i >= 0; i = M.dof_parent[i]) acc -= rowk[i] * x[i];
                x[k] = acc / rowk[k];
            }
        }
        __syncwarp();
        // Preconditioners, relaxation and warm start (lane per contact).
        if (lane < total) {
            float* c = C + lane * kContactWords;
            const int b = as_int(c[kCwBody]);
            const int na = M.anc_count[b];
            const int* anc = M.anc_dofs + b * kMaxDofs;
            const float* g = G + lane * 3 * ma;
            float Wm[3][3];
            for (int r = 0; r < 3; ++r)
                for (int cc = 0; cc < 3; ++cc) {
                    const float* x = R + (lane * 3 + cc) * rs;
                    float acc = 0.0f;
                    for (int k = 0; k < na; ++k) acc = fmaf(g[r * ma + k], x[anc[k]], acc);
                    Wm[r][cc] = acc + (r == cc ? c[kCwReg + r] : 0.0f);
                }
            float inv[3][3];
            if (!invert3x3_reg(Wm, inv)) {
                set_status(misc, MR_STEP_FACTORIZATION_FAILED, static_cast<unsigned>(lane));
            } else {
                for (int r = 0; r < 3; ++r)
                    for (int cc = 0; cc < 3; ++cc) c[kCwPre + r * 3 + cc] = inv[r][cc];
            }
            float rowsum = 0.0f, diag = 0.0f;
            for (int c2 = 0; c2 < total; ++c2) {
                const float* x = R + (c2 * 3) * rs;
                float acc = 0.0f;
                for (int k = 0; k < na; ++k) acc = fmaf(g[k], x[anc[k]], acc);
                rowsum += fabsf(acc);
                if (c2 == lane) diag = fabsf(acc) + c[kCwReg + 0];
            }
            c[kCwRelax] = rowsum > fmaxf(diag, kMatrixFloor) ? fminf(fmaxf(diag / rowsum, 1.0f / 32.0f), 1.0f) : 1.0f;
            const float3 warm = project_cone(ld3(c + kCwLambda), c[kCwMuU], c[kCwMuV]);
            st3(c + kCwLambda, warm);
            st3(c + kCwDelta, warm);
        }
        __syncwarp();
        if (as_int(misc[kMiscStatus]) != MR_STEP_SUCCESS) return false;
        // Jacobi sweeps: lane per contact proposes, lane per DoF applies.
        const int iters = velocity_iterations + (final_substep ? final_iterations : 0);
        for (int it = -1; it < iters; ++it) {
            if (it >= 0 && lane < total) {
                float* c = C + lane * kContactWords;
                const int b = as_int(c[kCwBody]);
                const int na = M.anc_count[b];
                const int* anc = M.anc_dofs + b * kMaxDofs;
                const float* g = G + lane * 3 * ma;
                float u0 = 0.0f, u1 = 0.0f, u2 = 0.0f;
                for (int k = 0; k < na; ++k) {
                    const float vk = vv[anc[k]];
                    u0 = fmaf(g[k], vk, u0);
                    u1 = fmaf(g[ma + k], vk, u1);
                    u2 = fmaf(g[2 * ma + k], vk, u2);
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
            // it == -1 applies the warm start.
            for (int d = lane; d < nv; d += 32) {
                float acc = 0.0f;
                for (int c2 = 0; c2 < total; ++c2) {
                    const float* dl = C + c2 * kContactWords + kCwDelta;
                    acc = fmaf(R[(c2 * 3 + 0) * rs + d], dl[0], acc);
                    acc = fmaf(R[(c2 * 3 + 1) * rs + d], dl[1], acc);
                    acc = fmaf(R[(c2 * 3 + 2) * rs + d], dl[2], acc);
                }
                vv[d] += acc;
            }
            __syncwarp();
        }
        if (as_int(misc[kMiscStatus]) != MR_STEP_SUCCESS) return false;
        // Impulses back into the manifold points (warm start of the next substep).
        if (lane < total) {
            const float* c = C + lane * kContactWords;
            const int slot = as_int(c[kCwSlot]);
            float* op = slots + (slot >> 2) * kManifoldWords + 8 + (slot & 3) * 12;
            op[9] = c[kCwLambda + 0];
            op[10] = c[kCwLambda + 1];
            op[11] = c[kCwLambda + 2];
        }
    }
    __syncwarp();

    // Joint limits on the post-solve velocity (mr_world_project_joint_limits).
    for (int d = lane; d < nv; d += 32) {
        const unsigned flags = M.dof_flags[d];
        float vel = vv[d];
        if (flags & MR_DOF_FLAG_VELOCITY_LIMIT) vel = fminf(fmaxf(vel, -M.v_max[d]), M.v_max[d]);
        const int qi = M.dof_q[d];
        if ((flags & MR_DOF_FLAG_POSITION_LIMIT) && qi >= 0) {
            const float pos = q[qi];
            vel = fminf(fmaxf(vel, (M.q_lower[d] - pos) / h), (M.q_upper[d] - pos) / h);
        }
        if (!isfinite(vel)) set_status(misc, MR_STEP_NONFINITE_RESULT, static_cast<unsigned>(d));
        vv[d] = vel;
    }
    __syncwarp();
    // Integration from the substep-start configuration
    // (mr_world_integrate_contact_state; no angle reduction).
    for (int d = lane; d < nv; d += 32) {
        const int qi = M.dof_q[d];
        if (qi >= 0 && !(M.floating && d < 6)) q[qi] = q[qi] + h * vv[d];
    }
    if (M.floating && lane == 0) {
        q[0] += h * vv[0];
        q[1] += h * vv[1];
        q[2] += h * vv[2];
        const float4 inc = so3_increment(h * f3(vv[3], vv[4], vv[5]), false);
        const float4 src = make_float4(q[3], q[4], q[5], q[6]);
        const float4 prod = qmul(inc, src);
        float4 out;
        if (!finite4(prod) || !(qdot(prod, prod) > 1.0e-12f)) {
            set_status(misc, MR_STEP_NONFINITE_RESULT, 3u);
        } else {
            out = qscale(prod, rsqrtf(qdot(prod, prod)));
            q[3] = out.x; q[4] = out.y; q[5] = out.z; q[6] = out.w;
        }
    }
    __syncwarp();
    for (int i = lane; i < M.nq; i += 32)
        if (!isfinite(q[i])) set_status(misc, MR_STEP_NONFINITE_RESULT, static_cast<unsigned>(i));
    __syncwarp();
    return as_int(misc[kMiscStatus]) == MR_STEP_SUCCESS;
}

template <bool kContact>
__global__ void __launch_bounds__(128) control_step_kernel(StepParams p, WarpLayout layout, int warps_per_block) {
    extern __shared__ float4 smem4[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int env = blockIdx.x * warps_per_block + warp;
    if (env >= p.env_count) return;
    const DeviceModel& M = *p.model;
    Warp w;
    w.lane = lane;
    w.s = reinterpret_cast<float*>(smem4) + warp * layout.total;
    w.L = &layout;
    w.M = p.model;
    float* s = w.s;
    float* misc = s + layout.misc;
    const int nq = M.nq, nv = M.nv;

    // Prepare: reset, checkpoint, actions (mr_metal_world_prepare).
    const bool reset = p.reset_masks != nullptr && p.reset_masks[env] != 0u;
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
    if (lane < 32) misc[lane] = 0.0f;
    __syncwarp();
    for (int a = lane; a < M.action_count; a += 32)
        s[layout.tgt + M.action_dof[a]] = p.actions[static_cast<size_t>(env) * M.action_count + a];
    if (kContact) {
        float* slots = s + layout.manifolds;
        const int words = M.np * kManifoldWords;
        if (reset) {
            for (int i = lane; i < words; i += 32) slots[i] = 0.0f;
        } else {
            const float4* src = reinterpret_cast<const float4*>(p.manifolds + static_cast<size_t>(env) * words);
            float4* dst = reinterpret_cast<float4*>(slots);
            for (int i = lane; i < words / 4; i += 32) dst[i] = src[i];
        }
    }
    const float friction_scale = kContact ? p.friction_scale[env] : 1.0f;
    __syncwarp();

    int failing_substep = -1;
    for (int sub = 0; sub < p.substeps; ++sub) {
        compute_drives(w);
        __syncwarp();
        bool ok = aba(w);
        if (ok) {
            if (kContact)
                ok = contact_substep(w, sub + 1 == p.substeps, p.velocity_iterations, p.final_velocity_iterations, friction_scale);
            else
                ok = integrate_free(w);
        }
        if (!ok) {
            failing_substep = sub;
            break;
        }
    }
    const unsigned code = static_cast<unsigned>(as_int(misc[kMiscStatus]));
    const bool success = code == MR_STEP_SUCCESS;
    // Capture + commit: a failed step publishes (and keeps) its checkpoint.
    float* qd = p.q + static_cast<size_t>(env) * nq;
    float* vd = p.v + static_cast<size_t>(env) * nv;
    const float* qsrc = s + (success ? layout.q : layout.qc);
    const float* vsrc = s + (success ? layout.v : layout.vc);
    float* obs = p.observations ? p.observations + static_cast<size_t>(env) * (nq + nv) : nullptr;
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
    if (kContact && (success || reset)) {
        const int words = M.np * kManifoldWords;
        float4* dst = reinterpret_cast<float4*>(p.manifolds + static_cast<size_t>(env) * words);
        if (success) {
            const float4* src = reinterpret_cast<const float4*>(s + layout.manifolds);
            for (int i = lane; i < words / 4; i += 32) dst[i] = src[i];
        } else {
            for (int i = lane; i < words / 4; i += 32) dst[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
    }
    if (lane == 0) {
        const unsigned contacts = kContact ? static_cast<unsigned>(as_int(misc[kMiscContactCount])) : 0u;
        if (p.status_codes) p.status_codes[env] = code;
        if (p.active_contacts) p.active_contacts[env] = success ? contacts : 0u;
        if (!success) {
            atomicAdd(p.stats + kStatFailedEnvs, 1u);
            atomicMin(p.stats + kStatFirstFailEnv, static_cast<unsigned>(env));
        }
        if (reset) atomicAdd(p.stats + kStatResets, 1u);
        if (kContact) {
            atomicMax(p.stats + kStatMaxContacts, contacts);
            atomicMax(p.stats + kStatMaxManifolds, static_cast<unsigned>(as_int(misc[kMiscManifoldCount])));
            atomicMax(p.stats + kStatMaxRawContacts, static_cast<unsigned>(as_int(misc[kMiscRawCount])));
            atomicMax(p.stats + kStatMaxCandidatePairs, static_cast<unsigned>(as_int(misc[kMiscCandidatePairs])));
            atomicMax(p.stats + kStatMaxIslands, static_cast<unsigned>(as_int(misc[kMiscIslands])));
        }
        (void)failing_substep;
    }
}

}  // namespace

// Host launcher: one control step of `env_count` environments.
cudaError_t launch_control_step(const StepParams& p, const WarpLayout& layout, bool contact, int warps_per_block,
                                cudaStream_t stream) {
    const int blocks = (p.env_count + warps_per_block - 1) / warps_per_block;
    const size_t smem = static_cast<size_t>(layout.total) * sizeof(float) * warps_per_block;
    if (contact) {
        control_step_kernel<true><<<blocks, 32 * warps_per_block, smem, stream>>>(p, layout, warps_per_block);
    } else {
        control_step_kernel<false><<<blocks, 32 * warps_per_block, smem, stream>>>(p, layout, warps_per_block);
    }
    return cudaGetLastError();
}

cudaError_t configure_control_step_kernels(size_t max_dynamic_smem) {
    cudaError_t e = cudaFuncSetAttribute(control_step_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(max_dynamic_smem));
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(control_step_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(max_dynamic_smem));
}

}  // namespace numi
