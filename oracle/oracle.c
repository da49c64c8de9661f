/*
 * ORACLE — test infrastructure only (see oracle.h).  FP64 restatement of
 * numi-lab's microstep.  Function comments cite the reference file:line
 * each one follows.  Nothing here is part of the product library.
 */
#include "oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define MAXB MR_B200_MAX_BODIES
#define MAXV MR_B200_MAX_DOFS
#define MAXQ MR_B200_MAX_Q
#define MAXS MR_B200_MAX_SHAPES
#define MAXP MR_B200_MAX_PAIRS
#define MAXC MR_B200_MAX_CONTACTS
#define MPTS ((int)MR_B200_MANIFOLD_POINTS)

static const double kFloatEps = 1.1920928955078125e-7; /* float epsilon, as the reference's pivot floors */
static const double kPivotFloor = 1.0e-12;
static const double kMatrixFloor = 1.0e-10;
static const double kCfm = 1.0e-2;
static const double kPad = 0.00000762939453125;
/* Discrete decisions taken within this distance of their threshold are
 * "band" decisions: FP32 rounding on the device may legitimately take the
 * other branch.  Counted per control step (OracleTrace.band_decisions). */
static const double kBand = 1.0e-5;
static const double kTieRelative = 1.0e-5;  /* manifold reduction ties */
/* Piles: a device control step departs from the oracle's trajectory by up to
 * ~5e-6 m within its substeps (stacked contacts amplify FP32 rounding), so
 * their decisions use a wider band. */
static const double kSceneBand = 5.0e-5;
static __thread uint32_t g_band;
static __thread double g_band_width = 1.0e-5;
static __thread double g_margin;  /* smallest |value - threshold| over the step's decisions */
/* Rounding-noise mode (test infrastructure for per-step parity bounds):
 * with a non-zero state, rn() multiplies a value by (1 + d), d uniform in
 * [-2^-24, 2^-24], the relative error of one FP32 rounding to nearest --
 * Monte Carlo arithmetic (Parker, 1997).  Applied to the intermediates an
 * FP32 implementation rounds (body poses and twists, joint accelerations,
 * contact Jacobians and response terms, impulse and velocity updates,
 * integration), a few noisy runs estimate how far FP32 rounding alone can
 * move this step's result.  Zero (the default) is exact FP64. */
static __thread uint64_t g_noise;
static double rn(double x) {
    if (!g_noise) return x;
    g_noise ^= g_noise << 13;
    g_noise ^= g_noise >> 7;
    g_noise ^= g_noise << 17;
    const double u = (double)(g_noise >> 11) * (1.0 / 9007199254740992.0);
    return x * (1.0 + (2.0 * u - 1.0) * 5.9604644775390625e-08);
}
void oracle_set_rounding_noise(uint64_t seed) { g_noise = seed ? (seed | 1u) : 0u; }
#define BAND(value, threshold)                                                       \
    do {                                                                             \
        const double d_ = fabs((double)(value) - (double)(threshold));               \
        if (d_ < g_margin) g_margin = d_;                                            \
        if (d_ <= g_band_width) g_band++;                                            \
    } while (0)

struct OracleWorld {
    MRModelWorldC w;
    MRModelJointC joints[MAXB];
    MRModelBodyC bodies[MAXB + 8];
    MRModelDofC dofs[MAXV];
    MRModelShapeC shapes[MAXS];
    MRModelMaterialC materials[8];
    MRModelPairC pairs[MAXP];
    uint32_t nb;            /* articulated bodies */
    double h;
    uint32_t substeps, iters, final_iters;
    int floating;
    int body_dof[MAXB];     /* -1 when none */
    double arm_eff[MAXV];
    int action_dof[MAXV];
    int quality;            /* contacts solved to convergence (oracle_world_set_quality) */
    OracleQualityConfig qcfg;
};

/* ------------------------------------------------------------------ */
/* Small vector helpers                                                 */
/* ------------------------------------------------------------------ */
typedef struct { double x, y, z; } v3;
typedef struct { double x, y, z, w; } q4;

static v3 V(double x, double y, double z) { v3 r = {x, y, z}; return r; }
static v3 vadd(v3 a, v3 b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
static v3 vsub(v3 a, v3 b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
static v3 vmul(v3 a, double s) { return V(a.x * s, a.y * s, a.z * s); }
static double vdot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static v3 vcross(v3 a, v3 b) { return V(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static double vlen(v3 a) { return sqrt(vdot(a, a)); }
static double vmaxabs(v3 a) { return fmax(fmax(fabs(a.x), fabs(a.y)), fabs(a.z)); }
static int vfinite(v3 a) { return isfinite(a.x) && isfinite(a.y) && isfinite(a.z); }
static v3 vld(const double* p) { return V(p[0], p[1], p[2]); }
static v3 vldf(const float* p) { return V(p[0], p[1], p[2]); }
static void vst(double* p, v3 a) { p[0] = a.x; p[1] = a.y; p[2] = a.z; }
static double vget(v3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
static v3 rn3(v3 a) { return V(rn(a.x), rn(a.y), rn(a.z)); }

static q4 Q(double x, double y, double z, double w) { q4 r = {x, y, z, w}; return r; }
static q4 qconj(q4 q) { return Q(-q.x, -q.y, -q.z, q.w); }
static q4 qmul(q4 l, q4 r) {
    return Q(l.w * r.x + l.x * r.w + l.y * r.z - l.z * r.y, l.w * r.y - l.x * r.z + l.y * r.w + l.z * r.x,
             l.w * r.z + l.x * r.y - l.y * r.x + l.z * r.w, l.w * r.w - (l.x * r.x + l.y * r.y + l.z * r.z));
}
static v3 qrot(q4 q, v3 v) {
    const v3 u = V(q.x, q.y, q.z);
    const v3 t = vmul(vcross(u, v), 2.0);
    return vadd(vadd(v, vmul(t, q.w)), vcross(u, t));
}
static v3 qrotinv(q4 q, v3 v) { return qrot(qconj(q), v); }
static int qfinite(q4 q) { return isfinite(q.x) && isfinite(q.y) && isfinite(q.z) && isfinite(q.w); }
static double qdot(q4 a, q4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
static q4 qldf(const float* p) { return Q(p[0], p[1], p[2], p[3]); }

/* normalizedQuaternion (ArticulatedABA.metal:101-121). */
static int qnormalize(q4 in, q4* out, int require_unit) {
    if (!qfinite(in)) return 0;
    const double n2 = qdot(in, in);
    if (!(n2 > 1.0e-12) || !isfinite(n2)) return 0;
    const double n = sqrt(n2);
    if (require_unit && fabs(n - 1.0) > 2.0e-5) return 0;
    *out = Q(in.x / n, in.y / n, in.z / n, in.w / n);
    return qfinite(*out);
}

/* SO(3) exponential increment (ArticulatedABA.metal:1469-1481 with angle
 * reduction; MetalWorldContact.metal:8919-8930 without). */
static q4 so3_increment(v3 rv, int reduce) {
    const double angle = vlen(rv);
    const double two_pi = 6.28318530717958647692;
    const double reduced = (reduce && angle > two_pi) ? fmod(angle, two_pi) : angle;
    const double half = 0.5 * reduced;
    const double s = angle > 1.0e-6 ? sin(half) / angle : 0.5 - angle * angle / 48.0;
    return Q(rv.x * s, rv.y * s, rv.z * s, cos(half));
}

static int sym6(int i, int j) { return i >= j ? i * (i + 1) / 2 + j : j * (j + 1) / 2 + i; }

/* ------------------------------------------------------------------ */
/* World construction                                                   */
/* ------------------------------------------------------------------ */
OracleWorld* oracle_world_create(const MRModelWorldC* world, const MRModelJointC* joints, const MRModelBodyC* bodies,
                                 const MRModelDofC* dofs, const MRModelShapeC* shapes, const MRModelMaterialC* materials,
                                 const MRModelPairC* pairs, double h, uint32_t substeps, uint32_t velocity_iterations,
                                 uint32_t final_velocity_iterations) {
    if (!world || world->body_count > MAXB + 8 || world->nv > MAXV || world->nq > MAXQ || world->shape_count > MAXS ||
        world->pair_count > MAXP || world->material_count > 8)
        return NULL;
    OracleWorld* o = (OracleWorld*)calloc(1, sizeof(OracleWorld));
    if (!o) return NULL;
    o->w = *world;
    memcpy(o->joints, joints, sizeof(MRModelJointC) * world->joint_count);
    memcpy(o->bodies, bodies, sizeof(MRModelBodyC) * world->body_count);
    memcpy(o->dofs, dofs, sizeof(MRModelDofC) * world->nv);
    if (world->shape_count) memcpy(o->shapes, shapes, sizeof(MRModelShapeC) * world->shape_count);
    if (world->material_count) memcpy(o->materials, materials, sizeof(MRModelMaterialC) * world->material_count);
    if (world->pair_count) memcpy(o->pairs, pairs, sizeof(MRModelPairC) * world->pair_count);
    o->nb = 0;
    while (o->nb < world->body_count && bodies[o->nb].articulated) o->nb++;
    o->h = h;
    o->substeps = substeps;
    o->iters = velocity_iterations;
    o->final_iters = final_velocity_iterations;
    o->floating = world->root_type == MR_ROOT_FLOATING;
    for (uint32_t b = 0; b < MAXB; ++b) o->body_dof[b] = -1;
    for (uint32_t b = 1; b < o->nb; ++b) {
        const MRModelJointC* j = &joints[bodies[b].inbound_joint];
        if (j->joint_type != MR_JOINT_FIXED) o->body_dof[b] = (int)j->v_index;
    }
    const int implicit = world->actuation_mode == MR_ACTUATION_IMPLICIT_POSITION;
    int a = 0;
    for (uint32_t k = 0; k < world->nv; ++k) {
        /* effectiveArmature (ArticulatedABA.metal:301-316). */
        double arm = dofs[k].drive[2];
        if (implicit && (dofs[k].flags & MR_DOF_FLAG_DRIVE))
            arm += h * (double)dofs[k].drive[1] + h * h * (double)dofs[k].drive[0];
        o->arm_eff[k] = arm;
        if ((dofs[k].flags & MR_DOF_FLAG_ACTUATED) && a < (int)world->action_count) o->action_dof[a++] = (int)k;
    }
    return o;
}

void oracle_world_destroy(OracleWorld* world) { free(world); }

/* ------------------------------------------------------------------ */
/* Drives (MetalWorld.metal:280-370; default actuator profile of       */
/* MetalWorld.mm:1376-1411 makes the envelope min(limit, stall)).      */
/* ------------------------------------------------------------------ */
void oracle_drive_efforts(const OracleWorld* o, const double* q, const double* v, const double* actions, double* tau) {
    double tgt[MAXV];
    for (uint32_t k = 0; k < o->w.nv; ++k) tgt[k] = 0.0;
    for (uint32_t a = 0; a < o->w.action_count; ++a) tgt[o->action_dof[a]] = actions[a];
    const int implicit = o->w.actuation_mode == MR_ACTUATION_IMPLICIT_POSITION;
    for (uint32_t k = 0; k < o->w.nv; ++k) {
        const MRModelDofC* d = &o->dofs[k];
        const double vel = v[k];
        double command = tgt[k];
        if (implicit) {
            command = 0.0;
            if ((d->flags & MR_DOF_FLAG_DRIVE) && d->q_index != MR_INVALID_INDEX) {
                double target = tgt[k];
                if (d->flags & MR_DOF_FLAG_POSITION_LIMIT) target = fmin(fmax(target, d->limits[0]), d->limits[1]);
                command = d->drive[0] * (target - q[d->q_index] - o->h * vel) - d->drive[1] * vel;
                const double dry = d->drive[3];
                if (dry > 0.0) {
                    if (fabs(vel) > 1.0e-4) command -= copysign(dry, vel);
                    else command -= fmin(fmax(command, -dry), dry);
                }
                if ((d->flags & MR_DOF_FLAG_EFFORT_LIMIT) && d->limits[3] > 0.0f)
                    command = fmin(fmax(command, -d->limits[3]), d->limits[3]);
            }
        }
        const double stall = ((d->flags & MR_DOF_FLAG_EFFORT_LIMIT) && d->limits[3] > 0.0f) ? d->limits[3] : FLT_MAX;
        const double envelope = fmin(d->limits[3], stall);
        tau[k] = fmin(fmax(command, -envelope), envelope);
    }
}

/* ------------------------------------------------------------------ */
/* Kinematics + ABA in the reference formulation: per-body COM frames,  */
/* classical accelerations, 21-entry symmetric inertias, traversal in   */
/* joint order (ArticulatedABA.metal:352-1578).                        */
/* ------------------------------------------------------------------ */
typedef struct {
    v3 pos[MAXB];
    q4 rot[MAXB];
    v3 w[MAXB];
    v3 v[MAXB];
    v3 ma[MAXB], ml[MAXB];   /* motion subspace */
    v3 ba[MAXB], bl[MAXB];   /* velocity-product bias accelerations */
    v3 r[MAXB];              /* parent COM -> body COM */
    v3 joint_pos[MAXB];
    v3 joint_axis[MAXB];
} Kin;

static uint32_t kinematics(const OracleWorld* o, const double* q, const double* v, Kin* k) {
    const uint32_t nb = o->nb;
    for (uint32_t i = 0; i < o->w.nq; ++i)
        if (!isfinite(q[i])) return MR_STEP_NONFINITE_INPUT;
    for (uint32_t i = 0; i < o->w.nv; ++i)
        if (!isfinite(v[i])) return MR_STEP_NONFINITE_INPUT;
    if (o->floating) {
        q4 rq;
        const v3 p = V(q[0], q[1], q[2]);
        if (!vfinite(p) || !qnormalize(Q(q[3], q[4], q[5], q[6]), &rq, 1)) return MR_STEP_NONFINITE_INPUT;
        k->pos[0] = p;
        k->rot[0] = rq;
        k->v[0] = V(v[0], v[1], v[2]);
        k->w[0] = V(v[3], v[4], v[5]);
    } else {
        k->pos[0] = V(0, 0, 0);
        k->rot[0] = Q(0, 0, 0, 1);
        k->v[0] = V(0, 0, 0);
        k->w[0] = V(0, 0, 0);
    }
    k->r[0] = V(0, 0, 0);
    k->ma[0] = k->ml[0] = k->ba[0] = k->bl[0] = V(0, 0, 0);
    for (uint32_t b = 1; b < nb; ++b) {
        const MRModelJointC* j = &o->joints[o->bodies[b].inbound_joint];
        const uint32_t p = j->parent_body;
        q4 prot, crot;
        if (!qnormalize(qldf(j->parent_rotation), &prot, 1) || !qnormalize(qldf(j->child_rotation), &crot, 1))
            return MR_STEP_UNSUPPORTED;
        const q4 pj = qmul(k->rot[p], prot);
        v3 axis = V(1, 0, 0);
        q4 motion = Q(0, 0, 0, 1);
        double qj = 0.0, qdj = 0.0;
        const int dof = o->body_dof[b];
        if (dof >= 0) {
            axis = vldf(j->axis);
            axis = vmul(axis, 1.0 / vlen(axis));
            qj = q[j->q_index];
            qdj = v[dof];
            if (j->joint_type == MR_JOINT_REVOLUTE || j->joint_type == MR_JOINT_CONTINUOUS) {
                const double hh = 0.5 * qj;
                motion = Q(axis.x * sin(hh), axis.y * sin(hh), axis.z * sin(hh), cos(hh));
            }
        }
        q4 rc;
        if (!qnormalize(qmul(qmul(pj, motion), qconj(crot)), &rc, 0)) return MR_STEP_NONFINITE_RESULT;
        k->rot[b] = rc;
        const v3 ja = qrot(pj, axis);
        const int prismatic = j->joint_type == MR_JOINT_PRISMATIC;
        v3 jp = vadd(k->pos[p], qrot(k->rot[p], vldf(j->parent_anchor)));
        if (prismatic) jp = vadd(jp, vmul(ja, qj));
        const v3 ca = qrot(rc, vldf(j->child_anchor));
        k->pos[b] = vsub(jp, ca);
        k->r[b] = vsub(k->pos[b], k->pos[p]);
        k->joint_pos[b] = jp;
        k->joint_axis[b] = ja;
        const v3 ptj = vsub(jp, k->pos[p]);
        const int has = dof >= 0;
        k->w[b] = vadd(k->w[p], (!prismatic && has) ? vmul(ja, qdj) : V(0, 0, 0));
        k->v[b] = vsub(vadd(vadd(k->v[p], vcross(k->w[p], ptj)), prismatic ? vmul(ja, qdj) : V(0, 0, 0)), vcross(k->w[b], ca));
        k->ma[b] = (has && !prismatic) ? ja : V(0, 0, 0);
        k->ml[b] = prismatic ? ja : (has ? vmul(vcross(ja, ca), -1.0) : V(0, 0, 0));
        k->ba[b] = (has && !prismatic) ? vmul(vcross(k->w[p], ja), qdj) : V(0, 0, 0);
        const v3 pc = prismatic ? vmul(vcross(k->w[p], ja), 2.0 * qdj) : V(0, 0, 0);
        k->bl[b] = vsub(vsub(vadd(vcross(k->w[p], vcross(k->w[p], ptj)), pc), vcross(k->ba[b], ca)), vcross(k->w[b], vcross(k->w[b], ca)));
        if (g_noise) {
            k->pos[b] = rn3(k->pos[b]);
            k->r[b] = rn3(k->r[b]);
            k->w[b] = rn3(k->w[b]);
            k->v[b] = rn3(k->v[b]);
            k->bl[b] = rn3(k->bl[b]);
            k->ba[b] = rn3(k->ba[b]);
            k->rot[b] = Q(rn(k->rot[b].x), rn(k->rot[b].y), rn(k->rot[b].z), rn(k->rot[b].w));
        }
        if (!vfinite(k->pos[b]) || !vfinite(k->w[b]) || !vfinite(k->v[b]) || !vfinite(k->bl[b])) return MR_STEP_NONFINITE_RESULT;
    }
    return MR_STEP_SUCCESS;
}

/* World inertia about the COM: R I R^T. */
static void world_inertia(const MRModelBodyC* body, q4 rot, double Iw[3][3]) {
    const v3 c[3] = {qrot(rot, V(1, 0, 0)), qrot(rot, V(0, 1, 0)), qrot(rot, V(0, 0, 1))};
    double R[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) R[i][j] = vget(c[j], i);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double acc = 0.0;
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) acc += R[i][a] * (double)body->inertia[a][b] * R[j][b];
            Iw[i][j] = acc;
        }
}

static double mte(v3 r, int row, int col) { /* motionTransformElement (ArticulatedABA.metal:160-190) */
    if (row == col) return 1.0;
    if (row < 3 || col >= 3) return 0.0;
    const int lr = row - 3;
    if (lr == 0 && col == 1) return r.z;
    if (lr == 0 && col == 2) return -r.y;
    if (lr == 1 && col == 0) return -r.z;
    if (lr == 1 && col == 2) return r.x;
    if (lr == 2 && col == 0) return r.y;
    if (lr == 2 && col == 1) return -r.x;
    return 0.0;
}

static double spatial(v3 a, v3 l, int i) { return i < 3 ? vget(a, i) : vget(l, i - 3); }

static uint32_t aba_core(const OracleWorld* o, const double* q, const double* v, const double* tau, const Kin* k, double* qdd) {
    const uint32_t nb = o->nb;
    double IA[MAXB][21], PA[MAXB][6], U[MAXB][6], D[MAXB], Ures[MAXB];
    for (uint32_t b = 0; b < nb; ++b) {
        const MRModelBodyC* body = &o->bodies[b];
        double Iw[3][3];
        world_inertia(body, k->rot[b], Iw);
        for (int e = 0; e < 21; ++e) IA[b][e] = 0.0;
        for (int i = 0; i < 3; ++i) {
            for (int j = 0; j <= i; ++j) IA[b][sym6(i, j)] = Iw[i][j];
            IA[b][sym6(3 + i, 3 + i)] = body->mass_inverse_mass[0];
        }
        const double m = body->mass_inverse_mass[0];
        const v3 fext = vmul(V(o->w.gravity[0], o->w.gravity[1], o->w.gravity[2]), m);
        const v3 Iwv = V(Iw[0][0] * k->w[b].x + Iw[0][1] * k->w[b].y + Iw[0][2] * k->w[b].z,
                         Iw[1][0] * k->w[b].x + Iw[1][1] * k->w[b].y + Iw[1][2] * k->w[b].z,
                         Iw[2][0] * k->w[b].x + Iw[2][1] * k->w[b].y + Iw[2][2] * k->w[b].z);
        v3 bt = vcross(k->w[b], Iwv);
        v3 bf = vmul(fext, -1.0);
        if (o->w.apply_body_damping) {
            bt = vadd(bt, vmul(k->w[b], body->damping_speed[1]));
            bf = vadd(bf, vmul(k->v[b], body->damping_speed[0]));
        }
        for (int i = 0; i < 6; ++i) PA[b][i] = spatial(bt, bf, i);
    }
    if (o->floating) {
        for (int a = 0; a < 3; ++a) {
            IA[0][sym6(3 + a, 3 + a)] += o->arm_eff[a];
            IA[0][sym6(a, a)] += o->arm_eff[3 + a];
            PA[0][a] -= tau[3 + a];
            PA[0][3 + a] -= tau[a];
        }
    }
    for (uint32_t b = nb - 1; b >= 1; --b) {
        const uint32_t p = o->bodies[b].parent_body;
        double prop[6];
        for (int i = 0; i < 6; ++i) {
            double s = 0.0;
            for (int j = 0; j < 6; ++j) s += IA[b][sym6(i, j)] * spatial(k->ba[b], k->bl[b], j);
            prop[i] = PA[b][i] + s;
        }
        const int dof = o->body_dof[b];
        if (dof >= 0) {
            double S[6], Ub[6];
            for (int i = 0; i < 6; ++i) S[i] = spatial(k->ma[b], k->ml[b], i);
            for (int i = 0; i < 6; ++i) {
                double s = 0.0;
                for (int j = 0; j < 6; ++j) s += IA[b][sym6(i, j)] * S[j];
                Ub[i] = s;
            }
            double den = o->arm_eff[dof];
            for (int i = 0; i < 6; ++i) den += S[i] * Ub[i];
            double maxI = 0.0;
            for (int e = 0; e < 21; ++e) maxI = fmax(maxI, fabs(IA[b][e]));
            if (!(den > fmax(kPivotFloor, maxI * 6.0 * kFloatEps)) || !isfinite(den)) return MR_STEP_FACTORIZATION_FAILED;
            double res = tau[dof];
            for (int i = 0; i < 6; ++i) res -= S[i] * prop[i];
            D[b] = den;
            Ures[b] = res;
            for (int i = 0; i < 6; ++i) { U[b][i] = Ub[i]; prop[i] += Ub[i] * (res / den); }
            for (int i = 0; i < 6; ++i)
                for (int j = 0; j <= i; ++j) IA[b][sym6(i, j)] -= Ub[i] * Ub[j] / den;
        }
        const v3 r = k->r[b];
        for (int i = 0; i < 6; ++i)
            for (int j = 0; j <= i; ++j) {
                double t = 0.0;
                for (int l = 0; l < 6; ++l) {
                    const double xl = mte(r, l, i);
                    if (xl == 0.0) continue;
                    for (int m = 0; m < 6; ++m) t += xl * IA[b][sym6(l, m)] * mte(r, m, j);
                }
                IA[p][sym6(i, j)] += t;
            }
        v3 pt = V(prop[0], prop[1], prop[2]);
        const v3 pf = V(prop[3], prop[4], prop[5]);
        pt = vadd(pt, vcross(r, pf));
        for (int i = 0; i < 6; ++i) PA[p][i] += spatial(pt, pf, i);
    }
    v3 aa[MAXB], al[MAXB];
    if (o->floating) {
        double L[36] = {0}, y[6], x[6];
        double maxI = 0.0;
        for (int e = 0; e < 21; ++e) maxI = fmax(maxI, fabs(IA[0][e]));
        const double floor = fmax(kPivotFloor, maxI * 6.0 * kFloatEps);
        for (int i = 0; i < 6; ++i)
            for (int j = 0; j <= i; ++j) {
                double val = IA[0][sym6(i, j)];
                for (int m = 0; m < j; ++m) val -= L[i * 6 + m] * L[j * 6 + m];
                if (i == j) {
                    if (!(val > floor) || !isfinite(val)) return MR_STEP_FACTORIZATION_FAILED;
                    L[i * 6 + i] = sqrt(val);
                } else {
                    L[i * 6 + j] = val / L[j * 6 + j];
                }
            }
        for (int i = 0; i < 6; ++i) {
            double val = -PA[0][i];
            for (int m = 0; m < i; ++m) val -= L[i * 6 + m] * y[m];
            y[i] = val / L[i * 6 + i];
        }
        for (int i = 5; i >= 0; --i) {
            double val = y[i];
            for (int m = i + 1; m < 6; ++m) val -= L[m * 6 + i] * x[m];
            x[i] = val / L[i * 6 + i];
        }
        aa[0] = V(x[0], x[1], x[2]);
        al[0] = V(x[3], x[4], x[5]);
        qdd[0] = x[3]; qdd[1] = x[4]; qdd[2] = x[5];
        qdd[3] = x[0]; qdd[4] = x[1]; qdd[5] = x[2];
    } else {
        aa[0] = al[0] = V(0, 0, 0);
    }
    for (uint32_t b = 1; b < nb; ++b) {
        const uint32_t p = o->bodies[b].parent_body;
        const v3 tpa = aa[p];
        const v3 tpl = vadd(al[p], vcross(aa[p], k->r[b]));
        v3 ang = vadd(tpa, k->ba[b]);
        v3 lin = vadd(tpl, k->bl[b]);
        const int dof = o->body_dof[b];
        if (dof >= 0) {
            double pp = 0.0;
            for (int i = 0; i < 6; ++i) pp += U[b][i] * spatial(tpa, tpl, i);
            const double acc = (Ures[b] - pp) / D[b];
            qdd[dof] = acc;
            ang = vadd(ang, vmul(k->ma[b], acc));
            lin = vadd(lin, vmul(k->ml[b], acc));
        }
        aa[b] = ang;
        al[b] = lin;
    }
    for (uint32_t d = 0; d < o->w.nv; ++d) {
        qdd[d] = rn(qdd[d]);
        if (!isfinite(qdd[d])) return MR_STEP_NONFINITE_RESULT;
    }
    (void)q; (void)v;
    return MR_STEP_SUCCESS;
}

uint32_t oracle_aba(const OracleWorld* o, const double* q, const double* v, const double* tau, double* qdd) {
    Kin k;
    const uint32_t st = kinematics(o, q, v, &k);
    if (st != MR_STEP_SUCCESS) return st;
    return aba_core(o, q, v, tau, &k, qdd);
}

/* ------------------------------------------------------------------ */
/* Point Jacobians and the dense mass matrix (analytic tree Jacobians, */
/* as the reference operator's point-Jacobian mode,                     */
/* ArticulatedOperator.metal:1139, and M = sum_b J_b^T I_b J_b).        */
/* ------------------------------------------------------------------ */
static void point_jacobian_k(const OracleWorld* o, const Kin* k, uint32_t body, v3 x, double* J /* 3 x nv */) {
    const uint32_t nv = o->w.nv;
    for (uint32_t i = 0; i < 3 * nv; ++i) J[i] = 0.0;
    uint32_t b = body;
    while (b != 0 && b != MR_INVALID_INDEX) {
        const int dof = o->body_dof[b];
        if (dof >= 0) {
            const MRModelJointC* j = &o->joints[o->bodies[b].inbound_joint];
            v3 col;
            if (j->joint_type == MR_JOINT_PRISMATIC) col = k->joint_axis[b];
            else col = vcross(k->joint_axis[b], vsub(x, k->joint_pos[b]));
            J[0 * nv + dof] = col.x; J[1 * nv + dof] = col.y; J[2 * nv + dof] = col.z;
        }
        b = o->bodies[b].parent_body;
    }
    if (o->floating) {
        const v3 rr = vsub(x, k->pos[0]);
        for (int a = 0; a < 3; ++a) {
            J[a * nv + a] = 1.0;
            const v3 e = V(a == 0, a == 1, a == 2);
            const v3 col = vcross(e, rr);
            J[0 * nv + 3 + a] = col.x; J[1 * nv + 3 + a] = col.y; J[2 * nv + 3 + a] = col.z;
        }
    }
}

static void angular_jacobian_k(const OracleWorld* o, const Kin* k, uint32_t body, double* J /* 3 x nv */) {
    const uint32_t nv = o->w.nv;
    for (uint32_t i = 0; i < 3 * nv; ++i) J[i] = 0.0;
    uint32_t b = body;
    while (b != 0 && b != MR_INVALID_INDEX) {
        const int dof = o->body_dof[b];
        if (dof >= 0) {
            const MRModelJointC* j = &o->joints[o->bodies[b].inbound_joint];
            if (j->joint_type != MR_JOINT_PRISMATIC) {
                J[0 * nv + dof] = k->joint_axis[b].x; J[1 * nv + dof] = k->joint_axis[b].y; J[2 * nv + dof] = k->joint_axis[b].z;
            }
        }
        b = o->bodies[b].parent_body;
    }
    if (o->floating)
        for (int a = 0; a < 3; ++a) J[a * nv + 3 + a] = 1.0;
}

static void mass_matrix_k(const OracleWorld* o, const Kin* k, double* Mm) {
    const uint32_t nv = o->w.nv;
    double Jv[3 * MAXV], Jw[3 * MAXV];
    for (uint32_t i = 0; i < nv * nv; ++i) Mm[i] = 0.0;
    for (uint32_t b = 0; b < o->nb; ++b) {
        const double m = o->bodies[b].mass_inverse_mass[0];
        double Iw[3][3];
        world_inertia(&o->bodies[b], k->rot[b], Iw);
        point_jacobian_k(o, k, b, k->pos[b], Jv);
        angular_jacobian_k(o, k, b, Jw);
        if (b == 0 && !o->floating) continue;
        for (uint32_t i = 0; i < nv; ++i)
            for (uint32_t j = 0; j < nv; ++j) {
                double s = 0.0;
                for (int a = 0; a < 3; ++a) s += m * Jv[a * nv + i] * Jv[a * nv + j];
                for (int a = 0; a < 3; ++a)
                    for (int c = 0; c < 3; ++c) s += Jw[a * nv + i] * Iw[a][c] * Jw[c * nv + j];
                Mm[i * nv + j] += s;
            }
    }
}

/* World COM position, orientation (xyzw) and linear / angular velocity of
 * every articulated body ([nb][13]) from the kinematics pass: the task
 * layer's body states (LocomotionTask.metal reads bodyStates). */
uint32_t oracle_body_states(const OracleWorld* o, const double* q, const double* v, double* out) {
    Kin* k = (Kin*)malloc(sizeof(Kin));
    if (!k) return MR_STEP_UNSUPPORTED;
    const uint32_t st = kinematics(o, q, v, k);
    if (st == MR_STEP_SUCCESS)
        for (uint32_t b = 0; b < o->nb; ++b) {
            double* r = out + 13 * b;
            r[0] = k->pos[b].x; r[1] = k->pos[b].y; r[2] = k->pos[b].z;
            r[3] = k->rot[b].x; r[4] = k->rot[b].y; r[5] = k->rot[b].z; r[6] = k->rot[b].w;
            r[7] = k->v[b].x; r[8] = k->v[b].y; r[9] = k->v[b].z;
            r[10] = k->w[b].x; r[11] = k->w[b].y; r[12] = k->w[b].z;
        }
    free(k);
    return st;
}

uint32_t oracle_mass_matrix(const OracleWorld* o, const double* q, double* mass) {
    double v0[MAXV] = {0};
    Kin k;
    const uint32_t st = kinematics(o, q, v0, &k);
    if (st != MR_STEP_SUCCESS) return st;
    mass_matrix_k(o, &k, mass);
    return MR_STEP_SUCCESS;
}

uint32_t oracle_point_jacobian(const OracleWorld* o, const double* q, uint32_t body, const double* local_point,
                               double* world_point, double* jacobian) {
    double v0[MAXV] = {0};
    Kin k;
    const uint32_t st = kinematics(o, q, v0, &k);
    if (st != MR_STEP_SUCCESS) return st;
    const v3 x = vadd(k.pos[body], qrot(k.rot[body], vld(local_point)));
    vst(world_point, x);
    point_jacobian_k(o, &k, body, x, jacobian);
    return MR_STEP_SUCCESS;
}

/* ------------------------------------------------------------------ */
/* Contact math helpers                                                 */
/* ------------------------------------------------------------------ */
void oracle_project_cone(const double* imp, double mu_u, double mu_v, double* out) {
    /* projectFrictionCone (MetalWorldContact.metal:482-509); no normal cap. */
    double x = fmax(imp[0], 0.0), y = imp[1], z = imp[2];
    const double lu = mu_u * x, lv = mu_v * x;
    if (!(lu > 0.0) || !(lv > 0.0)) {
        out[0] = x; out[1] = 0.0; out[2] = 0.0;
        return;
    }
    const double ns = (y * y) / (lu * lu) + (z * z) / (lv * lv);
    if (ns > 1.0) {
        const double s = 1.0 / sqrt(ns);
        y *= s;
        z *= s;
    }
    out[0] = x; out[1] = y; out[2] = z;
}

int oracle_invert3x3(const double* m, double* inv) {
    /* invert3x3 (MetalWorldContact.metal:540-623). */
    double scale = 0.0;
    for (int i = 0; i < 9; ++i) {
        if (!isfinite(m[i])) return 0;
        scale = fmax(scale, fabs(m[i]));
    }
    if (!(scale > kMatrixFloor)) return 0;
    double r[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r[i][j] = 0.5 * (m[i * 3 + j] + m[j * 3 + i]) / scale + (i == j ? kCfm : 0.0);
    const double c00 = r[1][1] * r[2][2] - r[1][2] * r[2][1];
    const double c01 = r[1][2] * r[2][0] - r[1][0] * r[2][2];
    const double c02 = r[1][0] * r[2][1] - r[1][1] * r[2][0];
    const double det = r[0][0] * c00 + r[0][1] * c01 + r[0][2] * c02;
    if (!(det > kMatrixFloor) || !isfinite(det)) return 0;
    const double rc = 1.0 / (det * scale);
    inv[0] = c00 * rc;
    inv[1] = (r[0][2] * r[2][1] - r[0][1] * r[2][2]) * rc;
    inv[2] = (r[0][1] * r[1][2] - r[0][2] * r[1][1]) * rc;
    inv[3] = c01 * rc;
    inv[4] = (r[0][0] * r[2][2] - r[0][2] * r[2][0]) * rc;
    inv[5] = (r[0][2] * r[1][0] - r[0][0] * r[1][2]) * rc;
    inv[6] = c02 * rc;
    inv[7] = (r[0][1] * r[2][0] - r[0][0] * r[2][1]) * rc;
    inv[8] = (r[0][0] * r[1][1] - r[0][1] * r[1][0]) * rc;
    for (int i = 0; i < 9; ++i)
        if (!isfinite(inv[i])) return 0;
    return 1;
}

static v3 stable_tangent(v3 n) { /* Collision.metal:5133-5145 */
    const v3 a = V(fabs(n.x), fabs(n.y), fabs(n.z));
    v3 ref;
    if (a.x <= a.y && a.x <= a.z) ref = V(1, 0, 0);
    else if (a.y <= a.z) ref = V(0, 1, 0);
    else ref = V(0, 0, 1);
    const v3 t = vcross(ref, n);
    return vmul(t, 1.0 / vlen(t));
}

static uint32_t feature_key(uint32_t type, uint32_t local) { return ((type & 0x0fu) << 28u) | (local & 0x0fffffffu); }

/* ------------------------------------------------------------------ */
/* Collider projection and plane narrowphase (Collision.metal:380-1000, */
/* 4379-4830, speculative margins :5794-6030).                          */
/* ------------------------------------------------------------------ */
typedef struct {
    uint32_t type;
    v3 center;
    q4 rot;
    v3 body_pos;
    q4 body_rot;
    v3 lower, upper, half, ep0, ep1, normal;
    double radius, half_length, offset;
} Shape;

static void make_shape(const OracleWorld* o, const Kin* k, uint32_t sh, double margin, Shape* s) {
    const MRModelShapeC* src = &o->shapes[sh];
    const MRModelBodyC* body = &o->bodies[src->body];
    memset(s, 0, sizeof(*s));
    s->type = src->shape_type;
    q4 lr;
    qnormalize(qldf(src->local_rotation), &lr, 0);
    if (body->articulated) {
        s->body_pos = k->pos[src->body];
        s->body_rot = k->rot[src->body];
    } else {
        s->body_pos = vldf(body->static_pose);
        qnormalize(qldf(body->static_pose + 4), &s->body_rot, 0);
    }
    s->center = vadd(s->body_pos, qrot(s->body_rot, vldf(src->local_position)));
    s->rot = qmul(s->body_rot, lr);
    const double base = src->contact_rest_bound[0];
    s->offset = base + margin;
    if (s->type == MR_SHAPE_PLANE) {
        const v3 n = qrot(s->rot, V(0, 1, 0));
        s->normal = vmul(n, 1.0 / vlen(n));
        return;
    }
    v3 ext;
    if (s->type == MR_SHAPE_SPHERE) {
        s->radius = src->dimensions[0];
        const double e = s->radius + base;
        ext = V(e, e, e);
        s->lower = vsub(s->center, ext);
        s->upper = vadd(s->center, ext);
    } else if (s->type == MR_SHAPE_CAPSULE) {
        s->radius = src->dimensions[0];
        s->half_length = src->dimensions[1];
        const v3 ax = qrot(s->rot, V(0, src->dimensions[1], 0));
        s->ep0 = vsub(s->center, ax);
        s->ep1 = vadd(s->center, ax);
        const double e = s->radius + base;
        s->lower = V(fmin(s->ep0.x, s->ep1.x) - e, fmin(s->ep0.y, s->ep1.y) - e, fmin(s->ep0.z, s->ep1.z) - e);
        s->upper = V(fmax(s->ep0.x, s->ep1.x) + e, fmax(s->ep0.y, s->ep1.y) + e, fmax(s->ep0.z, s->ep1.z) + e);
    } else {
        s->half = vldf(src->dimensions);
        const v3 bx = qrot(s->rot, V(1, 0, 0)), by = qrot(s->rot, V(0, 1, 0)), bz = qrot(s->rot, V(0, 0, 1));
        ext = V(fabs(bx.x) * s->half.x + fabs(by.x) * s->half.y + fabs(bz.x) * s->half.z + base,
                fabs(bx.y) * s->half.x + fabs(by.y) * s->half.y + fabs(bz.y) * s->half.z + base,
                fabs(bx.z) * s->half.x + fabs(by.z) * s->half.y + fabs(bz.z) * s->half.z + base);
        s->lower = vsub(s->center, ext);
        s->upper = vadd(s->center, ext);
    }
    const v3 sc = V(fmax(fabs(s->lower.x), fabs(s->upper.x)) + 1.0, fmax(fabs(s->lower.y), fabs(s->upper.y)) + 1.0,
                    fmax(fabs(s->lower.z), fabs(s->upper.z)) + 1.0);
    s->lower = vsub(vsub(s->lower, vmul(sc, kPad)), V(margin, margin, margin));
    s->upper = vadd(vadd(s->upper, vmul(sc, kPad)), V(margin, margin, margin));
}

static double shape_scale(const Shape* s) { /* worldShapeScale (Collision.metal:125-150) */
    return fmax(fmax(fmax(vmaxabs(s->center), vmaxabs(s->half)), fmax(vmaxabs(s->ep0), vmaxabs(s->ep1))),
                fmax(fmax(fabs(s->radius), fabs(s->half_length)), fmax(fabs(s->offset), fmax(vmaxabs(s->lower), vmaxabs(s->upper)))));
}

typedef struct {
    v3 normal;
    double sep;
    v3 pa, pb;
    uint32_t fa, fb;
} Raw;

typedef struct {
    double la[3], lb[3];
    uint32_t fa, fb, life;
    double imp[3];
    v3 wp;
    double sep, drift;
} Cand;

static unsigned long long ckey(const Cand* c) { return ((unsigned long long)c->fa << 32) | c->fb; }
static int cless(const Cand* a, const Cand* b) {
    if (a->sep != b->sep) return a->sep < b->sep;
    return ckey(a) < ckey(b);
}

/* Pair flag + raw contacts + buildPersistentWorldManifold +
 * reduceCandidates (Collision.metal:796-850, 4379-4830, 5115-5556). */
static int pair_manifold(const OracleWorld* o, const Kin* k, const double* margins, uint32_t pair, OracleManifold* slot,
                         int* candidate, Raw* raw_out, int* nraw_out) {
    const MRModelPairC* pr = &o->pairs[pair];
    Shape A, B;
    make_shape(o, k, pr->shape_a, margins[pr->shape_a], &A);
    make_shape(o, k, pr->shape_b, margins[pr->shape_b], &B);
    const int a_plane = A.type == MR_SHAPE_PLANE;
    const Shape* plane = a_plane ? &A : &B;
    const Shape* fin = a_plane ? &B : &A;
    *candidate = 0;
    {
        const v3 c = vmul(vadd(fin->lower, fin->upper), 0.5);
        const v3 hx = vmul(vsub(fin->upper, fin->lower), 0.5);
        const double scale = fmax(fmax(vmaxabs(plane->center), vmaxabs(fin->lower)),
                                  fmax(vmaxabs(fin->upper), fmax(fabs(plane->offset), fabs(fin->offset))));
        const double qpad = (scale + 1.0) * kPad;
        const v3 an = V(fabs(plane->normal.x), fabs(plane->normal.y), fabs(plane->normal.z));
        const double msd = vdot(plane->normal, vsub(c, plane->center)) - vdot(an, hx);
        BAND(msd, plane->offset + qpad);
        if (!(msd <= plane->offset + qpad)) {
            slot->count = 0;
            return 0;
        }
    }
    *candidate = 1;
    const double accepted = A.offset + B.offset + (fmax(shape_scale(&A), shape_scale(&B)) + 1.0) * kPad;
    Raw raw[8];
    int nraw = 0;
#define APPEND(surface, sep_, ffeat)                                                   \
    do {                                                                               \
        const v3 pp_ = vsub((surface), vmul(plane->normal, (sep_)));                  \
        Raw r_;                                                                        \
        if (!a_plane) {                                                                \
            r_.normal = vmul(plane->normal, -1.0); r_.pa = (surface); r_.pb = pp_;     \
            r_.fa = (ffeat); r_.fb = feature_key(MR_SHAPE_PLANE, 0u);                  \
        } else {                                                                       \
            r_.normal = plane->normal; r_.pa = pp_; r_.pb = (surface);                 \
            r_.fa = feature_key(MR_SHAPE_PLANE, 0u); r_.fb = (ffeat);                  \
        }                                                                              \
        r_.sep = (sep_);                                                               \
        raw[nraw++] = r_;                                                              \
    } while (0)
    if (pr->pair_class == MR_COLLISION_PAIR_SPHERE_PLANE) {
        const v3 surface = vsub(fin->center, vmul(plane->normal, fin->radius));
        const double sep = vdot(plane->normal, vsub(surface, plane->center));
        BAND(sep, accepted);
        if (sep <= accepted) APPEND(surface, sep, feature_key(MR_SHAPE_SPHERE, 0u));
    } else if (pr->pair_class == MR_COLLISION_PAIR_CAPSULE_PLANE) {
        for (uint32_t e = 0; e < 2; ++e) {
            const v3 surface = vsub(e == 0 ? fin->ep0 : fin->ep1, vmul(plane->normal, fin->radius));
            const double sep = vdot(plane->normal, vsub(surface, plane->center));
            BAND(sep, accepted);
            if (sep <= accepted) APPEND(surface, sep, feature_key(MR_SHAPE_CAPSULE, e));
        }
    } else if (pr->pair_class == MR_COLLISION_PAIR_BOX_PLANE) {
        for (uint32_t vtx = 0; vtx < 8; ++vtx) {
            const v3 local = V((vtx & 1) ? fin->half.x : -fin->half.x, (vtx & 2) ? fin->half.y : -fin->half.y,
                               (vtx & 4) ? fin->half.z : -fin->half.z);
            const v3 wpt = vadd(fin->center, qrot(fin->rot, local));
            const double sep = vdot(plane->normal, vsub(wpt, plane->center));
            BAND(sep, accepted);
            if (sep <= accepted) APPEND(wpt, sep, feature_key(MR_SHAPE_BOX, vtx));
        }
    }
#undef APPEND
    if (raw_out) {
        for (int i = 0; i < nraw; ++i) raw_out[i] = raw[i];
        *nraw_out = nraw;
    }
    if (nraw == 0) {
        slot->count = 0;
        return 0;
    }
    int deepest = 0;
    for (int i = 1; i < nraw; ++i) {
        const Raw* l = &raw[i];
        const Raw* r = &raw[deepest];
        if (l->sep < r->sep || (l->sep == r->sep && (l->fa < r->fa || (l->fa == r->fa && l->fb < r->fb)))) deepest = i;
    }
    v3 nw = raw[deepest].normal;
    nw = vmul(nw, 1.0 / vlen(nw));
    const v3 posA = A.body_pos, posB = B.body_pos;
    const q4 rotA = A.body_rot, rotB = B.body_rot;
    const double* thr = NULL;
    double thr_d[4];
    for (int i = 0; i < 4; ++i) thr_d[i] = o->w.manifold_thresholds[i];
    thr = thr_d;
    Cand c[12];
    int nc = 0;
    int old_ok = 0;
    v3 transported = V(0, 0, 0);
    double old_age = 0.0;
    if (slot->count > 0 && slot->count <= MPTS) {
        v3 on = qrot(rotA, vld(slot->normal_local));
        on = vmul(on, 1.0 / vlen(on));
        old_ok = vfinite(on) && vdot(on, nw) >= thr[3];
        BAND(vdot(on, nw), thr[3]);
        if (old_ok) {
            const v3 ot = qrot(rotA, vld(slot->tangent_local));
            transported = vsub(ot, vmul(nw, vdot(ot, nw)));
            old_age = slot->age;
            for (uint32_t i = 0; i < slot->count; ++i) {
                const OraclePoint* op = &slot->points[i];
                const v3 pa = vadd(posA, qrot(rotA, vld(op->anchor_a)));
                const v3 pb = vadd(posB, qrot(rotB, vld(op->anchor_b)));
                const v3 d = vsub(pb, pa);
                const double sep = vdot(d, nw);
                const double drift = vlen(vsub(d, vmul(nw, sep)));
                BAND(sep, thr[0]);
                BAND(drift, thr[1]);
                if (sep > thr[0] || drift > thr[1]) continue;
                Cand* cc = &c[nc++];
                for (int a = 0; a < 3; ++a) { cc->la[a] = op->anchor_a[a]; cc->lb[a] = op->anchor_b[a]; cc->imp[a] = op->impulses[a]; }
                cc->fa = op->feature_a;
                cc->fb = op->feature_b;
                cc->life = op->life == 0xffffffffu ? 0xffffffffu : op->life + 1u;
                cc->wp = vmul(vadd(pa, pb), 0.5);
                cc->sep = sep;
                cc->drift = drift;
            }
        }
    }
    const double merge2 = thr[2] * thr[2];
    for (int i = 0; i < nraw; ++i) {
        const Raw* r = &raw[i];
        const v3 la = qrotinv(rotA, vsub(r->pa, posA));
        const v3 lb = qrotinv(rotB, vsub(r->pb, posB));
        int match = -1;
        for (int m = 0; m < nc; ++m)
            if (c[m].fa == r->fa && c[m].fb == r->fb) { match = m; break; }
        if (match < 0)
            for (int m = 0; m < nc; ++m) {
                const v3 da = vsub(vld(c[m].la), la), db = vsub(vld(c[m].lb), lb);
                BAND(sqrt(vdot(da, da) + vdot(db, db)), sqrt(2.0 * merge2));
                if (vdot(da, da) + vdot(db, db) <= 2.0 * merge2) { match = m; break; }
            }
        if (match < 0) {
            if (nc >= 12) return -1;
            match = nc++;
            c[match].life = 0u;
            c[match].imp[0] = c[match].imp[1] = c[match].imp[2] = 0.0;
        }
        vst(c[match].la, la);
        vst(c[match].lb, lb);
        c[match].fa = r->fa;
        c[match].fb = r->fb;
        c[match].wp = vmul(vadd(r->pa, r->pb), 0.5);
        c[match].sep = r->sep;
        c[match].drift = 0.0;
    }
    for (int i = 1; i < nc; ++i) {
        Cand val = c[i];
        int d = i;
        while (d > 0 && cless(&val, &c[d - 1])) { c[d] = c[d - 1]; --d; }
        c[d] = val;
    }
    if (nc > MPTS) {
        if (nc > 1 && fabs(c[1].sep - c[0].sep) <= kBand) g_band++;
        int selected[12] = {0}, chosen[MPTS], count = 1;
        chosen[0] = 0;
        selected[0] = 1;
        for (int stage = 1; stage < MPTS; ++stage) {
            int best = -1;
            double best_score = -1.0;
            unsigned long long best_f = ~0ull;
            for (int i = 0; i < nc; ++i) {
                if (selected[i]) continue;
                double score;
                if (stage == 1) {
                    const v3 d = vsub(c[i].wp, c[chosen[0]].wp);
                    const v3 t = vsub(d, vmul(nw, vdot(d, nw)));
                    score = vdot(t, t);
                } else if (stage == 2) {
                    const v3 a = vsub(c[chosen[1]].wp, c[chosen[0]].wp);
                    const v3 bb = vsub(c[i].wp, c[chosen[0]].wp);
                    score = fabs(vdot(vcross(a, bb), nw));
                } else {
                    score = INFINITY;
                    for (int s = 0; s < count; ++s) {
                        const v3 d = vsub(c[i].wp, c[chosen[s]].wp);
                        const v3 t = vsub(d, vmul(nw, vdot(d, nw)));
                        score = fmin(score, vdot(t, t));
                    }
                }
                const unsigned long long f = ckey(&c[i]);
                /* Scores within a relative 1e-5 are ties (smaller feature key
                 * wins): box faces make exact ties structural, and the
                 * reference's absolute tolerances (Collision.cpp:2531-2544,
                 * Collision.metal:5247) leave them to rounding.  A gap within
                 * 10 % of the tie tolerance is a band decision. */
                const double tol = fmax(1.0e-12, kTieRelative * fmax(fabs(score), fabs(best_score)));
                if (best >= 0) {
                    const double gap = fabs(fabs(score - best_score) - tol);
                    if (gap <= 0.1 * tol) g_band++;
                }
                if (score > best_score + tol || (fabs(score - best_score) <= tol && f < best_f)) {
                    best = i; best_score = score; best_f = f;
                }
            }
            if (best >= 0) { chosen[count++] = best; selected[best] = 1; }
        }
        Cand red[MPTS];
        for (int i = 0; i < count; ++i) red[i] = c[chosen[i]];
        nc = count;
        for (int i = 0; i < nc; ++i) c[i] = red[i];
    }
    for (int i = 1; i < nc; ++i) {
        Cand val = c[i];
        const unsigned long long f = ckey(&val);
        int d = i;
        while (d > 0 && f < ckey(&c[d - 1])) { c[d] = c[d - 1]; --d; }
        c[d] = val;
    }
    v3 tw = transported;
    if (!old_ok || !vfinite(tw) || vdot(tw, tw) <= 1.0e-12) tw = stable_tangent(nw);
    else tw = vmul(tw, 1.0 / vlen(tw));
    vst(slot->normal_local, qrotinv(rotA, nw));
    slot->age = old_ok ? fmin(old_age + 1.0, 65535.0) : 0.0;
    vst(slot->tangent_local, qrotinv(rotA, tw));
    slot->count = (uint32_t)nc;
    for (int i = 0; i < MPTS; ++i) {
        OraclePoint* op = &slot->points[i];
        memset(op, 0, sizeof(*op));
        if (i < nc) {
            for (int a = 0; a < 3; ++a) { op->anchor_a[a] = c[i].la[a]; op->anchor_b[a] = c[i].lb[a]; op->impulses[a] = c[i].imp[a]; }
            op->feature_a = c[i].fa;
            op->feature_b = c[i].fb;
            op->life = c[i].life;
        }
    }
    return nc;
}

/* ------------------------------------------------------------------ */
/* Dense factor solves                                                  */
/* ------------------------------------------------------------------ */
static int cholesky(double* A, uint32_t n) { /* in place, lower */
    for (uint32_t j = 0; j < n; ++j) {
        double d = A[j * n + j];
        for (uint32_t k = 0; k < j; ++k) d -= A[j * n + k] * A[j * n + k];
        if (!(d > kPivotFloor) || !isfinite(d)) return 0;
        A[j * n + j] = sqrt(d);
        for (uint32_t i = j + 1; i < n; ++i) {
            double s = A[i * n + j];
            for (uint32_t k = 0; k < j; ++k) s -= A[i * n + k] * A[j * n + k];
            A[i * n + j] = s / A[j * n + j];
        }
    }
    return 1;
}

static void chol_solve(const double* L, uint32_t n, double* x) { /* solveCholesky (MetalWorldContact.metal:406-445) */
    for (uint32_t i = 0; i < n; ++i) {
        double s = x[i];
        for (uint32_t k = 0; k < i; ++k) s -= L[i * n + k] * x[k];
        x[i] = s / L[i * n + i];
    }
    for (int i = (int)n - 1; i >= 0; --i) {
        double s = x[i];
        for (uint32_t k = (uint32_t)i + 1; k < n; ++k) s -= L[k * n + i] * x[k];
        x[i] = s / L[i * n + i];
    }
}

/* ------------------------------------------------------------------ */
/* Converged contact solve (quality mode).  The problem is numi-lab's      */
/* exact-cone QP (QualityContactSolver.hpp:55-80): min 0.5 l'(W + R)l +    */
/* (u_free - u_target)'l over the friction cones.  Restated from the       */
/* library's solver: Newton steps on the factor-space primal              */
/* f(z) = 0.5|z|^2 + sum_c psi_c(u_free + Y_c'z), W = Y'Y, with the        */
/* closed-form R-metric cone projection, an exact line search (the root   */
/* of the monotone phi'(t) by safeguarded Newton steps in a bracket), a   */
/* continuation on the regularisation floor, and the stopping test        */
/* |z - Y l|_inf <= tol (1 + |z|_inf + |Y l|_inf).  Its                   */
/* answers are pinned to the reference's solveQualityContactProblem.      */
/* ------------------------------------------------------------------ */
static double q_project(const double* u, const double* tg, const double* rg_in, double mu, double rho, double* lam, double* D) {
    const double rg[3] = {fmax(rg_in[0], rho), fmax(rg_in[1], rho), fmax(rg_in[2], rho)};
    const double e0 = u[0] - tg[0], e1 = u[1] - tg[1], e2 = u[2] - tg[2];
    const double a0 = -e0 / rg[0], a1 = -e1 / rg[1], a2 = -e2 / rg[2];
    for (int i = 0; i < 6; ++i) D[i] = 0.0;
    if (!(mu > 0.0)) {
        lam[0] = fmax(a0, 0.0);
        lam[1] = lam[2] = 0.0;
        if (lam[0] > 0.0) D[0] = 1.0 / rg[0];
    } else {
        const double b1 = a1 / mu, b2 = a2 / mu, s = sqrt(b1 * b1 + b2 * b2);
        const double d0 = rg[0], dt = rg[1] * mu * mu;
        if (s <= a0) { /* sticking */
            lam[0] = a0; lam[1] = a1; lam[2] = a2;
            D[0] = 1.0 / rg[0]; D[3] = 1.0 / rg[1]; D[5] = 1.0 / rg[2];
        } else if (d0 * a0 <= -dt * s) { /* separating */
            lam[0] = lam[1] = lam[2] = 0.0;
        } else { /* sliding: on the cone surface */
            const double inv = 1.0 / (d0 + dt), rho = (d0 * a0 + dt * s) * inv, n1 = b1 / s, n2 = b2 / s;
            const double w = rho / (s * rg[1]);
            lam[0] = rho; lam[1] = mu * rho * n1; lam[2] = mu * rho * n2;
            D[0] = inv; D[1] = inv * mu * n1; D[2] = inv * mu * n2;
            D[3] = inv * mu * mu * n1 * n1 + w * (1.0 - n1 * n1);
            D[4] = inv * mu * mu * n1 * n2 - w * n1 * n2;
            D[5] = inv * mu * mu * n2 * n2 + w * (1.0 - n2 * n2);
        }
    }
    return -(0.5 * (rg[0] * lam[0] * lam[0] + rg[1] * lam[1] * lam[1] + rg[2] * lam[2] * lam[2]) + e0 * lam[0] + e1 * lam[1] +
             e2 * lam[2]);
}

/* f at x; impulses, derivatives and gradient when the outputs are given. */
static double q_eval(uint32_t nv, uint32_t nc, const double* Y, const double* uf, const double* tg, const double* rg,
                     const double* mu, double rho, const double* x, double* lam, double* D, double* grad) {
    double f = 0.0, l[3], d[6];
    for (uint32_t d0 = 0; d0 < nv; ++d0) f += 0.5 * x[d0] * x[d0];
    for (uint32_t c = 0; c < nc; ++c) {
        double u[3];
        for (int r = 0; r < 3; ++r) {
            u[r] = uf[3 * c + r];
            for (uint32_t k = 0; k < nv; ++k) u[r] += Y[(3 * c + r) * nv + k] * x[k];
        }
        f += q_project(u, tg + 3 * c, rg + 3 * c, mu[c], rho, l, d);
        if (lam) for (int r = 0; r < 3; ++r) lam[3 * c + r] = l[r];
        if (D) for (int i = 0; i < 6; ++i) D[6 * c + i] = d[i];
    }
    if (grad) {
        for (uint32_t k = 0; k < nv; ++k) {
            double acc = 0.0;
            for (uint32_t row = 0; row < 3 * nc; ++row) acc += Y[row * nv + k] * lam[row];
            grad[k] = x[k] - acc;
        }
    }
    return f;
}

/* Regularisation continuation: stages with every row's regularisation
 * raised to 3000x and 30x the floor (to scaled optimality 1e-3), then the
 * problem's own, each warm-started by the last. */
static const double kQStageFloor[2] = {3000.0, 30.0};
static const double kQStageTolerance = 1.0e-3;

uint32_t oracle_quality_solve(uint32_t nv, uint32_t nc, const double* Y, const double* ufree, const double* target,
                              const double* reg, const double* mu, const double* warm, const OracleQualityConfig* cfg,
                              double* lambda, double* zeta, OracleQualityOutcome* out) {
    double z[MAXV], grad[MAXV], dir[MAXV], H[MAXV * MAXV], D[6 * MAXC], U[3 * MAXC], Wd[3 * MAXC];
    OracleQualityOutcome o;
    memset(&o, 0, sizeof(o));
    o.status = 1;
    for (uint32_t k = 0; k < nv; ++k) {
        double acc = 0.0;
        if (warm)
            for (uint32_t row = 0; row < 3 * nc; ++row) acc += Y[row * nv + k] * warm[row];
        z[k] = acc;
    }
    double f = 0.0, scaled = 0.0;
    int broken = 0;
    for (int stage = 0; stage < 3 && !broken; ++stage) {
        const double rho = stage < 2 ? kQStageFloor[stage] * cfg->regularization_floor : 0.0;
        const double tol = stage < 2 ? kQStageTolerance : cfg->tolerance;
        f = q_eval(nv, nc, Y, ufree, target, reg, mu, rho, z, lambda, D, grad);
        for (;;) {
            double gm = 0.0, zm = 0.0, ym = 0.0;
            int finite = isfinite(f);
            for (uint32_t k = 0; k < nv; ++k) {
                gm = fmax(gm, fabs(grad[k]));
                zm = fmax(zm, fabs(z[k]));
                ym = fmax(ym, fabs(z[k] - grad[k]));
                finite &= isfinite(grad[k]) && isfinite(z[k]);
            }
            if (!finite) { o.status = 3; broken = 1; break; }
            scaled = gm / (1.0 + zm + ym);
            if (scaled <= tol) {
                if (stage == 2) o.status = 0;
                break;
            }
            if ((int)o.newton >= cfg->max_newton) { broken = 1; break; }
            /* I + sum_c Y_c D_c Y_c' */
            for (uint32_t i = 0; i < nv; ++i)
                for (uint32_t j = 0; j < nv; ++j) H[i * nv + j] = i == j ? 1.0 : 0.0;
            for (uint32_t c = 0; c < nc; ++c) {
                const double* Dc = D + 6 * c;
                const double M3[3][3] = {{Dc[0], Dc[1], Dc[2]}, {Dc[1], Dc[3], Dc[4]}, {Dc[2], Dc[4], Dc[5]}};
                for (uint32_t j = 0; j < nv; ++j) {
                    double e[3];
                    for (int r = 0; r < 3; ++r) {
                        e[r] = 0.0;
                        for (int t = 0; t < 3; ++t) e[r] += M3[r][t] * Y[(3 * c + t) * nv + j];
                    }
                    for (uint32_t i = j; i < nv; ++i)
                        H[i * nv + j] += Y[(3 * c) * nv + i] * e[0] + Y[(3 * c + 1) * nv + i] * e[1] + Y[(3 * c + 2) * nv + i] * e[2];
                }
            }
            for (uint32_t i = 0; i < nv; ++i)
                for (uint32_t j = i + 1; j < nv; ++j) H[i * nv + j] = H[j * nv + i];
            if (!cholesky(H, nv)) { o.status = 2; broken = 1; break; }
            for (uint32_t k = 0; k < nv; ++k) dir[k] = -grad[k];
            chol_solve(H, nv, dir);
            double slope = 0.0;
            for (uint32_t k = 0; k < nv; ++k) slope += grad[k] * dir[k];
            if (!(slope < 0.0))
                for (uint32_t k = 0; k < nv; ++k) dir[k] = -grad[k];
            /* Exact line search: phi'(t) = a + t b - sum_c l_c(u_c + t w_c)' w_c. */
            double a = 0.0, b = 0.0, slope0 = 0.0;
            for (uint32_t k = 0; k < nv; ++k) { a += dir[k] * z[k]; b += dir[k] * dir[k]; slope0 += dir[k] * grad[k]; }
            for (uint32_t c = 0; c < nc; ++c)
                for (int r = 0; r < 3; ++r) {
                    double u = ufree[3 * c + r], w = 0.0;
                    for (uint32_t k = 0; k < nv; ++k) { u += Y[(3 * c + r) * nv + k] * z[k]; w += Y[(3 * c + r) * nv + k] * dir[k]; }
                    U[3 * c + r] = u;
                    Wd[3 * c + r] = w;
                }
            double lo = 0.0, hi = INFINITY, t = 1.0, best = INFINITY, best_t = 1.0;
            for (int ls = 0; ls < cfg->max_line_search; ++ls) {
                double dt = a + t * b, h2 = b, l[3], Dc[6], u[3];
                for (uint32_t c = 0; c < nc; ++c) {
                    const double* w = Wd + 3 * c;
                    for (int r = 0; r < 3; ++r) u[r] = U[3 * c + r] + t * w[r];
                    q_project(u, target + 3 * c, reg + 3 * c, mu[c], rho, l, Dc);
                    dt -= l[0] * w[0] + l[1] * w[1] + l[2] * w[2];
                    h2 += w[0] * (Dc[0] * w[0] + Dc[1] * w[1] + Dc[2] * w[2]) + w[1] * (Dc[1] * w[0] + Dc[3] * w[1] + Dc[4] * w[2]) +
                          w[2] * (Dc[2] * w[0] + Dc[4] * w[1] + Dc[5] * w[2]);
                }
                o.line_search++;
                if (fabs(dt) < best) { best = fabs(dt); best_t = t; }
                if (fabs(dt) <= cfg->line_search_tolerance * fabs(slope0)) break;
                if (dt < 0.0) lo = t;
                else hi = t;
                double tn = t - dt / h2;
                if (!(tn > lo && tn < hi)) tn = isfinite(hi) ? 0.5 * (lo + hi) : 2.0 * t;
                if (isfinite(hi) && hi - lo <= 1.0e-14 * hi) break;
                t = tn;
            }
            for (uint32_t k = 0; k < nv; ++k) z[k] += best_t * dir[k];
            f = q_eval(nv, nc, Y, ufree, target, reg, mu, rho, z, lambda, D, grad);
            o.newton++;
        }
    }
    o.residual = scaled;
    o.objective = f;
    for (uint32_t c = 0; c < nc; ++c) {
        const double* l = lambda + 3 * c;
        const double lt = sqrt(l[1] * l[1] + l[2] * l[2]);
        o.cone = fmax(o.cone, fmax(-l[0], mu[c] > 0.0 ? lt - mu[c] * l[0] : lt));
        double w = 0.0;
        for (int r = 0; r < 3; ++r) {
            double u = ufree[3 * c + r];
            for (uint32_t k = 0; k < nv; ++k) u += Y[(3 * c + r) * nv + k] * z[k];
            w += l[r] * (u - target[3 * c + r] + reg[3 * c + r] * l[r]);
        }
        o.complementarity = fmax(o.complementarity, fabs(w));
    }
    if (zeta) for (uint32_t k = 0; k < nv; ++k) zeta[k] = z[k];
    if (out) *out = o;
    return o.status;
}

uint32_t oracle_quality_dense(uint32_t nv, uint32_t nc, const double* mass, const double* jacobian, const double* vf,
                              const double* target, const double* reg, const double* mu, const double* warm,
                              const OracleQualityConfig* cfg, double* lambda, double* velocity, OracleQualityOutcome* out) {
    static __thread double L[MAXV * MAXV], Y[3 * MAXC * MAXV];
    double uf[3 * MAXC], rg[3 * MAXC], w[MAXV];
    if (nv > MAXV || nc > MAXC) return 3;
    memcpy(L, mass, sizeof(double) * nv * nv);
    if (!cholesky(L, nv)) {
        if (out) { memset(out, 0, sizeof(*out)); out->status = 2; }
        return 2;
    }
    for (uint32_t row = 0; row < 3 * nc; ++row) {
        const double* g = jacobian + (size_t)row * nv;
        double* y = Y + (size_t)row * nv;
        for (uint32_t k = 0; k < nv; ++k) {
            double acc = g[k];
            for (uint32_t j = 0; j < k; ++j) acc -= L[k * nv + j] * y[j];
            y[k] = acc / L[k * nv + k];
        }
        uf[row] = 0.0;
        for (uint32_t d = 0; d < nv; ++d) uf[row] += g[d] * vf[d];
        rg[row] = fmax(reg[row], cfg->regularization_floor);
    }
    const uint32_t st = oracle_quality_solve(nv, nc, Y, uf, target, rg, mu, warm, cfg, lambda, NULL, out);
    for (uint32_t k = 0; k < nv; ++k) {
        w[k] = 0.0;
        for (uint32_t row = 0; row < 3 * nc; ++row) w[k] += Y[row * nv + k] * lambda[row];
    }
    for (int i = (int)nv - 1; i >= 0; --i) { /* L' x = w */
        double s = w[i];
        for (uint32_t k = (uint32_t)i + 1; k < nv; ++k) s -= L[k * nv + i] * w[k];
        w[i] = s / L[i * nv + i];
    }
    for (uint32_t k = 0; k < nv; ++k) velocity[k] = vf[k] + w[k];
    return st;
}

/* The last contact problem a control step on this thread handed to the
 * converged solve (for diagnosing the solver on recorded problems). */
static __thread uint32_t g_qlast_nv, g_qlast_nc;
static __thread double g_qlast[3 * MAXC * MAXV + 16 * MAXC];

uint32_t oracle_quality_last_problem(double* Y, double* ufree, double* target, double* reg, double* mu, double* warm, uint32_t* nv) {
    const uint32_t n = g_qlast_nc, m = g_qlast_nv;
    const double* p = g_qlast;
    if (Y) memcpy(Y, p, sizeof(double) * 3 * n * m);
    p += 3 * n * m;
    if (ufree) memcpy(ufree, p, sizeof(double) * 3 * n);
    p += 3 * n;
    if (target) memcpy(target, p, sizeof(double) * 3 * n);
    p += 3 * n;
    if (reg) memcpy(reg, p, sizeof(double) * 3 * n);
    p += 3 * n;
    if (mu) memcpy(mu, p, sizeof(double) * n);
    p += n;
    if (warm) memcpy(warm, p, sizeof(double) * 3 * n);
    if (nv) *nv = m;
    return n;
}

static void quality_record(uint32_t nv, uint32_t nc, const double* Y, const double* uf, const double* tg, const double* rg,
                           const double* mu, const double* warm) {
    double* p = g_qlast;
    g_qlast_nv = nv;
    g_qlast_nc = nc;
    memcpy(p, Y, sizeof(double) * 3 * nc * nv);
    p += 3 * nc * nv;
    memcpy(p, uf, sizeof(double) * 3 * nc);
    p += 3 * nc;
    memcpy(p, tg, sizeof(double) * 3 * nc);
    p += 3 * nc;
    memcpy(p, rg, sizeof(double) * 3 * nc);
    p += 3 * nc;
    memcpy(p, mu, sizeof(double) * nc);
    p += nc;
    memcpy(p, warm, sizeof(double) * 3 * nc);
}

void oracle_world_set_quality(OracleWorld* world, const OracleQualityConfig* cfg) {
    world->quality = cfg != NULL;
    if (cfg) world->qcfg = *cfg;
}

/* ------------------------------------------------------------------ */
/* Contact substep: scatter to ConstraintIR (Collision.metal:10253-10620), */
/* IR evaluation (MetalWorldContact.metal:3580-3990), Wave32 temporalCone */
/* solve (MetalWorldContact.metal:6142-7216), joint limits (:2878-2968),  */
/* integration (:8876-9050).                                            */
/* ------------------------------------------------------------------ */
typedef struct {
    uint32_t pair, point, body, new_impact;
    int b_side;
    v3 x, n, t, bt;
    double sep, target[3], reg[3], mu, lambda[3], P[9], relax, delta[3], rel[3];
    double G[3][MAXV];
} Contact;

/* One manifold point as a solver contact: world frame, Jacobian rows at
 * the free velocity, ConstraintIR evaluation (target velocity with the
 * speculative approach term, critically damped stabilisation and
 * restitution on a new impact; regularisation; static or dynamic friction
 * by slip) -- Collision.metal:10253-10620, MetalWorldContact.metal:3580-3990. */
static void prepare_contact(const OracleWorld* o, const Kin* k, const OracleManifold* slot, uint32_t p, int i, const double* vf,
                            double friction_scale, Contact* ct) {
    const uint32_t nv = o->w.nv;
    const double h = o->h;
    const MRModelPairC* pr = &o->pairs[p];
    const MRModelShapeC* sa = &o->shapes[pr->shape_a];
    const MRModelShapeC* sb = &o->shapes[pr->shape_b];
    const MRModelBodyC* ba = &o->bodies[sa->body];
    const MRModelBodyC* bb = &o->bodies[sb->body];
    v3 posA, posB;
    q4 rotA, rotB;
    if (ba->articulated) { posA = k->pos[sa->body]; rotA = k->rot[sa->body]; }
    else { posA = vldf(ba->static_pose); qnormalize(qldf(ba->static_pose + 4), &rotA, 0); }
    if (bb->articulated) { posB = k->pos[sb->body]; rotB = k->rot[sb->body]; }
    else { posB = vldf(bb->static_pose); qnormalize(qldf(bb->static_pose + 4), &rotB, 0); }
    v3 nw = qrot(rotA, vld(slot->normal_local));
    nw = vmul(nw, 1.0 / vlen(nw));
    v3 tw = qrot(rotA, vld(slot->tangent_local));
    tw = vsub(tw, vmul(nw, vdot(tw, nw)));
    tw = vdot(tw, tw) > 1.0e-12 ? vmul(tw, 1.0 / vlen(tw)) : stable_tangent(nw);
    const v3 bw = vcross(nw, tw);
    const MRModelMaterialC* ma = &o->materials[sa->material];
    const MRModelMaterialC* mb = &o->materials[sb->material];
    const double mu_s = sqrt(fmax(0.0, (double)ma->friction[0] * mb->friction[0])) * friction_scale;
    const double mu_d = sqrt(fmax(0.0, (double)ma->friction[1] * mb->friction[1])) * friction_scale;
    const double restitution = fmin(fmax(fmax(ma->response[0], mb->response[0]), 0.0), 1.0);
    const double rthr = fmax(ma->response[1], mb->response[1]);
    const double compliance = (double)ma->response[2] + mb->response[2];
    const double dissipation = (double)ma->response[3] + mb->response[3];
    const double rest = (double)sa->contact_rest_bound[1] + sb->contact_rest_bound[1];
    const OraclePoint* op = &slot->points[i];
    const v3 pa = rn3(vadd(posA, rn3(qrot(rotA, vld(op->anchor_a)))));
    const v3 pb = rn3(vadd(posB, rn3(qrot(rotB, vld(op->anchor_b)))));
    ct->pair = p;
    ct->point = (uint32_t)i;
    ct->x = vmul(vadd(pa, pb), 0.5);
    ct->sep = rn(vdot(vsub(pb, pa), nw) - rest);
    ct->n = nw; ct->t = tw; ct->bt = bw;
    ct->new_impact = op->life == 0u;
    ct->b_side = !ba->articulated;
    ct->body = ct->b_side ? sb->body : sa->body;
    for (int a = 0; a < 3; ++a) ct->lambda[a] = op->impulses[a];
    /* Jacobian rows and relative velocity at v_free. */
    double J[3 * MAXV];
    point_jacobian_k(o, k, ct->body, ct->x, J);
    const double sign = ct->b_side ? 1.0 : -1.0;
    const v3 dirs[3] = {nw, tw, bw};
    for (int r = 0; r < 3; ++r) {
        ct->rel[r] = 0.0;
        for (uint32_t d = 0; d < nv; ++d) {
            const double g = rn(sign * (vget(dirs[r], 0) * J[d] + vget(dirs[r], 1) * J[nv + d] + vget(dirs[r], 2) * J[2 * nv + d]));
            ct->G[r][d] = g;
            ct->rel[r] += g * vf[d];
        }
    }
    ct->target[0] = ct->sep > 0.0 ? -ct->sep / h : 0.0;
    ct->target[1] = ct->target[2] = 0.0;
    ct->reg[0] = fmax(compliance / (h * h) + dissipation / h, 0.0);
    ct->reg[1] = ct->reg[2] = 0.0;
    const double tau_c = 2.0 * h;
    const double err = fmin(ct->sep + o->w.solver_scales[3], 0.0);
    const double ratio = h / tau_c;
    const double den = 1.0 + 2.0 * ratio + ratio * ratio;
    double stab = -h * err / (tau_c * tau_c * den);
    stab = fmin(fmax(stab, 0.0), o->w.solver_scales[2]);
    if (ct->new_impact) {
        const double incoming = ct->rel[0] - ct->target[0];
        if (incoming < -rthr) stab = fmax(stab, -restitution * incoming);
    }
    ct->target[0] += stab;
    const double slip = sqrt(ct->rel[1] * ct->rel[1] + ct->rel[2] * ct->rel[2]);
    ct->mu = slip <= 1.0e-3 ? mu_s : mu_d;
}

/* Speculative collision margins of the articulated shapes for a substep
 * whose free velocity is vf (Collision.metal:5794-6030). */
static void speculative_margins(const OracleWorld* o, const double* vf, double* margins) {
    const uint32_t nv = o->w.nv, ns = o->w.shape_count;
    const double h = o->h;
    double gs = 0.0;
    for (uint32_t d = 0; d < nv; ++d) gs += fabs(vf[d]);
    for (uint32_t s = 0; s < ns; ++s) {
        margins[s] = 0.0;
        const MRModelShapeC* src = &o->shapes[s];
        if (o->bodies[src->body].articulated && src->shape_type != MR_SHAPE_PLANE) {
            double sweep = src->contact_rest_bound[2];
            if (!(sweep > 0.0) || !isfinite(sweep)) {
                if (src->shape_type == MR_SHAPE_SPHERE) sweep = src->dimensions[0];
                else if (src->shape_type == MR_SHAPE_CAPSULE) sweep = src->dimensions[0] + src->dimensions[1];
                else sweep = vlen(vldf(src->dimensions));
            }
            const double env = fmin(h * gs * fmax(sweep, 0.25), h * (double)o->w.speculative[1]);
            margins[s] = o->w.speculative[0] * env;
        }
    }
}

static uint32_t contact_substep(const OracleWorld* o, double* q, double* v, const double* vf, const Kin* k, OracleManifold* slots,
                                double friction_scale, int final_substep, OracleTrace* trace, uint32_t* fail_index) {
    const uint32_t nv = o->w.nv, np = o->w.pair_count;
    const double h = o->h;
    double margins[MAXS];
    speculative_margins(o, vf, margins);
    static __thread Contact C[MAXC];
    uint32_t total = 0, manifolds = 0;
    int counts[MAXP];
    for (uint32_t p = 0; p < np; ++p) {
        int cand = 0;
        counts[p] = pair_manifold(o, k, margins, p, &slots[p], &cand, NULL, NULL);
        if (counts[p] < 0) { *fail_index = p; return MR_STEP_NONFINITE_RESULT; }
        total += (uint32_t)counts[p];
        if (counts[p] > 0) manifolds++;
    }
    trace->manifold_count = manifolds;
    if (total > o->w.contact_capacity) { *fail_index = total; return MR_STEP_CONTACT_CAPACITY_OVERFLOW; }
    uint32_t c = 0;
    for (uint32_t p = 0; p < np; ++p)
        for (int i = 0; i < counts[p]; ++i, ++c) prepare_contact(o, k, &slots[p], p, i, vf, friction_scale, &C[c]);
    trace->contact_count = total;
    if (total > trace->max_contacts) trace->max_contacts = total;
    trace->island_count = total > 0 ? 1u : 0u;
    for (uint32_t d = 0; d < nv; ++d) v[d] = vf[d];
    if (total > 0) {
        double Mm[MAXV * MAXV];
        mass_matrix_k(o, k, Mm);
        for (uint32_t d = 0; d < nv; ++d) Mm[d * nv + d] += o->arm_eff[d];
        if (!cholesky(Mm, nv)) { *fail_index = 0; return MR_STEP_FACTORIZATION_FAILED; }
        static __thread double Rc[3 * MAXC][MAXV];
        for (uint32_t i = 0; i < total; ++i)
            for (int r = 0; r < 3; ++r) {
                for (uint32_t d = 0; d < nv; ++d) Rc[3 * i + r][d] = C[i].G[r][d];
                chol_solve(Mm, nv, Rc[3 * i + r]);
                for (uint32_t d = 0; d < nv; ++d) Rc[3 * i + r][d] = rn(Rc[3 * i + r][d]);
            }
        if (o->quality) {
            /* Converged solve of the same contact problem: factor rows
             * Y = L^-1 G' (W = G M^-1 G' = Y'Y), FP32-stored inputs. */
            static __thread double Yq[3 * MAXC * MAXV];
            double uf[3 * MAXC], tg[3 * MAXC], rg[3 * MAXC], muv[MAXC], warm[3 * MAXC], lam[3 * MAXC];
            for (uint32_t i = 0; i < total; ++i) {
                Contact* ct = &C[i];
                for (int r = 0; r < 3; ++r) {
                    double* y = Yq + (size_t)(3 * i + r) * nv;
                    for (uint32_t k = 0; k < nv; ++k) {
                        double acc = ct->G[r][k];
                        for (uint32_t j = 0; j < k; ++j) acc -= Mm[k * nv + j] * y[j];
                        y[k] = acc / Mm[k * nv + k];
                    }
                    for (uint32_t k = 0; k < nv; ++k) y[k] = rn(y[k]);
                    uf[3 * i + r] = rn(ct->rel[r]);
                    tg[3 * i + r] = ct->target[r];
                    rg[3 * i + r] = fmax(ct->reg[r], o->qcfg.regularization_floor);
                }
                muv[i] = ct->mu;
                oracle_project_cone(ct->lambda, ct->mu, ct->mu, warm + 3 * i);
            }
            OracleQualityOutcome qo;
            quality_record(nv, total, Yq, uf, tg, rg, muv, warm);
            const uint32_t qs = oracle_quality_solve(nv, total, Yq, uf, tg, rg, muv, warm, &o->qcfg, lam, NULL, &qo);
            if (qo.newton > trace->quality_newton) trace->quality_newton = qo.newton;
            trace->quality_line_search += qo.line_search;
            if (qs != 0) {
                *fail_index = qo.newton;
                return qs == 2 ? MR_STEP_FACTORIZATION_FAILED : (qs == 3 ? MR_STEP_NONFINITE_RESULT : MR_STEP_DID_NOT_CONVERGE);
            }
            for (uint32_t i = 0; i < total; ++i)
                for (int r = 0; r < 3; ++r) C[i].lambda[r] = lam[3 * i + r];
            for (uint32_t d = 0; d < nv; ++d) {
                double acc = 0.0;
                for (uint32_t i = 0; i < total; ++i)
                    for (int r = 0; r < 3; ++r) acc += Rc[3 * i + r][d] * lam[3 * i + r];
                v[d] = rn(v[d] + acc);
            }
        }
        for (uint32_t i = 0; i < total && !o->quality; ++i) {
            Contact* ct = &C[i];
            double W[9];
            for (int r = 0; r < 3; ++r)
                for (int s = 0; s < 3; ++s) {
                    double acc = 0.0;
                    for (uint32_t d = 0; d < nv; ++d) acc += ct->G[r][d] * Rc[3 * i + s][d];
                    W[r * 3 + s] = rn(acc + (r == s ? ct->reg[r] : 0.0));
                }
            if (!oracle_invert3x3(W, ct->P)) { *fail_index = i; return MR_STEP_FACTORIZATION_FAILED; }
            for (int e = 0; e < 9; ++e) ct->P[e] = rn(ct->P[e]);
            double rowsum = 0.0, diag = 0.0;
            for (uint32_t j = 0; j < total; ++j) {
                double acc = 0.0;
                for (uint32_t d = 0; d < nv; ++d) acc += ct->G[0][d] * Rc[3 * j][d];
                rowsum += fabs(acc);
                if (j == i) diag = fabs(acc) + ct->reg[0];
            }
            ct->relax = rowsum > fmax(diag, kMatrixFloor) ? fmin(fmax(diag / rowsum, 1.0 / 32.0), 1.0) : 1.0;
            double warm[3];
            oracle_project_cone(ct->lambda, ct->mu, ct->mu, warm);
            for (int a = 0; a < 3; ++a) { ct->lambda[a] = warm[a]; ct->delta[a] = warm[a]; }
        }
        const uint32_t iters = o->quality ? 0u : o->iters + (final_substep ? o->final_iters : 0u);
        for (int it = o->quality ? 0 : -1; it < (int)iters; ++it) {
            if (it >= 0) {
                for (uint32_t i = 0; i < total; ++i) {
                    Contact* ct = &C[i];
                    double u[3], rhs[3], prop[3], proj[3];
                    for (int r = 0; r < 3; ++r) {
                        u[r] = 0.0;
                        for (uint32_t d = 0; d < nv; ++d) u[r] += ct->G[r][d] * v[d];
                        rhs[r] = rn(ct->target[r] - rn(u[r]) - ct->reg[r] * ct->lambda[r]);
                    }
                    for (int r = 0; r < 3; ++r) prop[r] = ct->lambda[r] + ct->P[r * 3] * rhs[0] + ct->P[r * 3 + 1] * rhs[1] + ct->P[r * 3 + 2] * rhs[2];
                    oracle_project_cone(prop, ct->mu, ct->mu, proj);
                    for (int r = 0; r < 3; ++r) {
                        ct->delta[r] = rn(ct->relax * (proj[r] - ct->lambda[r]));
                    }
                    int finite = 1;
                    for (int r = 0; r < 3; ++r) finite &= isfinite(ct->lambda[r] + ct->delta[r]) && isfinite(ct->delta[r]);
                    if (!finite) { *fail_index = i; return MR_STEP_NONFINITE_RESULT; }
                    for (int r = 0; r < 3; ++r) ct->lambda[r] += ct->delta[r];
                }
            }
            for (uint32_t d = 0; d < nv; ++d) {
                double acc = 0.0;
                for (uint32_t i = 0; i < total; ++i)
                    for (int r = 0; r < 3; ++r) acc += Rc[3 * i + r][d] * C[i].delta[r];
                v[d] = rn(v[d] + acc);
            }
        }
        /* Diagnostics (MetalWorldContact.metal:7052-7110) and impulse write-back. */
        for (uint32_t i = 0; i < total; ++i) {
            Contact* ct = &C[i];
            double un = 0.0;
            for (uint32_t d = 0; d < nv; ++d) un += ct->G[0][d] * v[d];
            const double eq = un - ct->target[0] + ct->reg[0] * ct->lambda[0];
            const double resid = ct->lambda[0] > 1.0e-7 ? fabs(eq) : fmax(-eq, 0.0);
            if (resid > trace->max_normal_residual) trace->max_normal_residual = resid;
            const double lu = ct->mu * ct->lambda[0];
            double viol;
            if (lu > 0.0) viol = fmax(sqrt((ct->lambda[1] * ct->lambda[1] + ct->lambda[2] * ct->lambda[2]) / (lu * lu)) - 1.0, 0.0);
            else viol = sqrt(ct->lambda[1] * ct->lambda[1] + ct->lambda[2] * ct->lambda[2]);
            if (viol > trace->max_cone_violation) trace->max_cone_violation = viol;
            OraclePoint* op = &slots[ct->pair].points[ct->point];
            for (int a = 0; a < 3; ++a) op->impulses[a] = ct->lambda[a];
            OracleContact* oc = &trace->contacts[i];
            oc->pair = ct->pair;
            oc->point = ct->point;
            oc->feature_a = op->feature_a;
            oc->feature_b = op->feature_b;
            oc->body = ct->body;
            oc->new_impact = ct->new_impact;
            oc->separation = ct->sep;
            vst(oc->normal, ct->n);
            for (int a = 0; a < 3; ++a) oc->impulses[a] = ct->lambda[a];
        }
    }
    /* Joint limits on the post-solve velocity. */
    for (uint32_t d = 0; d < nv; ++d) {
        const MRModelDofC* dof = &o->dofs[d];
        double vel = v[d];
        if (dof->flags & MR_DOF_FLAG_VELOCITY_LIMIT) vel = fmin(fmax(vel, -dof->limits[2]), dof->limits[2]);
        if ((dof->flags & MR_DOF_FLAG_POSITION_LIMIT) && dof->q_index != MR_INVALID_INDEX) {
            const double pos = q[dof->q_index];
            vel = fmin(fmax(vel, (dof->limits[0] - pos) / h), (dof->limits[1] - pos) / h);
        }
        if (!isfinite(vel)) { *fail_index = d; return MR_STEP_NONFINITE_RESULT; }
        v[d] = vel;
    }
    /* Integration from the substep-start configuration. */
    for (uint32_t d = 0; d < nv; ++d) {
        const MRModelDofC* dof = &o->dofs[d];
        if (dof->q_index != MR_INVALID_INDEX && !(o->floating && d < 6)) q[dof->q_index] = rn(q[dof->q_index] + h * v[d]);
    }
    if (o->floating) {
        q[0] = rn(q[0] + h * v[0]);
        q[1] = rn(q[1] + h * v[1]);
        q[2] = rn(q[2] + h * v[2]);
        const q4 inc = so3_increment(V(h * v[3], h * v[4], h * v[5]), 0);
        q4 out;
        if (!qnormalize(qmul(inc, Q(q[3], q[4], q[5], q[6])), &out, 0)) { *fail_index = 3; return MR_STEP_NONFINITE_RESULT; }
        q[3] = out.x; q[4] = out.y; q[5] = out.z; q[6] = out.w;
    }
    for (uint32_t i = 0; i < o->w.nq; ++i)
        if (!isfinite(q[i])) { *fail_index = i; return MR_STEP_NONFINITE_RESULT; }
    return MR_STEP_SUCCESS;
}

/* Collision and ConstraintIR evaluation of one articulated environment at
 * configuration q with free velocity vf, for pinning against the reference's
 * CPU path (collideCpuReference, Collision.cpp:2959; assembleContactConstraints,
 * RigidBodyWorld.cpp:564; evaluateConstraintIR, ConstraintIR.cpp:1414).
 * `manifolds` [pair_count] are read and updated like a substep's.  With
 * speculative != 0 the shapes carry the substep's speculative margins, else
 * none (the CPU reference has none).  Raw contacts: 16 doubles each (shape
 * a, shape b, normal xyz, separation, point A xyz, point B xyz, feature A,
 * feature B, 0, 0).  Contact rows: ORACLE_CONTACT_ROW doubles each (shape a,
 * shape b, feature A, feature B, separation, normal xyz, point xyz, target
 * velocity n/t/b, regularisation n/t/b, effective mu, relative velocity
 * n/t/b at vf, new impact, speculative approach term -sep/h or 0).  Returns
 * a step status code. */
uint32_t oracle_articulated_contacts(const OracleWorld* o, const double* q, const double* vf, OracleManifold* manifolds,
                                     double friction_scale, int speculative, double* raw_out, uint32_t raw_cap,
                                     uint32_t* raw_count, double* rows_out, uint32_t rows_cap, uint32_t* row_count) {
    const uint32_t np = o->w.pair_count;
    g_band = 0;
    g_margin = INFINITY;
    *raw_count = 0;
    *row_count = 0;
    Kin k;
    uint32_t status = kinematics(o, q, vf, &k);
    if (status != MR_STEP_SUCCESS) return status;
    double margins[MAXS];
    if (speculative) speculative_margins(o, vf, margins);
    else for (uint32_t s = 0; s < o->w.shape_count; ++s) margins[s] = 0.0;
    int counts[MAXP];
    for (uint32_t p = 0; p < np; ++p) {
        int cand = 0, nraw = 0;
        Raw raw[8];
        counts[p] = pair_manifold(o, &k, margins, p, &manifolds[p], &cand, raw, &nraw);
        if (counts[p] < 0) return MR_STEP_NONFINITE_RESULT;
        for (int i = 0; i < nraw && *raw_count < raw_cap; ++i) {
            double* r = raw_out + 16 * (*raw_count)++;
            r[0] = o->pairs[p].shape_a;
            r[1] = o->pairs[p].shape_b;
            vst(r + 2, raw[i].normal);
            r[5] = raw[i].sep;
            vst(r + 6, raw[i].pa);
            vst(r + 9, raw[i].pb);
            r[12] = raw[i].fa;
            r[13] = raw[i].fb;
            r[14] = r[15] = 0.0;
        }
    }
    for (uint32_t p = 0; p < np; ++p)
        for (int i = 0; i < counts[p] && *row_count < rows_cap; ++i) {
            Contact ct;
            prepare_contact(o, &k, &manifolds[p], p, i, vf, friction_scale, &ct);
            double* r = rows_out + ORACLE_CONTACT_ROW * (*row_count)++;
            r[0] = o->pairs[p].shape_a;
            r[1] = o->pairs[p].shape_b;
            r[2] = manifolds[p].points[i].feature_a;
            r[3] = manifolds[p].points[i].feature_b;
            r[4] = ct.sep;
            vst(r + 5, ct.n);
            vst(r + 8, ct.x);
            for (int a = 0; a < 3; ++a) {
                r[11 + a] = ct.target[a];
                r[14 + a] = ct.reg[a];
                r[18 + a] = ct.rel[a];
            }
            r[17] = ct.mu;
            r[21] = ct.new_impact;
            r[22] = ct.sep > 0.0 ? -ct.sep / o->h : 0.0;
        }
    return MR_STEP_SUCCESS;
}

/* Free-motion commit (ArticulatedABA.metal:1446-1540). */
/* The device latches a free-motion step as non-finite when its FP32
 * arithmetic overflows.  The FP64 restatement takes the same decision when
 * a joint acceleration, the squared velocity that drives the bias forces
 * (their products reach |v|^2 x inertia) or the new velocity exceeds
 * FLT_MAX; a magnitude within a factor 1e6 of FLT_MAX is a band decision
 * (the device's intermediates may overflow a little earlier or later). */
static int beyond_float(double x) {
    const double a = fabs(x);
    if (a > (double)FLT_MAX * 1.0e-6 && a < (double)FLT_MAX * 1.0e6) g_band++;
    return !(a <= (double)FLT_MAX);
}

static uint32_t integrate_free(const OracleWorld* o, double* q, double* v, const double* qdd) {
    const uint32_t nv = o->w.nv;
    for (uint32_t d = 0; d < nv; ++d) {
        const double nvel = rn(v[d] + o->h * qdd[d]);
        const int over = beyond_float(qdd[d]) | beyond_float(v[d] * v[d]) | beyond_float(nvel);
        if (!isfinite(nvel) || over) return MR_STEP_NONFINITE_RESULT;
        v[d] = nvel;
    }
    if (o->floating) {
        q[0] += o->h * v[0];
        q[1] += o->h * v[1];
        q[2] += o->h * v[2];
        const q4 inc = so3_increment(V(o->h * v[3], o->h * v[4], o->h * v[5]), 1);
        q4 out;
        if (!qnormalize(qmul(inc, Q(q[3], q[4], q[5], q[6])), &out, 0)) return MR_STEP_NONFINITE_RESULT;
        q[3] = out.x; q[4] = out.y; q[5] = out.z; q[6] = out.w;
    }
    for (uint32_t b = 1; b < o->nb; ++b) {
        const int dof = o->body_dof[b];
        if (dof < 0) continue;
        const MRModelJointC* j = &o->joints[o->bodies[b].inbound_joint];
        q[j->q_index] = rn(q[j->q_index] + o->h * v[dof]);
    }
    for (uint32_t i = 0; i < o->w.nq; ++i)
        if (!isfinite(q[i])) return MR_STEP_NONFINITE_RESULT;
    return MR_STEP_SUCCESS;
}

/* One control step: prepare (reset + checkpoint), substeps, latch,
 * commit-or-restore (MetalWorld.metal:113-518, MetalWorldContact.metal:9051). */
uint32_t oracle_control_step(const OracleWorld* o, double* q, double* v, OracleManifold* manifolds, const double* actions,
                             double friction_scale, int reset, const double* reset_q, const double* reset_v,
                             OracleTrace* trace) {
    const uint32_t nq = o->w.nq, nv = o->w.nv, np = o->w.pair_count;
    OracleTrace local;
    if (!trace) trace = &local;
    memset(trace, 0, sizeof(*trace));
    g_band = 0;
    g_margin = INFINITY;
    trace->failing_substep = MR_INVALID_INDEX;
    trace->failing_index = MR_INVALID_INDEX;
    if (reset) {
        memcpy(q, reset_q, sizeof(double) * nq);
        memcpy(v, reset_v, sizeof(double) * nv);
        if (np) memset(manifolds, 0, sizeof(OracleManifold) * np);
    }
    double qc[MAXQ], vc[MAXV];
    static __thread OracleManifold mc[MAXP];
    memcpy(qc, q, sizeof(double) * nq);
    memcpy(vc, v, sizeof(double) * nv);
    if (np) memcpy(mc, manifolds, sizeof(OracleManifold) * np);
    uint32_t status = MR_STEP_SUCCESS;
    for (uint32_t s = 0; s < o->substeps; ++s) {
        double tau[MAXV], qdd[MAXV], vf[MAXV];
        oracle_drive_efforts(o, q, v, actions, tau);
        Kin k;
        status = kinematics(o, q, v, &k);
        uint32_t fail_index = MR_INVALID_INDEX;
        if (status == MR_STEP_SUCCESS) status = aba_core(o, q, v, tau, &k, qdd);
        if (status == MR_STEP_SUCCESS) {
            if (np > 0) {
                for (uint32_t d = 0; d < nv; ++d) {
                    vf[d] = rn(v[d] + o->h * qdd[d]);
                    if (!isfinite(vf[d])) status = MR_STEP_NONFINITE_RESULT;
                }
                if (status == MR_STEP_SUCCESS)
                    status = contact_substep(o, q, v, vf, &k, manifolds, friction_scale, s + 1 == o->substeps, trace, &fail_index);
            } else {
                status = integrate_free(o, q, v, qdd);
            }
        }
        if (status != MR_STEP_SUCCESS) {
            trace->failing_substep = s;
            trace->failing_index = fail_index;
            break;
        }
    }
    trace->status = status;
    trace->band_decisions = g_band;
    trace->min_decision_margin = g_margin;
    if (status != MR_STEP_SUCCESS) {
        memcpy(q, qc, sizeof(double) * nq);
        memcpy(v, vc, sizeof(double) * nv);
        if (np) memcpy(manifolds, mc, sizeof(OracleManifold) * np);
        trace->contact_count = 0;
    }
    return status;
}

/* ------------------------------------------------------------------ */
void oracle_manifold_from_device(const MRManifoldC* in, OracleManifold* out, uint32_t count) {
    for (uint32_t m = 0; m < count; ++m) {
        memset(&out[m], 0, sizeof(OracleManifold));
        for (int a = 0; a < 3; ++a) { out[m].normal_local[a] = in[m].normal_local[a]; out[m].tangent_local[a] = in[m].tangent_local[a]; }
        out[m].age = in[m].age;
        out[m].count = in[m].count;
        for (int p = 0; p < MPTS; ++p) {
            for (int a = 0; a < 3; ++a) {
                out[m].points[p].anchor_a[a] = in[m].points[p].anchor_a[a];
                out[m].points[p].anchor_b[a] = in[m].points[p].anchor_b[a];
                out[m].points[p].impulses[a] = in[m].points[p].impulses[a];
            }
            out[m].points[p].feature_a = in[m].points[p].feature_a;
            out[m].points[p].feature_b = in[m].points[p].feature_b;
            out[m].points[p].life = in[m].points[p].life;
        }
    }
}

void oracle_manifold_to_device(const OracleManifold* in, MRManifoldC* out, uint32_t count) {
    for (uint32_t m = 0; m < count; ++m) {
        memset(&out[m], 0, sizeof(MRManifoldC));
        for (int a = 0; a < 3; ++a) { out[m].normal_local[a] = (float)in[m].normal_local[a]; out[m].tangent_local[a] = (float)in[m].tangent_local[a]; }
        out[m].age = (float)in[m].age;
        out[m].count = in[m].count;
        for (int p = 0; p < MPTS; ++p) {
            for (int a = 0; a < 3; ++a) {
                out[m].points[p].anchor_a[a] = (float)in[m].points[p].anchor_a[a];
                out[m].points[p].anchor_b[a] = (float)in[m].points[p].anchor_b[a];
                out[m].points[p].impulses[a] = (float)in[m].points[p].impulses[a];
            }
            out[m].points[p].feature_a = in[m].points[p].feature_a;
            out[m].points[p].feature_b = in[m].points[p].feature_b;
            out[m].points[p].life = in[m].points[p].life;
        }
    }
}

/* Temporal-cone Jacobi iteration on an explicit Delassus problem, with the
 * same preconditioner / relaxation / projection as the contact substep. */
void oracle_temporal_cone_dense(uint32_t n, const double* W, const double* u0, const double* mu, uint32_t iterations, double* lambda) {
    const uint32_t m = 3 * n;
    double P[MAXC][9], relax[MAXC], delta[3 * MAXC], u[3 * MAXC];
    for (uint32_t i = 0; i < n; ++i) {
        double B[9];
        for (int r = 0; r < 3; ++r)
            for (int s = 0; s < 3; ++s) B[r * 3 + s] = W[(3 * i + r) * m + 3 * i + s];
        oracle_invert3x3(B, P[i]);
        double rowsum = 0.0, diag = 0.0;
        for (uint32_t j = 0; j < n; ++j) {
            const double a = W[(3 * i) * m + 3 * j];
            rowsum += fabs(a);
            if (i == j) diag = fabs(a);
        }
        relax[i] = rowsum > fmax(diag, kMatrixFloor) ? fmin(fmax(diag / rowsum, 1.0 / 32.0), 1.0) : 1.0;
        double warm[3];
        oracle_project_cone(&lambda[3 * i], mu[i], mu[i], warm);
        for (int a = 0; a < 3; ++a) lambda[3 * i + a] = warm[a];
    }
    for (uint32_t it = 0; it < iterations; ++it) {
        for (uint32_t r = 0; r < m; ++r) {
            double s = u0[r];
            for (uint32_t c = 0; c < m; ++c) s += W[r * m + c] * lambda[c];
            u[r] = s;
        }
        for (uint32_t i = 0; i < n; ++i) {
            double rhs[3], prop[3], proj[3];
            for (int r = 0; r < 3; ++r) rhs[r] = -u[3 * i + r];
            for (int r = 0; r < 3; ++r) prop[r] = lambda[3 * i + r] + P[i][r * 3] * rhs[0] + P[i][r * 3 + 1] * rhs[1] + P[i][r * 3 + 2] * rhs[2];
            oracle_project_cone(prop, mu[i], mu[i], proj);
            for (int r = 0; r < 3; ++r) delta[3 * i + r] = relax[i] * (proj[r] - lambda[3 * i + r]);
        }
        for (uint32_t r = 0; r < m; ++r) lambda[r] += delta[r];
    }
}

/* ================================================================== */
/* Free-body scene worlds: piles of spheres and boxes on a plane.       */
/* FP64 restatement of the device scene step (same stage order):       */
/* prediction (MetalWorldContact.metal:2509-2570), speculative sweep    */
/* (Collision.metal:5960-6030), pair flags (Collision.metal:7905-8180), */
/* analytic narrowphase (Collision.cpp:1106-2175: sphere-sphere,        */
/* sphere-box witness, box-box separating axes with vertex clipping,    */
/* sphere/box vs plane), persistent manifolds keyed by collider pair,   */
/* ConstraintIR, islands (ConstraintSolver.cpp:848-900), temporalCone   */
/* with free-body responses, speed clamps and exponential-map           */
/* integration.                                                         */
/* ================================================================== */

#define SNB ORACLE_SCENE_MAX_BODIES
#define SMAN ORACLE_SCENE_MANIFOLDS
#define SCON ORACLE_SCENE_CONTACTS
#define SCAND ORACLE_SCENE_CANDIDATES
#define SPAIRS (SNB * (SNB - 1) / 2 + SNB)
#define SHULL 1024 /* hull vertices of a scene's convex bodies */

struct OracleScene {
    uint32_t nb, np;
    double h;
    uint32_t substeps, iters, final_iters;
    double gravity[3], slop, max_dep, spec_scale, speed_env, thr[4];
    v3 plane_pos, ground_pos;
    q4 plane_rot, ground_rot;
    double plane_offset, plane_rest;
    uint32_t plane_material;
    uint32_t type[SNB], material[SNB];
    double dims[SNB][3], mass[SNB], inv_mass[SNB], damp_lin[SNB], damp_ang[SNB];
    double inv_inertia[SNB][3], max_lin[SNB], max_ang[SNB];
    double offset[SNB], rest[SNB], sweep[SNB];
    double fric[4][2], resp[4][4];
    uint8_t pa[SPAIRS], pb[SPAIRS], pc[SPAIRS];
    /* Convex bodies: hull vertices scaled by the body's dimensions. */
    int hull_first[SNB], hull_count[SNB];
    double hull[SHULL][3];
};

OracleScene* oracle_scene_create(const MRModelWorldC* w, const MRModelBodyC* bodies, const MRModelShapeC* shapes,
                                 const MRModelMaterialC* materials, const MRModelPairC* pairs, const float* hull_vertices,
                                 uint32_t hull_vertex_count, double h, uint32_t substeps, uint32_t iters, uint32_t final_iters) {
    OracleScene* s = (OracleScene*)calloc(1, sizeof(OracleScene));
    const uint32_t n = w->body_count - 1;
    s->nb = n;
    s->np = w->pair_count;
    s->h = h;
    s->substeps = substeps;
    s->iters = iters;
    s->final_iters = final_iters;
    for (int i = 0; i < 3; ++i) s->gravity[i] = w->gravity[i];
    s->slop = w->solver_scales[3];
    s->max_dep = w->solver_scales[2];
    s->spec_scale = w->speculative[0];
    s->speed_env = w->speculative[1];
    for (int i = 0; i < 4; ++i) s->thr[i] = w->manifold_thresholds[i];
    const MRModelShapeC* plane = &shapes[n];
    const MRModelBodyC* ground = &bodies[n];
    s->plane_pos = V(ground->static_pose[0] + plane->local_position[0], ground->static_pose[1] + plane->local_position[1],
                     ground->static_pose[2] + plane->local_position[2]);
    /* The device stores the normalised rotation in FP32. */
    {
        const double qx = plane->local_rotation[0], qy = plane->local_rotation[1], qz = plane->local_rotation[2],
                     qw = plane->local_rotation[3];
        const double nr = sqrt(qx * qx + qy * qy + qz * qz + qw * qw);
        s->plane_rot = Q((float)(qx / nr), (float)(qy / nr), (float)(qz / nr), (float)(qw / nr));
    }
    s->ground_pos = V(ground->static_pose[0], ground->static_pose[1], ground->static_pose[2]);
    {
        const double qx = ground->static_pose[4], qy = ground->static_pose[5], qz = ground->static_pose[6],
                     qw = ground->static_pose[7];
        const double nr = sqrt(qx * qx + qy * qy + qz * qz + qw * qw);
        s->ground_rot = Q((float)(qx / nr), (float)(qy / nr), (float)(qz / nr), (float)(qw / nr));
    }
    s->plane_offset = plane->contact_rest_bound[0];
    s->plane_rest = plane->contact_rest_bound[1];
    s->plane_material = plane->material;
    for (uint32_t b = 0; b < n; ++b) {
        s->type[b] = shapes[b].shape_type;
        s->material[b] = shapes[b].material;
        for (int i = 0; i < 3; ++i) s->dims[b][i] = shapes[b].dimensions[i];
        if (shapes[b].shape_type == MR_SHAPE_CONVEX) {
            int used = 0;
            for (uint32_t a = 0; a < b; ++a) used += s->hull_count[a];
            if (!hull_vertices || shapes[b].hull_count == 0 || used + (int)shapes[b].hull_count > SHULL ||
                shapes[b].hull_first + shapes[b].hull_count > hull_vertex_count) {
                free(s);
                return NULL;
            }
            s->hull_first[b] = used;
            s->hull_count[b] = (int)shapes[b].hull_count;
            for (uint32_t i = 0; i < shapes[b].hull_count; ++i)
                for (int c = 0; c < 3; ++c)
                    s->hull[used + i][c] = (double)hull_vertices[4 * (shapes[b].hull_first + i) + c] * shapes[b].dimensions[c];
        }
        s->mass[b] = bodies[b].mass_inverse_mass[0];
        s->inv_mass[b] = bodies[b].mass_inverse_mass[1];
        s->damp_lin[b] = w->apply_body_damping ? bodies[b].damping_speed[0] : 0.0;
        s->damp_ang[b] = w->apply_body_damping ? bodies[b].damping_speed[1] : 0.0;
        for (int i = 0; i < 3; ++i) s->inv_inertia[b][i] = (float)(1.0f / bodies[b].inertia[i][i]);
        s->max_lin[b] = bodies[b].damping_speed[2];
        s->max_ang[b] = bodies[b].damping_speed[3];
        s->offset[b] = shapes[b].contact_rest_bound[0];
        s->rest[b] = shapes[b].contact_rest_bound[1];
        s->sweep[b] = shapes[b].contact_rest_bound[2];
    }
    for (uint32_t i = 0; i < w->material_count && i < 4; ++i) {
        s->fric[i][0] = materials[i].friction[0];
        s->fric[i][1] = materials[i].friction[1];
        for (int k = 0; k < 4; ++k) s->resp[i][k] = materials[i].response[k];
    }
    for (uint32_t p = 0; p < s->np; ++p) {
        s->pa[p] = (uint8_t)pairs[p].shape_a;
        s->pb[p] = (uint8_t)pairs[p].shape_b;
        s->pc[p] = (uint8_t)pairs[p].pair_class;
    }
    return s;
}

void oracle_scene_destroy(OracleScene* s) { free(s); }

typedef struct {
    int type;
    v3 c;
    q4 r;
    v3 half;
    double radius, offset;
    v3 lo, hi, normal;
    v3 e0, e1; /* capsule segment endpoints (local -Y / +Y ends) */
    v3 axis, bx, bz; /* cylinder axis (local +Y) and disk basis */
    double hl;       /* cylinder half length */
    v3 bpos; /* pose of the collider's body: the frame of its manifold anchors */
    q4 brot;
    const double* hull; /* convex: scaled local hull vertices, xyz each */
    int hull_count;
} SCol;

typedef struct {
    double lo[SNB][3], hi[SNB][3], margin[SNB];
    v3 pos[SNB], lin[SNB], ang[SNB];
    q4 rot[SNB];
    double iiw[SNB][6];
} SState;

static void scol(const OracleScene* s, const SState* st, uint32_t b, SCol* o) {
    if (b >= s->nb) {
        o->type = MR_SHAPE_PLANE;
        o->c = s->plane_pos;
        o->r = s->plane_rot;
        const v3 n = qrot(o->r, V(0, 1, 0));
        o->normal = vmul(n, 1.0 / vlen(n));
        o->half = V(0, 0, 0);
        o->radius = 0.0;
        o->offset = s->plane_offset;
        o->lo = o->hi = V(0, 0, 0);
        o->e0 = o->e1 = o->c;
        o->axis = o->bx = o->bz = V(0, 0, 0);
        o->hl = 0.0;
        o->bpos = s->ground_pos;
        o->brot = s->ground_rot;
        o->hull = NULL;
        o->hull_count = 0;
        return;
    }
    o->type = (int)s->type[b];
    o->hull = s->hull[s->hull_first[b]];
    o->hull_count = o->type == MR_SHAPE_CONVEX ? s->hull_count[b] : 0;
    o->c = st->pos[b];
    o->r = st->rot[b];
    o->half = V(s->dims[b][0], s->dims[b][1], s->dims[b][2]);
    o->radius = s->dims[b][0];
    o->offset = s->offset[b] + st->margin[b];
    o->lo = V(st->lo[b][0], st->lo[b][1], st->lo[b][2]);
    o->hi = V(st->hi[b][0], st->hi[b][1], st->hi[b][2]);
    if (o->type == MR_SHAPE_CAPSULE) {
        const v3 axis = qrot(o->r, V(0, s->dims[b][1], 0));
        o->e0 = vsub(o->c, axis);
        o->e1 = vadd(o->c, axis);
    } else {
        o->e0 = o->e1 = o->c;
    }
    o->hl = s->dims[b][1];
    if (o->type == MR_SHAPE_CYLINDER) {
        /* Collision.metal:759-784: unit axis, disk basis X orthogonalised
         * against it, Z = X x axis. */
        const v3 ax = qrot(o->r, V(0, 1, 0));
        o->axis = vmul(ax, 1.0 / vlen(ax));
        v3 bx = qrot(o->r, V(1, 0, 0));
        bx = vsub(bx, vmul(o->axis, vdot(o->axis, bx)));
        o->bx = vmul(bx, 1.0 / vlen(bx));
        const v3 bz = vcross(o->bx, o->axis);
        o->bz = vmul(bz, 1.0 / vlen(bz));
    } else {
        o->axis = o->bx = o->bz = V(0, 0, 0);
    }
    o->normal = V(0, 0, 0);
    o->bpos = o->c;
    o->brot = o->r;
}

static double scol_scale(const SCol* k) {
    return fmax(fmax(vmaxabs(k->c), vmaxabs(k->half)),
                fmax(fabs(k->radius), fmax(fabs(k->offset), fmax(vmaxabs(k->lo), vmaxabs(k->hi)))));
}
static v3 sbox_axis(const SCol* b, int a) { return qrot(b->r, V(a == 0, a == 1, a == 2)); }
static double sbox_radius(const SCol* b, v3 ax) {
    return fabs(vdot(ax, sbox_axis(b, 0))) * b->half.x + fabs(vdot(ax, sbox_axis(b, 1))) * b->half.y +
           fabs(vdot(ax, sbox_axis(b, 2))) * b->half.z;
}
static v3 sbox_vertex(const SCol* b, int v) {
    return vadd(b->c, qrot(b->r, V((v & 1) ? b->half.x : -b->half.x, (v & 2) ? b->half.y : -b->half.y,
                                   (v & 4) ? b->half.z : -b->half.z)));
}
static int sinside(v3 p, const SCol* b, double infl) {
    const v3 l = qrotinv(b->r, vsub(p, b->c));
    BAND(fabs(l.x), b->half.x + infl);
    BAND(fabs(l.y), b->half.y + infl);
    BAND(fabs(l.z), b->half.z + infl);
    return fabs(l.x) <= b->half.x + infl && fabs(l.y) <= b->half.y + infl && fabs(l.z) <= b->half.z + infl;
}
static v3 sbox_support(const SCol* b, v3 d) {
    v3 out = b->c;
    for (int a = 0; a < 3; ++a) {
        const v3 ax = sbox_axis(b, a);
        const double he = a == 0 ? b->half.x : (a == 1 ? b->half.y : b->half.z);
        BAND(vdot(d, ax), 0.0); /* an edge across the normal: either end supports */
        out = vadd(out, vmul(ax, vdot(d, ax) >= 0.0 ? he : -he));
    }
    return out;
}
static v3 scoincident(uint32_t a, uint32_t b) {
    const uint32_t hsh = a * 73856093u ^ b * 19349663u;
    const uint32_t axis = hsh % 3u;
    const double sign = (hsh & 4u) == 0u ? 1.0 : -1.0;
    return V(axis == 0 ? sign : 0.0, axis == 1 ? sign : 0.0, axis == 2 ? sign : 0.0);
}

typedef struct {
    int n;
    uint32_t status; /* a support-mapped query that failed (MR_STEP_*), else 0 */
    uint32_t path;   /* support-mapped queries: 0 GJK distance, 3 EPA, 1 MPR */
    double sep[8];
    v3 pa[8], pb[8];
    uint32_t fa[8], fb[8];
} SRaw;

static void sraw_add(SRaw* r, v3 pa, v3 pb, double sep, uint32_t fa, uint32_t fb) {
    if (r->n >= 8) return;
    r->pa[r->n] = rn3(pa);
    r->pb[r->n] = rn3(pb);
    r->sep[r->n] = rn(sep);
    r->fa[r->n] = fa;
    r->fb[r->n] = fb;
    r->n++;
}

/* Segment helpers of the capsule classes (Collision.cpp:1169-1336). */
static const double kSceneTiny = 1.0e-14; /* Collision.cpp:48, Collision.metal:10 */
static uint32_t scap_feature(double t) { return t <= 0.0 ? 0u : (t >= 1.0 ? 1u : 2u); }

static v3 sstable_segment_normal(v3 da, v3 db, uint32_t ia, uint32_t ib) {
    const v3 cr = vcross(da, db);
    if (vdot(cr, cr) > kSceneTiny) return vmul(cr, 1.0 / vlen(cr));
    v3 dir;
    if (vdot(da, da) > kSceneTiny) dir = vmul(da, 1.0 / vlen(da));
    else if (vdot(db, db) > kSceneTiny) dir = vmul(db, 1.0 / vlen(db));
    else return scoincident(ia, ib);
    const double ax = fabs(dir.x), ay = fabs(dir.y), az = fabs(dir.z);
    const v3 ref = (ax <= ay && ax <= az) ? V(1, 0, 0) : (ay <= az ? V(0, 1, 0) : V(0, 0, 1));
    v3 out = vcross(dir, ref);
    out = vmul(out, 1.0 / vlen(out));
    return (((ia * 73856093u) ^ (ib * 19349663u)) & 4u) ? vmul(out, -1.0) : out;
}

/* Clamp of a segment parameter with the feature decisions at 0 and 1 taken
 * in length units (band). */
static double sclamp01(double t, double len) {
    BAND(t * len, 0.0);
    BAND(t * len, len);
    return fmin(fmax(t, 0.0), 1.0);
}

static v3 sclosest_on_segment(v3 x, v3 e0, v3 e1, double* t) {
    const v3 seg = vsub(e1, e0);
    const double sq = vdot(seg, seg);
    if (!(sq > kSceneTiny)) { *t = 0.0; return e0; }
    *t = sclamp01(vdot(vsub(x, e0), seg) / sq, sqrt(sq));
    return vadd(e0, vmul(seg, *t));
}

static void sclosest_segments(v3 a0, v3 a1, v3 b0, v3 b1, v3* pa, v3* pb, double* ta, double* tb) {
    const v3 da = vsub(a1, a0), db = vsub(b1, b0), off = vsub(a0, b0);
    const double sa = vdot(da, da), sb = vdot(db, db), pa_ = vdot(da, off), pb_ = vdot(db, off);
    const double la = sqrt(sa), lb = sqrt(sb);
    *ta = 0.0;
    *tb = 0.0;
    if (!(sa > kSceneTiny) && !(sb > kSceneTiny)) { *pa = a0; *pb = b0; return; }
    if (!(sa > kSceneTiny)) {
        *tb = sclamp01(pb_ / sb, lb);
    } else {
        const double cp = vdot(da, db);
        if (!(sb > kSceneTiny)) {
            *ta = sclamp01(-pa_ / sa, la);
        } else {
            const double den = sa * sb - cp * cp;
            /* Near-parallel segments: the FP32 test may go the other way. */
            if (fabs(den - kSceneTiny * sa * sb) <= 64.0 * kFloatEps * sa * sb) g_band++;
            if (den > kSceneTiny * sa * sb) *ta = sclamp01((cp * pb_ - pa_ * sb) / den, la);
            *tb = (cp * *ta + pb_) / sb;
            BAND(*tb * lb, 0.0);
            BAND(*tb * lb, lb);
            if (*tb < 0.0) {
                *tb = 0.0;
                *ta = sclamp01(-pa_ / sa, la);
            } else if (*tb > 1.0) {
                *tb = 1.0;
                *ta = sclamp01((cp - pa_) / sa, la);
            }
        }
    }
    *pa = vadd(a0, vmul(da, *ta));
    *pb = vadd(b0, vmul(db, *tb));
}

typedef struct {
    v3 normal, cap_point, box_point;
    double sep, t_cap;
    uint32_t box_feature;
} SCapBox;

/* Capsule-box witness (Collision.cpp:1462-1690, Collision.metal:1241). */
static SCapBox scapsule_box(const SCol* cap, const SCol* box, uint32_t ic, uint32_t ib) {
    SCapBox w;
    const v3 s0 = qrotinv(box->r, vsub(cap->e0, box->c)), s1 = qrotinv(box->r, vsub(cap->e1, box->c));
    const v3 dir = vsub(s1, s0);
    const double he[3] = {box->half.x, box->half.y, box->half.z};
    const double st[3] = {s0.x, s0.y, s0.z}, dd[3] = {dir.x, dir.y, dir.z};
    const double seglen = vlen(dir);
    double enter = 0.0, exit_ = 1.0;
    int inside = 1;
    for (int a = 0; a < 3; ++a) {
        if (fabs(dd[a]) <= kSceneTiny) {
            BAND(fabs(st[a]), he[a]);
            if (st[a] < -he[a] || st[a] > he[a]) inside = 0;
            continue;
        }
        double t0 = (-he[a] - st[a]) / dd[a], t1 = (he[a] - st[a]) / dd[a];
        if (t0 > t1) { const double t = t0; t0 = t1; t1 = t; }
        enter = fmax(enter, t0);
        exit_ = fmin(exit_, t1);
        BAND(enter * seglen, exit_ * seglen);
        if (enter > exit_) inside = 0;
    }
    if (inside) {
        w.t_cap = fmin(fmax(0.5 * (enter + exit_), 0.0), 1.0);
        const v3 core = vadd(s0, vmul(dir, w.t_cap));
        const double cc[3] = {core.x, core.y, core.z};
        const double dist[3] = {he[0] - fabs(cc[0]), he[1] - fabs(cc[1]), he[2] - fabs(cc[2])};
        int axis = 0;
        BAND(dist[1], dist[0]);
        if (dist[1] < dist[axis]) axis = 1;
        BAND(dist[2], dist[axis]);
        if (dist[2] < dist[axis]) axis = 2;
        BAND(cc[axis], 0.0);
        const double sign = cc[axis] >= 0.0 ? 1.0 : -1.0;
        const v3 outward = V(axis == 0 ? sign : 0.0, axis == 1 ? sign : 0.0, axis == 2 ? sign : 0.0);
        v3 lbox = core;
        if (axis == 0) lbox.x = sign * he[0];
        else if (axis == 1) lbox.y = sign * he[1];
        else lbox.z = sign * he[2];
        const v3 ln = vmul(outward, -1.0);
        w.normal = qrot(box->r, ln);
        w.cap_point = vadd(box->c, qrot(box->r, vadd(core, vmul(ln, cap->radius))));
        w.box_point = vadd(box->c, qrot(box->r, lbox));
        w.sep = -dist[axis] - cap->radius;
        w.box_feature = 27u + 2u * (uint32_t)axis + (sign > 0.0 ? 1u : 0u);
        return w;
    }
    double best = INFINITY, best_t = 0.0, best_d = INFINITY;
    v3 best_seg = s0, best_box = s0;
    uint32_t best_f = 0xffffffffu;
#define SCONSIDER(SP, BP, T, F)                                                                  \
    do {                                                                                         \
        const v3 d_ = vsub((BP), (SP));                                                          \
        const double sq_ = vdot(d_, d_);                                                         \
        const double tol_ = 1.0e-12 * (1.0 + fmax(isfinite(best) ? best : 0.0, sq_));          \
        if (isfinite(best_d)) BAND(sqrt(sq_), best_d);                                           \
        if (!isfinite(best) || sq_ < best - tol_ || (fabs(sq_ - best) <= tol_ && (F) < best_f)) { \
            best = sq_;                                                                          \
            best_d = sqrt(sq_);                                                                  \
            best_seg = (SP);                                                                     \
            best_box = (BP);                                                                     \
            best_t = (T);                                                                        \
            best_f = (F);                                                                        \
        }                                                                                        \
    } while (0)
    for (int e = 0; e < 2; ++e) {
        const v3 sp = e == 0 ? s0 : s1;
        const v3 bp = V(fmin(fmax(sp.x, -he[0]), he[0]), fmin(fmax(sp.y, -he[1]), he[1]), fmin(fmax(sp.z, -he[2]), he[2]));
        SCONSIDER(sp, bp, (double)e, (uint32_t)e);
    }
    uint32_t feature = 2u;
    for (int va = 0; va < 3; ++va) {
        const int f0 = (va + 1) % 3, f1 = (va + 2) % 3;
        for (int sg = 0; sg < 4; ++sg) {
            double c0[3], c1[3];
            c0[va] = -he[va];
            c1[va] = he[va];
            c0[f0] = c1[f0] = ((sg & 1) ? 1.0 : -1.0) * he[f0];
            c0[f1] = c1[f1] = ((sg & 2) ? 1.0 : -1.0) * he[f1];
            v3 pa, pb;
            double ta, tb;
            sclosest_segments(s0, s1, V(c0[0], c0[1], c0[2]), V(c1[0], c1[1], c1[2]), &pa, &pb, &ta, &tb);
            SCONSIDER(pa, pb, ta, feature);
            ++feature;
        }
    }
#undef SCONSIDER
    const double dist = sqrt(fmax(best, 0.0));
    const v3 ln = dist > kSceneTiny ? vmul(vsub(best_box, best_seg), 1.0 / dist) : qrotinv(box->r, scoincident(ic, ib));
    w.normal = qrot(box->r, ln);
    w.cap_point = vadd(box->c, qrot(box->r, vadd(best_seg, vmul(ln, cap->radius))));
    w.box_point = vadd(box->c, qrot(box->r, best_box));
    w.sep = dist - cap->radius;
    w.t_cap = best_t;
    w.box_feature = 64u + best_f;
    return w;
}

/* ---- Support-mapped queries: GJK, EPA and the cylinder patch ---------------
 * Restates the reference's primitive-GJK class (MR_WORLD_WORK_PRIMITIVE_GJK,
 * Collision.metal:8026-8045): supports 1756-1972, simplex reduction
 * 1974-2296, gjkDistance 2298-2427, epaPenetration 2511-2783, the support
 * patch 3279-3432 and supportMappedContacts 3434-3620.  The device kernel
 * runs the same steps in FP32; the query cache that warm-starts the
 * reference's GJK direction is not kept (the first direction is always the
 * centre difference).  EPA orients its faces against an interior point
 * (see sface).  A query that neither EPA nor the MPR fallback resolves
 * fails the step with MR_STEP_DID_NOT_CONVERGE, as in the reference. */
#define GJK_ITERS 32  /* MR_GJK_MAX_ITERATIONS, engine_types.h:56 */
#define EPA_ITERS 48  /* MR_EPA_MAX_ITERATIONS */
#define EPA_VERTS 64  /* MR_EPA_VERTEX_CAPACITY */
#define EPA_FACES 128 /* MR_EPA_FACE_CAPACITY */
static const double kCylAlign = 1.0e-6; /* Collision.metal:21 */
enum { kCylNegRing = 0u, kCylPosRing = 4u, kCylNegSide = 8u, kCylPosSide = 9u, kCylNegRim = 10u, kCylPosRim = 11u };
/* Weight / barycentric near-ties that may pick another feature in FP32. */
static const double kFeatureTie = 1.0e-4;

typedef struct {
    v3 w, pa, pb; /* Minkowski point A - B and its two supports */
    uint32_t fa, fb;
} SSup;

static v3 sdeterministic(uint32_t key) {
    const uint32_t axis = key % 3u;
    const double sign = (key & 4u) == 0u ? 1.0 : -1.0;
    return V(axis == 0 ? sign : 0.0, axis == 1 ? sign : 0.0, axis == 2 ? sign : 0.0);
}

/* Support point of a finite shape along d (normalised here). */
static v3 ssupport(const SCol* k, uint32_t index, v3 d, uint32_t* feat) {
    const double dd = vdot(d, d);
    d = (!(dd > kSceneTiny) || !isfinite(dd)) ? sdeterministic(index) : vmul(d, 1.0 / sqrt(dd));
    if (k->type == MR_SHAPE_SPHERE) {
        *feat = feature_key(MR_SHAPE_SPHERE, 0u);
        return vadd(k->c, vmul(d, k->radius));
    }
    if (k->type == MR_SHAPE_CAPSULE) {
        const double proj = vdot(d, vsub(k->e1, k->e0));
        BAND(proj, 0.0);
        const int pos = proj >= 0.0;
        *feat = feature_key(MR_SHAPE_CAPSULE, pos ? 1u : 0u);
        return vadd(pos ? k->e1 : k->e0, vmul(d, k->radius));
    }
    if (k->type == MR_SHAPE_BOX) {
        const v3 l = qrotinv(k->r, d);
        /* A direction across a face or edge picks its vertex by rounding. */
        BAND(l.x, 0.0);
        BAND(l.y, 0.0);
        BAND(l.z, 0.0);
        uint32_t v = 0u;
        v3 p = V(-k->half.x, -k->half.y, -k->half.z);
        if (l.x >= 0.0) { v |= 1u; p.x = k->half.x; }
        if (l.y >= 0.0) { v |= 2u; p.y = k->half.y; }
        if (l.z >= 0.0) { v |= 4u; p.z = k->half.z; }
        *feat = feature_key(MR_SHAPE_BOX, v);
        return vadd(k->c, qrot(k->r, p));
    }
    if (k->type == MR_SHAPE_CONVEX) {
        /* The vertex of largest projection, the lowest index on a tie
         * (Collision.metal:1899-1936); a near tie is a band decision. */
        const v3 l = qrotinv(k->r, d);
        double best = -INFINITY, second = -INFINITY;
        int bi = 0;
        for (int i = 0; i < k->hull_count; ++i) {
            const double pr = k->hull[3 * i] * l.x + k->hull[3 * i + 1] * l.y + k->hull[3 * i + 2] * l.z;
            if (pr > best) { second = best; best = pr; bi = i; }
            else if (pr > second) second = pr;
        }
        if (k->hull_count > 1) BAND(best - second, 0.0);
        *feat = feature_key(MR_SHAPE_CONVEX, (uint32_t)bi);
        return vadd(k->c, qrot(k->r, V(k->hull[3 * bi], k->hull[3 * bi + 1], k->hull[3 * bi + 2])));
    }
    /* cylinder */
    const double axial = vdot(d, k->axis);
    const v3 radial = vsub(d, vmul(k->axis, axial));
    const double rsq = vdot(radial, radial);
    const v3 rdir = rsq > kSceneTiny ? vmul(radial, 1.0 / sqrt(rsq)) : k->bx;
    const int pos = axial >= 0.0;
    uint32_t local = pos ? kCylPosRim : kCylNegRim;
    BAND(fabs(axial), kCylAlign);
    if (fabs(axial) <= kCylAlign) {
        const double x = vdot(rdir, k->bx), z = vdot(rdir, k->bz);
        local = 32u + (fabs(x) >= fabs(z) ? (x >= 0.0 ? 0u : 1u) : (z >= 0.0 ? 2u : 3u));
    } else if (rsq <= kSceneTiny) {
        local = pos ? 17u : 16u;
    }
    *feat = feature_key(MR_SHAPE_CYLINDER, local);
    return vadd(vadd(k->c, vmul(k->axis, pos ? k->hl : -k->hl)), vmul(rdir, k->radius));
}

static void sminkowski(const SCol* A, const SCol* B, uint32_t ia, uint32_t ib, v3 d, SSup* o) {
    o->pa = ssupport(A, ia, d, &o->fa);
    o->pb = ssupport(B, ib, vmul(d, -1.0), &o->fb);
    o->w = vsub(o->pa, o->pb);
}

/* Closest point to the origin on triangle abc with its barycentric weights
 * (the Voronoi-region walk of Ericson, Real-Time Collision Detection 5.1.5). */
static v3 sclosest_triangle(v3 a, v3 b, v3 c, double* wt) {
    const v3 ab = vsub(b, a), ac = vsub(c, a), ap = vmul(a, -1.0);
    const double d1 = vdot(ab, ap), d2 = vdot(ac, ap);
    if (d1 <= 0.0 && d2 <= 0.0) { wt[0] = 1; wt[1] = 0; wt[2] = 0; return a; }
    const v3 bp = vmul(b, -1.0);
    const double d3 = vdot(ab, bp), d4 = vdot(ac, bp);
    if (d3 >= 0.0 && d4 <= d3) { wt[0] = 0; wt[1] = 1; wt[2] = 0; return b; }
    const double vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) {
        const double den = d1 - d3, v = den > kSceneTiny ? d1 / den : 0.0;
        wt[0] = 1.0 - v; wt[1] = v; wt[2] = 0;
        return vadd(a, vmul(ab, v));
    }
    const v3 cp = vmul(c, -1.0);
    const double d5 = vdot(ab, cp), d6 = vdot(ac, cp);
    if (d6 >= 0.0 && d5 <= d6) { wt[0] = 0; wt[1] = 0; wt[2] = 1; return c; }
    const double vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) {
        const double den = d2 - d6, w = den > kSceneTiny ? d2 / den : 0.0;
        wt[0] = 1.0 - w; wt[1] = 0; wt[2] = w;
        return vadd(a, vmul(ac, w));
    }
    const double va = d3 * d6 - d5 * d4;
    if (va <= 0.0 && (d4 - d3) >= 0.0 && (d5 - d6) >= 0.0) {
        const double den = (d4 - d3) + (d5 - d6), w = den > kSceneTiny ? (d4 - d3) / den : 0.0;
        wt[0] = 0; wt[1] = 1.0 - w; wt[2] = w;
        return vadd(b, vmul(vsub(c, b), w));
    }
    const double den = va + vb + vc;
    if (!(fabs(den) > kSceneTiny) || !isfinite(den)) { wt[0] = 1; wt[1] = 0; wt[2] = 0; return a; }
    const double v = vb / den, w = vc / den;
    wt[0] = 1.0 - v - w; wt[1] = v; wt[2] = w;
    return vadd(vadd(a, vmul(ab, v)), vmul(ac, w));
}

/* Drops vertices of weight <= 1e-7 (keeps the heaviest if none is left)
 * and renormalises. */
static void scompress(SSup* sx, int* n, double* wt) {
    SSup keep[4];
    double kw[4];
    int m = 0, best = 0;
    for (int i = 1; i < *n; ++i)
        if (wt[i] > wt[best]) best = i;
    for (int i = 0; i < *n; ++i)
        if (wt[i] > 1.0e-7) { keep[m] = sx[i]; kw[m] = wt[i]; ++m; }
    if (m == 0) { keep[0] = sx[best]; kw[0] = 1.0; m = 1; }
    double tot = 0.0;
    for (int i = 0; i < m; ++i) tot += kw[i];
    const double inv = tot > kSceneTiny ? 1.0 / tot : 1.0;
    for (int i = 0; i < m; ++i) { sx[i] = keep[i]; wt[i] = kw[i] * inv; }
    *n = m;
}

static double striple(v3 a, v3 b, v3 c) { return vdot(a, vcross(b, c)); }

/* Closest point of the simplex to the origin; returns 1 when a tetrahedron
 * contains it. */
static int sclosest_simplex(SSup* sx, int* n, double* wt, v3* closest) {
    if (*n == 1) { wt[0] = 1.0; *closest = sx[0].w; return 0; }
    if (*n == 2) {
        const v3 a = sx[0].w, e = vsub(sx[1].w, a);
        const double den = vdot(e, e);
        const double t = den > kSceneTiny ? fmin(fmax(-vdot(a, e) / den, 0.0), 1.0) : 0.0;
        wt[0] = 1.0 - t;
        wt[1] = t;
        *closest = vadd(a, vmul(e, t));
        scompress(sx, n, wt);
        return 0;
    }
    if (*n == 3) {
        *closest = sclosest_triangle(sx[0].w, sx[1].w, sx[2].w, wt);
        scompress(sx, n, wt);
        return 0;
    }
    const v3 a = sx[0].w, ab = vsub(sx[1].w, a), ac = vsub(sx[2].w, a), ad = vsub(sx[3].w, a);
    const double det = striple(ab, ac, ad);
    if (fabs(det) > kSceneTiny && isfinite(det)) {
        const v3 na = vmul(a, -1.0);
        const double u = striple(na, ac, ad) / det, v = striple(ab, na, ad) / det, w = striple(ab, ac, na) / det;
        const double base = 1.0 - u - v - w, tol = -2.0e-6;
        if (base >= tol && u >= tol && v >= tol && w >= tol) {
            wt[0] = base; wt[1] = u; wt[2] = v; wt[3] = w;
            *closest = V(0, 0, 0);
            return 1;
        }
    }
    static const int faces[4][3] = {{0, 1, 2}, {0, 3, 1}, {0, 2, 3}, {1, 3, 2}};
    double best = INFINITY, bw[4] = {0, 0, 0, 0};
    v3 bp = V(0, 0, 0);
    for (int f = 0; f < 4; ++f) {
        double tw[3];
        const v3 p = sclosest_triangle(sx[faces[f][0]].w, sx[faces[f][1]].w, sx[faces[f][2]].w, tw);
        const double dist = vdot(p, p);
        if (dist < best) {
            best = dist;
            bp = p;
            bw[0] = bw[1] = bw[2] = bw[3] = 0.0;
            for (int k = 0; k < 3; ++k) bw[faces[f][k]] = tw[k];
        }
    }
    *closest = bp;
    for (int i = 0; i < 4; ++i) wt[i] = bw[i];
    scompress(sx, n, wt);
    return 0;
}

typedef struct {
    uint32_t status;
    uint32_t path; /* how it was resolved: 0 GJK distance, 3 EPA, 1 MPR, 2 support-axis witness (the reference's `fallback`) */
    v3 normal, pa, pb;
    double sep;
    uint32_t fa, fb;
} SQuery;

/* Witness of the simplex: weighted supports, features of the heaviest vertex. */
static void switness(const SSup* sx, int n, const double* wt, SQuery* q) {
    q->pa = q->pb = V(0, 0, 0);
    int best = 0;
    for (int i = 0; i < n; ++i) {
        q->pa = vadd(q->pa, vmul(sx[i].pa, wt[i]));
        q->pb = vadd(q->pb, vmul(sx[i].pb, wt[i]));
        if (wt[i] > wt[best]) best = i;
    }
    for (int i = 0; i < n; ++i)
        if (i != best && wt[best] - wt[i] <= kFeatureTie) g_band++;
    q->fa = sx[best].fa;
    q->fb = sx[best].fb;
}

/* GJK distance; returns 1 on overlap (the simplex then seeds EPA). */
static int sgjk(const SCol* A, const SCol* B, uint32_t ia, uint32_t ib, double scale, SSup* sx, int* n, double* wt,
                SQuery* q) {
    const double tol = 32.0 * kFloatEps * scale;
    v3 d = vsub(B->c, A->c);
    if (vdot(d, d) <= kSceneTiny) d = sdeterministic(ia * 65537u + ib);
    *n = 1;
    sminkowski(A, B, ia, ib, d, &sx[0]);
    wt[0] = 1.0;
    v3 closest = sx[0].w;
    double prev = INFINITY;
    for (int it = 0; it < GJK_ITERS; ++it) {
        const double dsq = vdot(closest, closest);
        if (dsq <= tol * tol) { q->status = MR_STEP_SUCCESS; q->sep = -0.0; return 1; }
        d = vmul(closest, -1.0);
        SSup cand;
        sminkowski(A, B, ia, ib, d, &cand);
        int dup = 0;
        for (int i = 0; i < *n; ++i) {
            const v3 e = vsub(cand.w, sx[i].w);
            dup = dup || vdot(e, e) <= tol * tol;
        }
        /* Advance measured along the unit direction; the reference's
         * unnormalised measure (Collision.metal:2372-2376) lets the distance
         * exceed the true one by tol / distance below 1 m. */
        const double advance = vdot(cand.w, d) - vdot(closest, d);
        int done = dup || advance <= tol * vlen(d);
        if (!done) {
            sx[(*n)++] = cand;
            if (sclosest_simplex(sx, n, wt, &closest)) { q->status = MR_STEP_SUCCESS; q->sep = -0.0; return 1; }
            const double upd = vdot(closest, closest);
            done = prev < INFINITY && prev - upd <= tol * tol;
            prev = upd;
        }
        if (done) {
            switness(sx, *n, wt, q);
            const v3 delta = vsub(q->pb, q->pa);
            const double dist = vlen(delta);
            q->normal = dist > tol ? vmul(delta, 1.0 / dist) : vmul(d, 1.0 / vlen(d));
            q->sep = dist;
            q->status = MR_STEP_SUCCESS;
            return 0;
        }
    }
    q->status = MR_STEP_DID_NOT_CONVERGE;
    return 0;
}

typedef struct {
    int a, b, c, active;
    v3 n;
    double dist;
} SFace;

/* Face abc with its outward unit normal and the origin's distance to its
 * plane.  Outward is taken against `inside`, a point interior to the
 * polytope (the centroid of the initial tetrahedron); the reference orients
 * by the origin's side, which is the same whenever the origin is off the
 * face plane, and ambiguous for a face through the origin (the simplex of a
 * touching or collinear GJK exit), which this keeps outward. */
static int sface(const SSup* vx, int a, int b, int c, v3 inside, SFace* f) {
    v3 n = vcross(vsub(vx[b].w, vx[a].w), vsub(vx[c].w, vx[a].w));
    const double nn = vdot(n, n);
    if (!(nn > kSceneTiny) || !isfinite(nn)) return 0;
    n = vmul(n, 1.0 / sqrt(nn));
    int second = b, third = c;
    if (vdot(n, vsub(vx[a].w, inside)) < 0.0) { n = vmul(n, -1.0); second = c; third = b; }
    const double dist = vdot(n, vx[a].w);
    f->a = a; f->b = second; f->c = third; f->active = 1; f->n = n; f->dist = dist;
    return isfinite(dist);
}

static void shorizon(int* ea, int* eb, int* ne, int a, int b) {
    for (int e = 0; e < *ne; ++e)
        if (ea[e] == b && eb[e] == a) {
            --*ne;
            ea[e] = ea[*ne];
            eb[e] = eb[*ne];
            return;
        }
    if (*ne < 3 * EPA_FACES) { ea[*ne] = a; eb[*ne] = b; ++*ne; }
}

/* EPA from the GJK simplex; returns 1 with the penetration witness. */
static int sepa(const SCol* A, const SCol* B, uint32_t ia, uint32_t ib, double scale, const SSup* seed, int nseed, SQuery* q) {
    static __thread SSup vx[EPA_VERTS];
    static __thread SFace fc[EPA_FACES];
    static __thread int ea[3 * EPA_FACES], eb[3 * EPA_FACES];
    int nv = nseed;
    for (int i = 0; i < nseed; ++i) vx[i] = seed[i];
    static const double dirs[6][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {-1, 0, 0}, {0, -1, 0}, {0, 0, -1}};
    for (int k = 0; nv < 4 && k < 6; ++k) {
        SSup cand;
        sminkowski(A, B, ia, ib, V(dirs[k][0], dirs[k][1], dirs[k][2]), &cand);
        int dup = 0;
        for (int i = 0; i < nv; ++i) {
            const v3 e = vsub(cand.w, vx[i].w);
            dup = dup || vdot(e, e) <= 1.0e-12;
        }
        if (!dup) vx[nv++] = cand;
    }
    if (nv < 4) return 0;
    for (int f = 0; f < EPA_FACES; ++f) fc[f].active = 0;
    const v3 inside = vmul(vadd(vadd(vx[0].w, vx[1].w), vadd(vx[2].w, vx[3].w)), 0.25);
    static const int init[4][3] = {{0, 1, 2}, {0, 3, 1}, {0, 2, 3}, {1, 3, 2}};
    int nf = 0;
    for (int f = 0; f < 4; ++f)
        if (sface(vx, init[f][0], init[f][1], init[f][2], inside, &fc[nf])) ++nf;
    if (nf < 4) return 0;
    const double tol = 64.0 * kFloatEps * scale;
    for (int it = 0; it < EPA_ITERS; ++it) {
        int best = -1;
        double bd = INFINITY;
        for (int f = 0; f < nf; ++f)
            if (fc[f].active && fc[f].dist < bd) { bd = fc[f].dist; best = f; }
        if (best < 0) return 0;
        SSup cand;
        sminkowski(A, B, ia, ib, fc[best].n, &cand);
        const double sd = vdot(fc[best].n, cand.w);
        int dup = 0;
        for (int i = 0; i < nv; ++i) {
            const v3 e = vsub(cand.w, vx[i].w);
            dup = dup || vdot(e, e) <= tol * tol;
        }
        if (dup || sd - bd <= tol) {
            const SFace F = fc[best];
            double bc[3];
            sclosest_triangle(vx[F.a].w, vx[F.b].w, vx[F.c].w, bc);
            q->pa = vadd(vadd(vmul(vx[F.a].pa, bc[0]), vmul(vx[F.b].pa, bc[1])), vmul(vx[F.c].pa, bc[2]));
            q->pb = vadd(vadd(vmul(vx[F.a].pb, bc[0]), vmul(vx[F.b].pb, bc[1])), vmul(vx[F.c].pb, bc[2]));
            int fv = F.a;
            double fw = bc[0];
            if (bc[1] > fw) { fv = F.b; fw = bc[1]; }
            if (bc[2] > fw) { fv = F.c; fw = bc[2]; }
            for (int k = 0; k < 3; ++k) {
                const int vk = k == 0 ? F.a : (k == 1 ? F.b : F.c);
                if (vk != fv && fw - bc[k] <= kFeatureTie) g_band++;
            }
            q->fa = vx[fv].fa;
            q->fb = vx[fv].fb;
            /* The closest face's outward normal of A - B is the direction
             * that separates B from A: the A -> B contact normal of every
             * other class.  (Collision.metal:2680 writes its negation.) */
            q->normal = F.n;
            q->sep = -bd;
            q->status = MR_STEP_SUCCESS;
            q->path = 3u;
            return vfinite(q->pa) && vfinite(q->pb) && vfinite(q->normal) && isfinite(q->sep);
        }
        if (nv >= EPA_VERTS) return 0;
        const int nvx = nv++;
        vx[nvx] = cand;
        int ne = 0;
        for (int f = 0; f < nf; ++f) {
            if (!fc[f].active || vdot(fc[f].n, vsub(cand.w, vx[fc[f].a].w)) <= tol) continue;
            shorizon(ea, eb, &ne, fc[f].a, fc[f].b);
            shorizon(ea, eb, &ne, fc[f].b, fc[f].c);
            shorizon(ea, eb, &ne, fc[f].c, fc[f].a);
            fc[f].active = 0;
        }
        if (ne == 0) return 0;
        for (int e = 0; e < ne; ++e) {
            int dst = -1;
            for (int f = 0; f < nf; ++f)
                if (!fc[f].active) { dst = f; break; }
            if (dst < 0) {
                if (nf >= EPA_FACES) return 0;
                dst = nf++;
            }
            if (!sface(vx, ea[e], eb[e], nvx, inside, &fc[dst])) fc[dst].active = 0;
        }
    }
    return 0;
}

/* MPR fallback (Collision.metal:2786-3193): portal discovery from the
 * centres' difference, then portal refinement; the witness is the portal
 * triangle's point nearest the origin, taken along that direction and
 * never reported as separation (the fallback runs only after an overlap or
 * a GJK that did not converge). */
static int smpr_witness(const SCol* A, const SCol* B, uint32_t ia, uint32_t ib, const SSup* portal, SQuery* q) {
    double wt[3];
    const v3 closest = sclosest_triangle(portal[1].w, portal[2].w, portal[3].w, wt);
    q->pa = vadd(vadd(vmul(portal[1].pa, wt[0]), vmul(portal[2].pa, wt[1])), vmul(portal[3].pa, wt[2]));
    q->pb = vadd(vadd(vmul(portal[1].pb, wt[0]), vmul(portal[2].pb, wt[1])), vmul(portal[3].pb, wt[2]));
    int fv = 1;
    double fw = wt[0];
    if (wt[1] > fw) { fv = 2; fw = wt[1]; }
    if (wt[2] > fw) { fv = 3; fw = wt[2]; }
    for (int k = 0; k < 3; ++k)
        if (k + 1 != fv && fw - wt[k] <= kFeatureTie) g_band++;
    q->fa = portal[fv].fa;
    q->fb = portal[fv].fb;
    v3 d = closest;
    double dist = vlen(d);
    const v3 centres = vsub(B->c, A->c);
    if (!(dist > kSceneTiny)) { d = centres; dist = vlen(d); }
    d = !(dist > kSceneTiny) ? sdeterministic(ia * 65537u + ib) : vmul(d, 1.0 / dist);
    if (vdot(d, centres) < 0.0) d = vmul(d, -1.0);
    double sep = vdot(vsub(q->pb, q->pa), d);
    if (sep > 0.0) { d = vmul(d, -1.0); sep = -sep; }
    q->status = MR_STEP_SUCCESS;
    q->path = 1u;
    q->normal = d;
    q->sep = fmin(sep, -0.0);
    return vfinite(q->pa) && vfinite(q->pb) && vfinite(q->normal) && isfinite(q->sep);
}

static int smpr(const SCol* A, const SCol* B, uint32_t ia, uint32_t ib, double scale, SQuery* q) {
    SSup portal[4];
    memset(portal, 0, sizeof(portal));
    portal[0].pa = A->c;
    portal[0].pb = B->c;
    portal[0].w = vsub(A->c, B->c);
    const double tol = 64.0 * kFloatEps * scale;
    if (vdot(portal[0].w, portal[0].w) <= tol * tol) portal[0].w = vadd(portal[0].w, vmul(sdeterministic(ia * 65537u + ib), tol));
    v3 d = vmul(portal[0].w, -1.0);
    d = vmul(d, 1.0 / vlen(d));
    sminkowski(A, B, ia, ib, d, &portal[1]);
    if (vdot(portal[1].w, d) < -tol) return 0;
    d = vcross(portal[0].w, portal[1].w);
    double dd = vdot(d, d);
    if (!(dd > tol * tol)) { portal[2] = portal[3] = portal[1]; return smpr_witness(A, B, ia, ib, portal, q); }
    d = vmul(d, 1.0 / sqrt(dd));
    sminkowski(A, B, ia, ib, d, &portal[2]);
    if (vdot(portal[2].w, d) < -tol) return 0;
    d = vcross(vsub(portal[1].w, portal[0].w), vsub(portal[2].w, portal[0].w));
    dd = vdot(d, d);
    if (!(dd > tol * tol)) { portal[3] = portal[2]; return smpr_witness(A, B, ia, ib, portal, q); }
    d = vmul(d, 1.0 / sqrt(dd));
    if (vdot(d, portal[0].w) > 0.0) {
        const SSup t = portal[1];
        portal[1] = portal[2];
        portal[2] = t;
        d = vmul(d, -1.0);
    }
    int found = 0;
    for (int it = 0; it < GJK_ITERS; ++it) {
        sminkowski(A, B, ia, ib, d, &portal[3]);
        if (vdot(portal[3].w, d) < -tol) return 0;
        if (vdot(vcross(portal[1].w, portal[3].w), portal[0].w) < -tol) {
            portal[2] = portal[3];
        } else if (vdot(vcross(portal[3].w, portal[2].w), portal[0].w) < -tol) {
            portal[1] = portal[3];
        } else {
            found = 1;
            break;
        }
        d = vcross(vsub(portal[1].w, portal[0].w), vsub(portal[2].w, portal[0].w));
        dd = vdot(d, d);
        if (!(dd > tol * tol)) { portal[3] = portal[2]; return smpr_witness(A, B, ia, ib, portal, q); }
        d = vmul(d, 1.0 / sqrt(dd));
    }
    if (!found) return 0;
    for (int it = 0; it < EPA_ITERS; ++it) {
        d = vcross(vsub(portal[2].w, portal[1].w), vsub(portal[3].w, portal[1].w));
        dd = vdot(d, d);
        if (!(dd > kSceneTiny) || !isfinite(dd)) return smpr_witness(A, B, ia, ib, portal, q);
        d = vmul(d, 1.0 / sqrt(dd));
        SSup cand;
        sminkowski(A, B, ia, ib, d, &cand);
        const double cp = vdot(cand.w, d);
        const double pp = fmin(vdot(portal[1].w, d), fmin(vdot(portal[2].w, d), vdot(portal[3].w, d)));
        if (cp - pp <= tol || it + 1 == EPA_ITERS) return smpr_witness(A, B, ia, ib, portal, q);
        const v3 cc = vcross(cand.w, portal[0].w);
        if (vdot(portal[1].w, cc) > 0.0) {
            if (vdot(portal[2].w, cc) > 0.0) portal[1] = cand;
            else portal[3] = cand;
        } else if (vdot(portal[3].w, cc) > 0.0) {
            portal[2] = cand;
        } else {
            portal[1] = cand;
        }
    }
    return 0;
}

static void spatch_add(SRaw* raw, v3 pa, v3 pb, double sep, uint32_t fa, uint32_t fb, double tol2) {
    for (int i = 0; i < raw->n; ++i) {
        const v3 da = vsub(raw->pa[i], pa), db = vsub(raw->pb[i], pb);
        if (vdot(da, da) <= tol2 && vdot(db, db) <= tol2) return;
    }
    sraw_add(raw, pa, pb, sep, fa, fb);
}

/* Extra points of a cylinder's or hull's contact patch
 * (Collision.metal:3327-3432): supports of the sampled shape -- a cylinder,
 * else a hull, A first -- along the query normal tilted by 2e-4 towards the
 * disk basis (cylinder cap contact), the axis (cylinder side contact) or
 * the contact plane's tangents (hull). */
static void spatch(const SCol* A, const SCol* B, uint32_t ia, uint32_t ib, double scale, const SQuery* q, SRaw* raw) {
    const int cyl_a = A->type == MR_SHAPE_CYLINDER, cyl_b = B->type == MR_SHAPE_CYLINDER;
    const int hull = A->type == MR_SHAPE_CONVEX || B->type == MR_SHAPE_CONVEX;
    if (!cyl_a && !cyl_b && !hull) return;
    const double dtol = 32.0 * kFloatEps * scale;
    const int sample_a = cyl_a || (!cyl_b && A->type == MR_SHAPE_CONVEX);
    const SCol* k = sample_a ? A : B;
    const uint32_t kidx = sample_a ? ia : ib;
    const v3 sn = sample_a ? q->normal : vmul(q->normal, -1.0);
    v3 dirs[4];
    int nd = 0;
    if (k->type == MR_SHAPE_CYLINDER) {
        const double align = fabs(vdot(sn, k->axis));
        BAND(align, 0.95);
        BAND(align, 0.20);
        if (align >= 0.95) {
            dirs[0] = k->bx; dirs[1] = vmul(k->bx, -1.0); dirs[2] = k->bz; dirs[3] = vmul(k->bz, -1.0);
            nd = 4;
        } else if (align <= 0.20) {
            dirs[0] = k->axis; dirs[1] = vmul(k->axis, -1.0);
            nd = 2;
        }
    } else {
        /* contactPatchTangent: the normal crossed with the world axis of
         * its smallest absolute component. */
        const v3 n = q->normal;
        const double ax = fabs(n.x), ay = fabs(n.y), az = fabs(n.z);
        const v3 ref = ax <= ay && ax <= az ? V(1, 0, 0) : (ay <= az ? V(0, 1, 0) : V(0, 0, 1));
        v3 t = vcross(n, ref);
        t = vmul(t, 1.0 / vlen(t));
        const v3 bt = vcross(n, t);
        dirs[0] = t; dirs[1] = vmul(t, -1.0); dirs[2] = bt; dirs[3] = vmul(bt, -1.0);
        nd = 4;
    }
    for (int i = 0; i < nd; ++i) {
        uint32_t f;
        const v3 p = ssupport(k, kidx, vadd(sn, vmul(dirs[i], 2.0e-4)), &f);
        const v3 pa = sample_a ? p : vsub(p, vmul(q->normal, q->sep));
        const v3 pb = sample_a ? vadd(p, vmul(q->normal, q->sep)) : p;
        spatch_add(raw, pa, pb, q->sep, sample_a ? f : q->fa, sample_a ? q->fb : f, dtol * dtol);
    }
}

/* Penetration witness of the hull path (Collision.metal:3129-3260): among
 * the centre-to-centre direction and the three local axes of each collider,
 * oriented from A towards B, the axis of largest separation
 * dot(support_B(-axis) - support_A(axis), axis).  No previous-substep query
 * direction is tried (no query cache is kept). */
static int ssupport_axis_witness(const SCol* A, const SCol* B, uint32_t ia, uint32_t ib, SQuery* q) {
    const v3 delta = vsub(B->c, A->c);
    v3 axes[7];
    axes[0] = delta;
    for (int a = 0; a < 3; ++a) {
        const v3 e = V(a == 0, a == 1, a == 2);
        axes[1 + 2 * a] = qrot(A->r, e);
        axes[2 + 2 * a] = qrot(B->r, e);
    }
    int found = 0;
    double second = -INFINITY;
    for (int i = 0; i < 7; ++i) {
        v3 axis = axes[i];
        const double a2 = vdot(axis, axis);
        if (!(a2 > kSceneTiny) || !isfinite(a2)) continue;
        axis = vmul(axis, 1.0 / sqrt(a2));
        if (vdot(delta, delta) > kSceneTiny && vdot(axis, delta) < 0.0) axis = vmul(axis, -1.0);
        uint32_t fa, fb;
        const v3 pa = ssupport(A, ia, axis, &fa);
        const v3 pb = ssupport(B, ib, vmul(axis, -1.0), &fb);
        const double sep = vdot(vsub(pb, pa), axis);
        if (!isfinite(sep)) return 0;
        if (!found || sep > q->sep) {
            if (found) second = q->sep;
            found = 1;
            q->normal = axis;
            q->sep = sep;
            q->pa = pa;
            q->pb = pb;
            q->fa = fa;
            q->fb = fb;
        } else if (sep > second) {
            second = sep;
        }
    }
    if (!found) return 0;
    if (isfinite(second)) BAND(q->sep - second, 0.0);
    q->sep = fmin(q->sep, -0.0);
    q->status = MR_STEP_SUCCESS;
    q->path = 2;
    return vfinite(q->pa) && vfinite(q->pb) && vfinite(q->normal) && isfinite(q->sep);
}

/* Contacts of a support-mapped pair; the pair's normal (A -> B).  Cylinder
 * pairs resolve an overlap by EPA, then MPR; pairs with a hull by the
 * support-axis witness (Collision.metal:3623-3720), a hull on the plane by
 * its deepest vertex. */
static v3 ssupport_mapped(const SCol* A, const SCol* B, uint32_t ia, uint32_t ib, double acc, SRaw* raw) {
    if (B->type == MR_SHAPE_PLANE) {
        uint32_t f;
        const v3 p = ssupport(A, ia, vmul(B->normal, -1.0), &f);
        const double sep = vdot(B->normal, vsub(p, B->c));
        BAND(sep, acc);
        if (sep <= acc) sraw_add(raw, p, vsub(p, vmul(B->normal, sep)), sep, f, feature_key(MR_SHAPE_PLANE, 0u));
        return vmul(B->normal, -1.0);
    }
    const int hull = A->type == MR_SHAPE_CONVEX || B->type == MR_SHAPE_CONVEX;
    const double scale = fmax(scol_scale(A), scol_scale(B)) + 1.0;
    SSup sx[4];
    double wt[4] = {0, 0, 0, 0};
    int n = 0;
    SQuery q;
    memset(&q, 0, sizeof(q));
    q.normal = V(0, 0, 1);
    const int overlap = sgjk(A, B, ia, ib, scale, sx, &n, wt, &q);
    if (q.status != MR_STEP_SUCCESS && q.status != MR_STEP_DID_NOT_CONVERGE) { raw->status = q.status; return q.normal; }
    if (hull) {
        if ((overlap || q.status == MR_STEP_DID_NOT_CONVERGE) && !ssupport_axis_witness(A, B, ia, ib, &q)) {
            raw->status = MR_STEP_DID_NOT_CONVERGE;
            return q.normal;
        }
    } else if (overlap) {
        /* Primitive pairs resolve with EPA first, MPR second (Collision.metal:3518-3560). */
        if (!sepa(A, B, ia, ib, scale, sx, n, &q) && !smpr(A, B, ia, ib, scale, &q)) {
            raw->status = MR_STEP_DID_NOT_CONVERGE;
            return q.normal;
        }
    } else if (q.status == MR_STEP_DID_NOT_CONVERGE) {
        if (!smpr(A, B, ia, ib, scale, &q)) { raw->status = MR_STEP_DID_NOT_CONVERGE; return q.normal; }
    }
    raw->path = q.path;
    BAND(q.sep, acc);
    if (q.sep <= acc) {
        sraw_add(raw, q.pa, q.pb, q.sep, q.fa, q.fb);
        spatch(A, B, ia, ib, scale, &q, raw);
    }
    return q.normal;
}

/* Cylinder on the plane (Collision.metal:4627-4800, Collision.cpp:2240-2390):
 * a cap face parallel to the plane gives its four-point ring plus the exact
 * rim support, a side parallel to it the two rim ends, any other pose the
 * one extremal rim point. */
static void scylinder_plane(const SCol* A, const SCol* P, double acc, SRaw* raw) {
    const v3 pn = P->normal;
    const uint32_t plane_key = feature_key(MR_SHAPE_PLANE, 0);
    const double axial = vdot(pn, A->axis), rx = vdot(pn, A->bx), rz = vdot(pn, A->bz);
    const v3 rproj = vadd(vmul(A->bx, rx), vmul(A->bz, rz));
    const double rsq = fmax(0.0, rx * rx + rz * rz);
    BAND(rsq, kCylAlign * kCylAlign);
    if (rsq <= kCylAlign * kCylAlign) {
        const int pos = axial < 0.0;
        const v3 cap = vadd(A->c, vmul(A->axis, pos ? A->hl : -A->hl));
        const uint32_t base = pos ? kCylPosRing : kCylNegRing;
        const v3 dirs[4] = {A->bx, vmul(A->bx, -1.0), A->bz, vmul(A->bz, -1.0)};
        for (int i = 0; i < 4; ++i) {
            const v3 surface = vadd(cap, vmul(dirs[i], A->radius));
            const double sep = vdot(pn, vsub(surface, P->c));
            BAND(sep, acc);
            if (sep <= acc) sraw_add(raw, surface, vsub(surface, vmul(pn, sep)), sep, feature_key(MR_SHAPE_CYLINDER, base + (uint32_t)i), plane_key);
        }
        if (rsq > 0.0) {
            const v3 surface = vadd(cap, vmul(rproj, -A->radius / sqrt(rsq)));
            const double sep = vdot(pn, vsub(surface, P->c));
            BAND(sep, acc);
            if (sep <= acc)
                sraw_add(raw, surface, vsub(surface, vmul(pn, sep)), sep, feature_key(MR_SHAPE_CYLINDER, pos ? kCylPosRim : kCylNegRim),
                         plane_key);
        }
        return;
    }
    const v3 rdir = vmul(rproj, -1.0 / sqrt(rsq));
    BAND(fabs(axial), kCylAlign);
    if (fabs(axial) <= kCylAlign) {
        for (int i = 0; i < 2; ++i) {
            const v3 surface = vadd(vadd(A->c, vmul(A->axis, i ? A->hl : -A->hl)), vmul(rdir, A->radius));
            const double sep = vdot(pn, vsub(surface, P->c));
            BAND(sep, acc);
            if (sep <= acc)
                sraw_add(raw, surface, vsub(surface, vmul(pn, sep)), sep, feature_key(MR_SHAPE_CYLINDER, i ? kCylPosSide : kCylNegSide),
                         plane_key);
        }
        return;
    }
    const int pos = axial < 0.0;
    const v3 surface = vadd(vadd(A->c, vmul(A->axis, pos ? A->hl : -A->hl)), vmul(rdir, A->radius));
    const double sep = vdot(pn, vsub(surface, P->c));
    BAND(sep, acc);
    if (sep <= acc)
        sraw_add(raw, surface, vsub(surface, vmul(pn, sep)), sep, feature_key(MR_SHAPE_CYLINDER, pos ? kCylPosRim : kCylNegRim), plane_key);
}

static v3 snarrow(const SCol* A, const SCol* B, int cls, uint32_t ia, uint32_t ib, double acc, SRaw* raw) {
    raw->n = 0;
    raw->status = 0;
    raw->path = 0;
    if (cls == MR_COLLISION_PAIR_CONVEX) return ssupport_mapped(A, B, ia, ib, acc, raw);
    if (cls == MR_COLLISION_PAIR_SPHERE_SPHERE) {
        const v3 d = vsub(B->c, A->c);
        const double len = vlen(d);
        const v3 n = len > kSceneTiny ? vmul(d, 1.0 / len) : scoincident(ia, ib);
        const double sep = len - A->radius - B->radius;
        BAND(sep, acc);
        if (sep <= acc) sraw_add(raw, vadd(A->c, vmul(n, A->radius)), vsub(B->c, vmul(n, B->radius)), sep,
                                 feature_key(MR_SHAPE_SPHERE, 0), feature_key(MR_SHAPE_SPHERE, 0));
        return n;
    }
    if (cls == MR_COLLISION_PAIR_SPHERE_BOX) {
        const int sphere_a = A->type == MR_SHAPE_SPHERE;
        const SCol* sp = sphere_a ? A : B;
        const SCol* bx = sphere_a ? B : A;
        const v3 lc = qrotinv(bx->r, vsub(sp->c, bx->c));
        v3 cl = V(fmin(fmax(lc.x, -bx->half.x), bx->half.x), fmin(fmax(lc.y, -bx->half.y), bx->half.y),
                  fmin(fmax(lc.z, -bx->half.z), bx->half.z));
        BAND(fabs(lc.x), bx->half.x);
        BAND(fabs(lc.y), bx->half.y);
        BAND(fabs(lc.z), bx->half.z);
        const v3 ld = vsub(cl, lc);
        const double dist = vlen(ld);
        v3 n;
        double sep;
        uint32_t feat;
        if (dist > kSceneTiny) {
            n = qrot(bx->r, vmul(ld, 1.0 / dist));
            sep = dist - sp->radius;
#define SREG(c, he) ((c) < -(he) ? 0u : ((c) > (he) ? 2u : 1u))
            feat = SREG(lc.x, bx->half.x) + 3u * SREG(lc.y, bx->half.y) + 9u * SREG(lc.z, bx->half.z);
#undef SREG
        } else {
            const double dx = bx->half.x - fabs(lc.x), dy = bx->half.y - fabs(lc.y), dz = bx->half.z - fabs(lc.z);
            int axis = 0;
            double dm = dx;
            if (dy < dm) { axis = 1; dm = dy; }
            if (dz < dm) { axis = 2; dm = dz; }
            const double coord = axis == 0 ? lc.x : (axis == 1 ? lc.y : lc.z);
            const double sign = coord >= 0.0 ? 1.0 : -1.0;
            const v3 outward = V(axis == 0 ? sign : 0.0, axis == 1 ? sign : 0.0, axis == 2 ? sign : 0.0);
            if (axis == 0) cl.x = sign * bx->half.x;
            else if (axis == 1) cl.y = sign * bx->half.y;
            else cl.z = sign * bx->half.z;
            n = qrot(bx->r, vmul(outward, -1.0));
            sep = -dm - sp->radius;
            feat = 27u + 2u * (uint32_t)axis + (sign > 0.0 ? 1u : 0u);
        }
        const v3 box_point = vadd(bx->c, qrot(bx->r, cl));
        BAND(sep, acc);
        if (sep <= acc) {
            const v3 sphere_point = vadd(sp->c, vmul(n, sp->radius));
            if (sphere_a) sraw_add(raw, sphere_point, box_point, sep, feature_key(MR_SHAPE_SPHERE, 0), feature_key(MR_SHAPE_BOX, feat));
            else sraw_add(raw, box_point, sphere_point, sep, feature_key(MR_SHAPE_BOX, feat), feature_key(MR_SHAPE_SPHERE, 0));
        }
        return sphere_a ? n : vmul(n, -1.0);
    }
    if (cls == MR_COLLISION_PAIR_SPHERE_CAPSULE) {
        const int sphere_a = A->type == MR_SHAPE_SPHERE;
        const SCol* sp = sphere_a ? A : B;
        const SCol* cp = sphere_a ? B : A;
        double t;
        const v3 on = sclosest_on_segment(sp->c, cp->e0, cp->e1, &t);
        const v3 delta = vsub(on, sp->c);
        const double d = vlen(delta);
        const v3 n = d > kSceneTiny ? vmul(delta, 1.0 / d)
                                    : sstable_segment_normal(vsub(cp->e1, cp->e0), V(0, 0, 0), sphere_a ? ia : ib, sphere_a ? ib : ia);
        const double sep = d - sp->radius - cp->radius;
        BAND(sep, acc);
        if (sep <= acc) {
            const v3 ps = vadd(sp->c, vmul(n, sp->radius)), pc = vsub(on, vmul(n, cp->radius));
            const uint32_t fs = feature_key(MR_SHAPE_SPHERE, 0), fc = feature_key(MR_SHAPE_CAPSULE, scap_feature(t));
            if (sphere_a) sraw_add(raw, ps, pc, sep, fs, fc);
            else sraw_add(raw, pc, ps, sep, fc, fs);
        }
        return sphere_a ? n : vmul(n, -1.0);
    }
    if (cls == MR_COLLISION_PAIR_CAPSULE_CAPSULE) {
        v3 pa, pb;
        double ta, tb;
        sclosest_segments(A->e0, A->e1, B->e0, B->e1, &pa, &pb, &ta, &tb);
        const v3 delta = vsub(pb, pa);
        const double d = vlen(delta);
        const v3 n = d > kSceneTiny ? vmul(delta, 1.0 / d) : sstable_segment_normal(vsub(A->e1, A->e0), vsub(B->e1, B->e0), ia, ib);
        const double sep = d - A->radius - B->radius;
        BAND(sep, acc);
        if (sep <= acc)
            sraw_add(raw, vadd(pa, vmul(n, A->radius)), vsub(pb, vmul(n, B->radius)), sep,
                     feature_key(MR_SHAPE_CAPSULE, scap_feature(ta)), feature_key(MR_SHAPE_CAPSULE, scap_feature(tb)));
        return n;
    }
    if (cls == MR_COLLISION_PAIR_CAPSULE_BOX) {
        const int capsule_a = A->type == MR_SHAPE_CAPSULE;
        const SCol* cp = capsule_a ? A : B;
        const SCol* bx = capsule_a ? B : A;
        const SCapBox w = scapsule_box(cp, bx, capsule_a ? ia : ib, capsule_a ? ib : ia);
        BAND(w.sep, acc);
        if (w.sep <= acc) {
            const uint32_t fc = feature_key(MR_SHAPE_CAPSULE, scap_feature(w.t_cap)), fb = feature_key(MR_SHAPE_BOX, w.box_feature);
            if (capsule_a) sraw_add(raw, w.cap_point, w.box_point, w.sep, fc, fb);
            else sraw_add(raw, w.box_point, w.cap_point, w.sep, fb, fc);
        }
        return capsule_a ? w.normal : vmul(w.normal, -1.0);
    }
    if (cls == MR_COLLISION_PAIR_BOX_BOX) {
        const v3 cd = vsub(B->c, A->c);
        double best_sep = -INFINITY;
        v3 best_n = scoincident(ia, ib);
        int best_axis = 0;
        double best_err = 0.0;
        const double reach = vlen(A->half) + vlen(B->half);
        int index = -1; /* position in the list of accepted axes (Collision.cpp:1818-1842) */
        for (int k = 0; k < 15; ++k) {
            v3 axis;
            double axis_len = 1.0;
            if (k < 3) axis = sbox_axis(A, k);
            else if (k < 6) axis = sbox_axis(B, k - 3);
            else {
                const v3 cr = vcross(sbox_axis(A, (k - 6) / 3), sbox_axis(B, (k - 6) % 3));
                const double sq = vdot(cr, cr);
                /* Edge pairs within |sin| = 1e-6 of parallel give no axis
                 * (Collision.metal:1600-1612); near the floor the FP32 cross
                 * product may fall on the other side. */
                if (fabs(sq - 1e-12) <= 16.0 * kFloatEps * (sq + 1e-12) + 1e-13) g_band++;
                if (!(sq > 1e-12)) continue;
                axis_len = sqrt(sq);
                axis = vmul(cr, 1.0 / axis_len);
            }
            ++index;
            const double proj = vdot(cd, axis);
            if (proj < 0.0 || (proj == 0.0 && vdot(axis, best_n) < 0.0)) axis = vmul(axis, -1.0);
            const double sep = fabs(proj) - sbox_radius(A, axis) - sbox_radius(B, axis);
            /* FP32 sensitivity of this axis' separation: an edge-edge axis
             * carries the rounding of its cross product amplified by 1/|cross|. */
            const double err = 8.0 * kFloatEps * (vlen(cd) + reach) / axis_len;
            if (fabs(sep - acc) <= err) g_band++;
            BAND(sep, acc);
            if (sep > acc) return axis;
            const double tol = 1.0e-7 * (1.0 + fmax(fabs(best_sep), fabs(sep))); /* Collision.metal:1628-1638 */
            if (isfinite(best_sep) && fabs(sep - best_sep) <= err + best_err) g_band++;
            if (!isfinite(best_sep) || sep > best_sep + tol || (fabs(sep - best_sep) <= tol && index < best_axis)) {
                best_sep = sep;
                best_n = axis;
                best_axis = index;
                best_err = err;
            }
        }
        const double near_b = vdot(B->c, best_n) - sbox_radius(B, best_n);
        const double far_a = vdot(A->c, best_n) + sbox_radius(A, best_n);
        for (int v = 0; v < 8; ++v) {
            const v3 pa = sbox_vertex(A, v);
            if (!sinside(pa, B, acc)) continue;
            const double sep = near_b - vdot(pa, best_n);
            BAND(sep, acc);
            if (sep <= acc)
                sraw_add(raw, pa, vadd(pa, vmul(best_n, sep)), sep, feature_key(MR_SHAPE_BOX, (uint32_t)v),
                         feature_key(MR_SHAPE_BOX, 128u + (uint32_t)best_axis));
        }
        for (int v = 0; v < 8; ++v) {
            const v3 pb = sbox_vertex(B, v);
            if (!sinside(pb, A, acc)) continue;
            const double sep = vdot(pb, best_n) - far_a;
            BAND(sep, acc);
            if (sep <= acc)
                sraw_add(raw, vsub(pb, vmul(best_n, sep)), pb, sep, feature_key(MR_SHAPE_BOX, 128u + (uint32_t)best_axis),
                         feature_key(MR_SHAPE_BOX, (uint32_t)v));
        }
        if (raw->n == 0) {
            const v3 pa = sbox_support(A, best_n), pb = sbox_support(B, vmul(best_n, -1.0));
            sraw_add(raw, pa, pb, vdot(vsub(pb, pa), best_n), feature_key(MR_SHAPE_BOX, 256u + (uint32_t)best_axis),
                     feature_key(MR_SHAPE_BOX, 256u + (uint32_t)best_axis));
        }
        return best_n;
    }
    {
        const v3 pn = B->normal;
        const uint32_t plane_key = feature_key(MR_SHAPE_PLANE, 0);
        if (cls == MR_COLLISION_PAIR_SPHERE_PLANE) {
            const v3 surface = vsub(A->c, vmul(pn, A->radius));
            const double sep = vdot(pn, vsub(surface, B->c));
            BAND(sep, acc);
            if (sep <= acc) sraw_add(raw, surface, vsub(surface, vmul(pn, sep)), sep, feature_key(MR_SHAPE_SPHERE, 0), plane_key);
        } else if (cls == MR_COLLISION_PAIR_CAPSULE_PLANE) {
            for (int e = 0; e < 2; ++e) {
                const v3 surface = vsub(e == 0 ? A->e0 : A->e1, vmul(pn, A->radius));
                const double sep = vdot(pn, vsub(surface, B->c));
                BAND(sep, acc);
                if (sep <= acc)
                    sraw_add(raw, surface, vsub(surface, vmul(pn, sep)), sep, feature_key(MR_SHAPE_CAPSULE, (uint32_t)e), plane_key);
            }
        } else if (cls == MR_COLLISION_PAIR_CYLINDER_PLANE) {
            scylinder_plane(A, B, acc, raw);
        } else if (cls == MR_COLLISION_PAIR_BOX_PLANE) {
            for (int v = 0; v < 8; ++v) {
                const v3 w = sbox_vertex(A, v);
                const double sep = vdot(pn, vsub(w, B->c));
                BAND(sep, acc);
                if (sep <= acc) sraw_add(raw, w, vsub(w, vmul(pn, sep)), sep, feature_key(MR_SHAPE_BOX, (uint32_t)v), plane_key);
            }
        }
        return vmul(pn, -1.0);
    }
}

typedef struct {
    double la[3], lb[3];
    uint32_t fa, fb, life;
    double imp[3];
    v3 wp;
    double sep;
} SCand;

static unsigned long long sckey(const SCand* c) { return ((unsigned long long)c->fa << 32) | c->fb; }

/* Persistent manifold of one pair (same decisions as the device builder). */
static int sbuild(const OracleScene* s, const OracleManifold* old, const SRaw* raw, v3 raw_normal, OracleManifold* out, v3 posA,
                  q4 rotA, v3 posB, q4 rotB) {
    memset(out, 0, sizeof(*out));
    if (raw->n == 0) return 0;
    for (int i = 0; i < raw->n; ++i)
        if (!isfinite(raw->sep[i]) || !vfinite(raw->pa[i]) || !vfinite(raw->pb[i])) return -1;
    const v3 nw = vmul(raw_normal, 1.0 / vlen(raw_normal));
    if (!vfinite(nw)) return -1;
    SCand c[12];
    int nc = 0, old_ok = 0;
    v3 transported = V(0, 0, 0);
    double old_age = 0.0;
    const int old_count = old ? (int)old->count : 0;
    if (old_count > 0 && old_count <= 4) {
        v3 on = qrot(rotA, vld(old->normal_local));
        on = vmul(on, 1.0 / vlen(on));
        BAND(vdot(on, nw), s->thr[3]);
        old_ok = vfinite(on) && vdot(on, nw) >= s->thr[3];
        if (old_ok) {
            const v3 ot = qrot(rotA, vld(old->tangent_local));
            transported = vsub(ot, vmul(nw, vdot(ot, nw)));
            old_age = old->age;
            for (int i = 0; i < old_count; ++i) {
                const OraclePoint* op = &old->points[i];
                const v3 pa = vadd(posA, qrot(rotA, vld(op->anchor_a)));
                const v3 pb = vadd(posB, qrot(rotB, vld(op->anchor_b)));
                const v3 d = vsub(pb, pa);
                const double sep = vdot(d, nw);
                const double drift = vlen(vsub(d, vmul(nw, sep)));
                BAND(sep, s->thr[0]);
                BAND(drift, s->thr[1]);
                if (sep > s->thr[0] || drift > s->thr[1]) continue;
                SCand* k = &c[nc++];
                for (int a = 0; a < 3; ++a) { k->la[a] = op->anchor_a[a]; k->lb[a] = op->anchor_b[a]; k->imp[a] = op->impulses[a]; }
                k->fa = op->feature_a;
                k->fb = op->feature_b;
                k->life = op->life == 0xffffffffu ? 0xffffffffu : op->life + 1u;
                k->wp = vmul(vadd(pa, pb), 0.5);
                k->sep = sep;
            }
        }
    }
    const double merge2 = s->thr[2] * s->thr[2];
    for (int r = 0; r < raw->n; ++r) {
        const v3 la = qrotinv(rotA, vsub(raw->pa[r], posA));
        const v3 lb = qrotinv(rotB, vsub(raw->pb[r], posB));
        int match = -1;
        for (int k = 0; k < nc && match < 0; ++k)
            if (c[k].fa == raw->fa[r] && c[k].fb == raw->fb[r]) match = k;
        for (int k = 0; k < nc && match < 0; ++k) {
            const v3 da = vsub(vld(c[k].la), la), db = vsub(vld(c[k].lb), lb);
            BAND(sqrt(vdot(da, da) + vdot(db, db)), sqrt(2.0 * merge2));
            if (vdot(da, da) + vdot(db, db) <= 2.0 * merge2) match = k;
        }
        if (match < 0) {
            if (nc >= 12) return -1;
            match = nc++;
            c[match].life = 0u;
            c[match].imp[0] = c[match].imp[1] = c[match].imp[2] = 0.0;
        }
        vst(c[match].la, la);
        vst(c[match].lb, lb);
        c[match].fa = raw->fa[r];
        c[match].fb = raw->fb[r];
        c[match].wp = vmul(vadd(raw->pa[r], raw->pb[r]), 0.5);
        c[match].sep = raw->sep[r];
    }
    if (nc > 4) {
        for (int i = 1; i < nc; ++i) {
            SCand val = c[i];
            int d = i;
            while (d > 0 && (val.sep < c[d - 1].sep || (val.sep == c[d - 1].sep && sckey(&val) < sckey(&c[d - 1])))) {
                c[d] = c[d - 1];
                --d;
            }
            c[d] = val;
        }
        if (fabs(c[1].sep - c[0].sep) <= g_band_width) g_band++;
        int selected[12] = {0}, chosen[4], count = 1;
        chosen[0] = 0;
        selected[0] = 1;
        for (int stage = 1; stage < 4; ++stage) {
            int best = -1;
            double best_score = -1.0;
            unsigned long long best_f = ~0ull;
            for (int i = 0; i < nc; ++i) {
                if (selected[i]) continue;
                double score;
                if (stage == 1) {
                    const v3 d = vsub(c[i].wp, c[chosen[0]].wp);
                    const v3 t = vsub(d, vmul(nw, vdot(d, nw)));
                    score = vdot(t, t);
                } else if (stage == 2) {
                    score = fabs(vdot(vcross(vsub(c[chosen[1]].wp, c[chosen[0]].wp), vsub(c[i].wp, c[chosen[0]].wp)), nw));
                } else {
                    score = INFINITY;
                    for (int k = 0; k < count; ++k) {
                        const v3 d = vsub(c[i].wp, c[chosen[k]].wp);
                        const v3 t = vsub(d, vmul(nw, vdot(d, nw)));
                        score = fmin(score, vdot(t, t));
                    }
                }
                const unsigned long long f = sckey(&c[i]);
                const double tol = fmax(1.0e-12, kTieRelative * fmax(fabs(score), fabs(best_score)));
                if (best >= 0 && fabs(fabs(score - best_score) - tol) <= 0.1 * tol) g_band++;
                if (score > best_score + tol || (fabs(score - best_score) <= tol && f < best_f)) {
                    best = i;
                    best_score = score;
                    best_f = f;
                }
            }
            if (best >= 0) { chosen[count++] = best; selected[best] = 1; }
        }
        SCand red[4];
        for (int i = 0; i < count; ++i) red[i] = c[chosen[i]];
        nc = count;
        for (int i = 0; i < nc; ++i) c[i] = red[i];
    }
    for (int i = 1; i < nc; ++i) {
        SCand val = c[i];
        int d = i;
        while (d > 0 && sckey(&val) < sckey(&c[d - 1])) { c[d] = c[d - 1]; --d; }
        c[d] = val;
    }
    v3 tw = transported;
    if (!old_ok || !vfinite(tw) || vdot(tw, tw) <= 1.0e-12) tw = stable_tangent(nw);
    else tw = vmul(tw, 1.0 / vlen(tw));
    vst(out->normal_local, qrotinv(rotA, nw));
    out->age = old_ok ? fmin(old_age + 1.0, 65535.0) : 0.0;
    vst(out->tangent_local, qrotinv(rotA, tw));
    out->count = (uint32_t)nc;
    for (int i = 0; i < nc; ++i) {
        OraclePoint* op = &out->points[i];
        for (int a = 0; a < 3; ++a) { op->anchor_a[a] = c[i].la[a]; op->anchor_b[a] = c[i].lb[a]; op->impulses[a] = c[i].imp[a]; }
        op->feature_a = c[i].fa;
        op->feature_b = c[i].fb;
        op->life = c[i].life;
    }
    return nc;
}

static void sym3_world(q4 q, const double* inv, double* out) {
    const v3 c0 = qrot(q, V(1, 0, 0)), c1 = qrot(q, V(0, 1, 0)), c2 = qrot(q, V(0, 0, 1));
    const double R[3][3] = {{c0.x, c1.x, c2.x}, {c0.y, c1.y, c2.y}, {c0.z, c1.z, c2.z}};
    int k = 0;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j <= i; ++j) {
            double acc = 0.0;
            for (int m = 0; m < 3; ++m) acc += R[i][m] * inv[m] * R[j][m];
            out[k++] = acc;
        }
}
static v3 sym3_apply(const double* S, v3 x) {
    return V(S[0] * x.x + S[1] * x.y + S[3] * x.z, S[1] * x.x + S[2] * x.y + S[4] * x.z, S[3] * x.x + S[4] * x.y + S[5] * x.z);
}

typedef struct {
    int a, b;  /* b < 0: plane */
    v3 ra, rb, n, t, bt;
    double target[3], reg, mu, lambda[3], P[9], relax, delta[3];
    int slot, point, new_impact;
    double sep, rthr, restitution, mu_d;
} SCon;

static void sprepare(const OracleScene* s, SState* st) {
    const double h = s->h;
    for (uint32_t b = 0; b < s->nb; ++b) {
        st->lin[b] = rn3(vadd(vmul(st->lin[b], exp(-h * s->damp_lin[b])), vmul(V(s->gravity[0], s->gravity[1], s->gravity[2]), h)));
        st->ang[b] = rn3(vmul(st->ang[b], exp(-h * s->damp_ang[b])));
    }
}

static uint32_t sbounds(const OracleScene* s, SState* st, uint32_t* fail_index) {
    const double h = s->h;
    for (uint32_t b = 0; b < s->nb; ++b) {
        q4 qn;
        if (!qnormalize(st->rot[b], &qn, 1)) { *fail_index = b; return MR_STEP_NONFINITE_INPUT; }
        st->rot[b] = qn;
        sym3_world(qn, s->inv_inertia[b], st->iiw[b]);
        const v3 c = st->pos[b];
        const v3 fc = vadd(c, vmul(st->lin[b], h));
        q4 fr = qmul(so3_increment(vmul(st->ang[b], h), 0), qn);
        fr = Q(fr.x / sqrt(qdot(fr, fr)), fr.y / sqrt(qdot(fr, fr)), fr.z / sqrt(qdot(fr, fr)), fr.w / sqrt(qdot(fr, fr)));
        /* Chord of the sweep sphere over the substep's rotation: the
         * reference's 2 r sqrt(1 - cos^2), cos = |q . q_next|, written as
         * 2 r |sin(h |w| / 2)| (the same value; no cancellation near rest). */
        const double chord = 2.0 * s->sweep[b] * fabs(sin(0.5 * h * vlen(st->ang[b])));
        const double env = fmin(vlen(vsub(fc, c)) + chord, h * s->speed_env);
        const double margin = s->spec_scale * env;
        st->margin[b] = margin;
        v3 e0, e1;
        if (s->type[b] == MR_SHAPE_SPHERE) {
            e0 = e1 = V(s->dims[b][0], s->dims[b][0], s->dims[b][0]);
        } else if (s->type[b] == MR_SHAPE_CAPSULE) {
            const double r = s->dims[b][0];
            const v3 a0 = qrot(qn, V(0, s->dims[b][1], 0)), a1 = qrot(fr, V(0, s->dims[b][1], 0));
            e0 = V(fabs(a0.x) + r, fabs(a0.y) + r, fabs(a0.z) + r);
            e1 = V(fabs(a1.x) + r, fabs(a1.y) + r, fabs(a1.z) + r);
        } else if (s->type[b] == MR_SHAPE_CYLINDER) {
            /* Collision.cpp:719-740: per component |a_i| hl + sqrt(1 - a_i^2) r. */
            const double r = s->dims[b][0], hl = s->dims[b][1];
            const q4 rs[2] = {qn, fr};
            v3 ex[2];
            for (int k = 0; k < 2; ++k) {
                const v3 a = qrot(rs[k], V(0, 1, 0));
                ex[k] = V(fabs(a.x) * hl + sqrt(fmax(0.0, 1.0 - a.x * a.x)) * r,
                          fabs(a.y) * hl + sqrt(fmax(0.0, 1.0 - a.y * a.y)) * r,
                          fabs(a.z) * hl + sqrt(fmax(0.0, 1.0 - a.z * a.z)) * r);
            }
            e0 = ex[0];
            e1 = ex[1];
        } else {
            const q4 rs[2] = {qn, fr};
            v3 ex[2];
            for (int k = 0; k < 2; ++k) {
                const v3 bx = qrot(rs[k], V(1, 0, 0)), by = qrot(rs[k], V(0, 1, 0)), bz = qrot(rs[k], V(0, 0, 1));
                ex[k] = vadd(vadd(vmul(V(fabs(bx.x), fabs(bx.y), fabs(bx.z)), s->dims[b][0]),
                                  vmul(V(fabs(by.x), fabs(by.y), fabs(by.z)), s->dims[b][1])),
                             vmul(V(fabs(bz.x), fabs(bz.y), fabs(bz.z)), s->dims[b][2]));
            }
            e0 = ex[0];
            e1 = ex[1];
        }
        const double o = s->offset[b];
        double lo[3] = {fmin(c.x - e0.x, fc.x - e1.x) - o, fmin(c.y - e0.y, fc.y - e1.y) - o, fmin(c.z - e0.z, fc.z - e1.z) - o};
        double hi[3] = {fmax(c.x + e0.x, fc.x + e1.x) + o, fmax(c.y + e0.y, fc.y + e1.y) + o, fmax(c.z + e0.z, fc.z + e1.z) + o};
        for (int i = 0; i < 3; ++i) {
            const double sc = fmax(fabs(lo[i]), fabs(hi[i])) + 1.0;
            st->lo[b][i] = lo[i] - sc * kPad - margin;
            st->hi[b][i] = hi[i] + sc * kPad + margin;
        }
    }
    return MR_STEP_SUCCESS;
}

static int sflag(const OracleScene* s, const SState* st, uint32_t a, uint32_t b) {
    if (b >= s->nb) {
        const v3 pn = qrot(s->plane_rot, V(0, 1, 0));
        const v3 n = vmul(pn, 1.0 / vlen(pn));
        const v3 la = V(st->lo[a][0], st->lo[a][1], st->lo[a][2]), ha = V(st->hi[a][0], st->hi[a][1], st->hi[a][2]);
        const v3 center = vmul(vadd(la, ha), 0.5), halfx = vmul(vsub(ha, la), 0.5);
        const double off = s->offset[a] + st->margin[a];
        const double scale = fmax(fmax(vmaxabs(s->plane_pos), vmaxabs(la)), fmax(vmaxabs(ha), fmax(fabs(s->plane_offset), fabs(off))));
        const v3 an = V(fabs(n.x), fabs(n.y), fabs(n.z));
        const double msd = vdot(n, vsub(center, s->plane_pos)) - vdot(an, halfx);
        BAND(msd, s->plane_offset + (scale + 1.0) * kPad);
        return msd <= s->plane_offset + (scale + 1.0) * kPad;
    }
    int ok = 1;
    for (int i = 0; i < 3; ++i) {
        BAND(st->lo[a][i], st->hi[b][i]);
        BAND(st->lo[b][i], st->hi[a][i]);
        ok = ok && st->lo[a][i] <= st->hi[b][i] && st->lo[b][i] <= st->hi[a][i];
    }
    return ok;
}

static uint32_t squery(const OracleScene* s, const double* q, uint32_t a, uint32_t b, double margin_a, double margin_b, int cls,
                       double* out, uint32_t* status, uint32_t* path) {
    SState* st = (SState*)calloc(1, sizeof(SState));
    for (uint32_t k = 0; k < s->nb; ++k) {
        st->pos[k] = vld(q + 7 * k);
        q4 r = Q(q[7 * k + 3], q[7 * k + 4], q[7 * k + 5], q[7 * k + 6]);
        qnormalize(r, &st->rot[k], 0);
    }
    st->margin[a] = margin_a;
    if (b < s->nb) st->margin[b] = margin_b;
    SCol A, B;
    scol(s, st, a, &A);
    scol(s, st, b, &B);
    if (cls < 0) {
        cls = MR_COLLISION_PAIR_UNSUPPORTED;
        for (uint32_t p = 0; p < s->np; ++p)
            if (s->pa[p] == a && s->pb[p] == b) cls = s->pc[p];
    }
    const double acc = A.offset + B.offset + (fmax(scol_scale(&A), scol_scale(&B)) + 1.0) * kPad;
    SRaw raw;
    const v3 n = snarrow(&A, &B, cls, a, b, acc, &raw);
    for (int i = 0; i < raw.n; ++i) {
        double* o = out + 12 * i;
        vst(o, n);
        o[3] = raw.sep[i];
        vst(o + 4, raw.pa[i]);
        vst(o + 7, raw.pb[i]);
        o[10] = raw.fa[i];
        o[11] = raw.fb[i];
    }
    if (status) *status = raw.status;
    if (path) *path = raw.path;
    free(st);
    return (uint32_t)raw.n;
}

uint32_t oracle_scene_raw_contacts(const OracleScene* s, const double* q, uint32_t a, uint32_t b, double margin_a,
                                   double margin_b, double* out) {
    return squery(s, q, a, b, margin_a, margin_b, -1, out, NULL, NULL);
}

/* One pair under a given pair class: MR_COLLISION_PAIR_CONVEX runs the
 * support-mapped query (GJK / EPA / MPR) on shapes an analytic class also
 * handles, so the two can be compared.  `out` as oracle_scene_raw_contacts;
 * `status` receives a failed query's MR_STEP_* code (0 on success), `path`
 * how a support-mapped query was resolved (0 GJK distance, 3 EPA, 1 MPR). */
uint32_t oracle_scene_pair_query(const OracleScene* s, const double* q, uint32_t a, uint32_t b, uint32_t pair_class, double* out,
                                 uint32_t* status, uint32_t* path) {
    return squery(s, q, a, b, 0.0, 0.0, (int)pair_class, out, status, path);
}

void oracle_scene_table_from_device(const float* words, uint32_t count, OracleSceneSlot* out) {
    for (uint32_t i = 0; i < count; ++i) {
        const float* w = words + (size_t)i * 57;
        memcpy(&out[i].key, w + 56, 4);
        oracle_manifold_from_device((const MRManifoldC*)w, &out[i].m, 1);
    }
}

uint32_t oracle_scene_step(const OracleScene* s, double* q, double* v, OracleSceneSlot* table, uint32_t* count, double friction,
                           OracleSceneTrace* trace) {
    memset(trace, 0, sizeof(*trace));
    for (uint32_t b = 0; b < 64; ++b) trace->island_of[b] = 0xffffffffu;
    g_band = 0;
    g_band_width = kSceneBand;
    g_margin = INFINITY;
    const uint32_t nb = s->nb;
    const double h = s->h;
    SState* st = (SState*)calloc(1, sizeof(SState));
    OracleSceneSlot* cur = (OracleSceneSlot*)calloc(SMAN, sizeof(OracleSceneSlot));
    OracleSceneSlot* nxt = (OracleSceneSlot*)calloc(SMAN, sizeof(OracleSceneSlot));
    SCon* C = (SCon*)calloc(SCON, sizeof(SCon));
    uint32_t mcount = *count, status = MR_STEP_SUCCESS, fail_index = 0;
    memcpy(cur, table, mcount * sizeof(OracleSceneSlot));
    for (uint32_t b = 0; b < nb; ++b) {
        st->pos[b] = vld(q + 7 * b);
        st->rot[b] = Q(q[7 * b + 3], q[7 * b + 4], q[7 * b + 5], q[7 * b + 6]);
        st->lin[b] = vld(v + 6 * b);
        st->ang[b] = vld(v + 6 * b + 3);
    }
    for (uint32_t sub = 0; sub < s->substeps && status == MR_STEP_SUCCESS; ++sub) {
        const int final_substep = sub + 1 == s->substeps;
        sprepare(s, st);
        for (uint32_t b = 0; b < nb; ++b)
            if (!vfinite(st->lin[b]) || !vfinite(st->ang[b])) { status = MR_STEP_NONFINITE_RESULT; fail_index = b; }
        if (status) break;
        status = sbounds(s, st, &fail_index);
        if (status) break;
        uint16_t cand[SCAND];
        uint32_t ncand = 0;
        for (uint32_t p = 0; p < s->np; ++p)
            if (sflag(s, st, s->pa[p], s->pb[p])) {
                if (ncand >= SCAND) { status = MR_STEP_PAIR_CAPACITY_OVERFLOW; fail_index = ncand; break; }
                cand[ncand++] = (uint16_t)p;
            }
        if (status) break;
        if (ncand > trace->candidate_pairs) trace->candidate_pairs = ncand;
        uint32_t ncount = 0, raw_total = 0;
        for (uint32_t ci = 0; ci < ncand && !status; ++ci) {
            const uint32_t p = cand[ci], a = s->pa[p], b = s->pb[p];
            const uint32_t key = a * 65u + b;
            const OracleManifold* old = NULL;
            for (uint32_t m = 0; m < mcount; ++m)
                if (cur[m].key == key) old = &cur[m].m;
            SCol A, B;
            scol(s, st, a, &A);
            scol(s, st, b, &B);
            const double acc = A.offset + B.offset + (fmax(scol_scale(&A), scol_scale(&B)) + 1.0) * kPad;
            SRaw raw;
            const v3 n = snarrow(&A, &B, s->pc[p], a, b, acc, &raw);
            if (raw.status) { status = raw.status; fail_index = key; break; }
            raw_total += (uint32_t)raw.n;
            OracleManifold built;
            const int np_ = sbuild(s, old, &raw, n, &built, A.bpos, A.brot, B.bpos, B.brot);
            if (np_ < 0) { status = MR_STEP_NONFINITE_RESULT; break; }
            if (np_ > 0) {
                if (ncount >= SMAN) { status = MR_STEP_MANIFOLD_CAPACITY_OVERFLOW; fail_index = ncount + 1; break; }
                nxt[ncount].key = key;
                nxt[ncount].m = built;
                ++ncount;
            }
        }
        if (status) break;
        { OracleSceneSlot* t = cur; cur = nxt; nxt = t; }
        mcount = ncount;
        if (mcount > trace->manifold_count) trace->manifold_count = mcount;
        if (raw_total > trace->raw_count) trace->raw_count = raw_total;
        /* Contacts in manifold order. */
        uint32_t total = 0;
        for (uint32_t m = 0; m < mcount; ++m) total += cur[m].m.count;
        if (total > SCON) { status = MR_STEP_CONTACT_CAPACITY_OVERFLOW; fail_index = total; break; }
        total = 0;
        for (uint32_t m = 0; m < mcount; ++m) {
            const OracleManifold* mf = &cur[m].m;
            const uint32_t a = cur[m].key / 65u, b = cur[m].key % 65u;
            const int plane_b = b >= nb;
            const v3 posA = st->pos[a];
            const q4 rotA = st->rot[a];
            const v3 posB = plane_b ? s->ground_pos : st->pos[b];
            const q4 rotB = plane_b ? s->ground_rot : st->rot[b];
            v3 nw = qrot(rotA, vld(mf->normal_local));
            nw = vmul(nw, 1.0 / vlen(nw));
            v3 tw = qrot(rotA, vld(mf->tangent_local));
            tw = vsub(tw, vmul(nw, vdot(tw, nw)));
            tw = vdot(tw, tw) > 1e-12 ? vmul(tw, 1.0 / vlen(tw)) : stable_tangent(nw);
            const v3 bw = vcross(nw, tw);
            const uint32_t ma = s->material[a], mb = plane_b ? s->plane_material : s->material[b];
            const double mu_s = sqrt(fmax(0.0, s->fric[ma][0] * s->fric[mb][0])) * friction;
            const double mu_d = sqrt(fmax(0.0, s->fric[ma][1] * s->fric[mb][1])) * friction;
            const double rest = s->rest[a] + (plane_b ? s->plane_rest : s->rest[b]);
            for (uint32_t i = 0; i < mf->count; ++i) {
                const OraclePoint* op = &mf->points[i];
                SCon* c = &C[total++];
                const v3 pa = rn3(vadd(posA, rn3(qrot(rotA, vld(op->anchor_a)))));
                const v3 pb = rn3(vadd(posB, rn3(qrot(rotB, vld(op->anchor_b)))));
                const v3 pw = vmul(vadd(pa, pb), 0.5);
                c->sep = rn(vdot(vsub(pb, pa), nw) - rest);
                c->a = (int)a;
                c->b = plane_b ? -1 : (int)b;
                c->ra = rn3(vsub(pw, posA));
                c->rb = rn3(vsub(pw, posB));
                c->n = nw;
                c->t = tw;
                c->bt = bw;
                c->new_impact = op->life == 0u;
                c->slot = (int)m;
                c->point = (int)i;
                for (int k = 0; k < 3; ++k) c->lambda[k] = op->impulses[k];
                c->target[0] = c->sep > 0.0 ? -c->sep / h : 0.0;
                c->target[1] = c->target[2] = 0.0;
                c->reg = fmax((s->resp[ma][2] + s->resp[mb][2]) / (h * h) + (s->resp[ma][3] + s->resp[mb][3]) / h, 0.0);
                c->mu = mu_s;
                c->mu_d = mu_d;
                c->restitution = fmin(fmax(fmax(s->resp[ma][0], s->resp[mb][0]), 0.0), 1.0);
                c->rthr = fmax(s->resp[ma][1], s->resp[mb][1]);
            }
        }
        trace->contact_count = total;
        /* IR evaluation at the predicted velocities; blocks; relaxation. */
        for (uint32_t i = 0; i < total; ++i) {
            SCon* c = &C[i];
            const v3 va = rn3(vadd(st->lin[c->a], rn3(vcross(st->ang[c->a], c->ra))));
            const v3 vb = c->b >= 0 ? rn3(vadd(st->lin[c->b], rn3(vcross(st->ang[c->b], c->rb)))) : V(0, 0, 0);
            const v3 dv = vsub(vb, va);
            const v3 dirs[3] = {c->n, c->t, c->bt};
            const double rel[3] = {vdot(dv, dirs[0]), vdot(dv, dirs[1]), vdot(dv, dirs[2])};
            const double tau_c = 2.0 * h, ratio = h / tau_c;
            const double err = fmin(c->sep + s->slop, 0.0);
            double stab = -h * err / (tau_c * tau_c * (1.0 + 2.0 * ratio + ratio * ratio));
            stab = fmin(fmax(stab, 0.0), s->max_dep);
            if (c->new_impact) {
                const double incoming = rel[0] - c->target[0];
                if (c->restitution > 0.0) BAND(incoming, -c->rthr);
                if (incoming < -c->rthr) stab = fmax(stab, -c->restitution * incoming);
            }
            c->target[0] = rn(c->target[0] + stab);
            const double slip = sqrt(rel[1] * rel[1] + rel[2] * rel[2]);
            if (c->mu_d != c->mu) BAND(slip, 1e-3);
            if (!(slip <= 1e-3)) c->mu = c->mu_d;
            double W[9] = {0};
            for (int side = 0; side < 2; ++side) {
                const int body = side ? c->b : c->a;
                if (body < 0) continue;
                const v3 r = side ? c->rb : c->ra;
                for (int x = 0; x < 3; ++x)
                    for (int y = 0; y < 3; ++y) {
                        const v3 rx = vcross(r, dirs[x]), ry = vcross(r, dirs[y]);
                        W[x * 3 + y] = rn(W[x * 3 + y] + s->inv_mass[body] * vdot(dirs[x], dirs[y]) + vdot(rx, sym3_apply(st->iiw[body], ry)));
                    }
            }
            double rowsum = 0.0;
            for (uint32_t j = 0; j < total; ++j) {
                const SCon* d = &C[j];
                double w = 0.0;
                int shared = 0;
                for (int t = 0; t < 2; ++t) {
                    const int bi = t ? c->b : c->a;
                    if (bi < 0) continue;
                    const int tj = d->a == bi ? 0 : (d->b == bi ? 1 : -1);
                    if (tj < 0) continue;
                    shared = 1;
                    const double si = t ? 1.0 : -1.0, sj = tj ? 1.0 : -1.0;
                    const v3 ri = t ? c->rb : c->ra, rj = tj ? d->rb : d->ra;
                    w += si * sj * (s->inv_mass[bi] * vdot(c->n, d->n) + vdot(vcross(ri, c->n), sym3_apply(st->iiw[bi], vcross(rj, d->n))));
                }
                if (shared) rowsum += fabs(w);
            }
            const double diag = fabs(W[0]) + c->reg;
            W[0] += c->reg;
            for (int e = 0; e < 9; ++e) W[e] = rn(W[e]);
            if (!oracle_invert3x3(W, c->P)) { status = MR_STEP_FACTORIZATION_FAILED; fail_index = i; break; }
            for (int e = 0; e < 9; ++e) c->P[e] = rn(c->P[e]);
            c->relax = rowsum > fmax(diag, kMatrixFloor) ? fmin(fmax(diag / rowsum, 1.0 / 32.0), 1.0) : 1.0;
            double warm[3];
            oracle_project_cone(c->lambda, c->mu, c->mu, warm);
            for (int k = 0; k < 3; ++k) { c->lambda[k] = warm[k]; c->delta[k] = warm[k]; }
        }
        if (status) break;
        /* Islands (min-root union find over dynamic bodies): a diagnostic,
         * counted on the final substep (the solve is island-independent). */
        if (total > 0 && final_substep) {
            int parent[SNB], touched[SNB] = {0};
            for (uint32_t b = 0; b < nb; ++b) parent[b] = (int)b;
            for (uint32_t i = 0; i < total; ++i) {
                int x = C[i].a;
                touched[x] = 1;
                if (C[i].b >= 0) {
                    int y = C[i].b;
                    touched[y] = 1;
                    while (parent[x] != x) x = parent[x];
                    while (parent[y] != y) y = parent[y];
                    if (x != y) parent[x > y ? x : y] = x < y ? x : y;
                }
            }
            uint32_t islands = 0, island_of_root[SNB];
            for (uint32_t b = 0; b < nb; ++b) {
                int r = (int)b;
                while (parent[r] != r) r = parent[r];
                island_of_root[b] = 0xffffffffu;
                if (touched[b] && r == (int)b) island_of_root[b] = islands++;
            }
            if (islands > trace->islands) trace->islands = islands;
            trace->island_contacts = total < 256 ? total : 256;
            for (uint32_t i = 0; i < trace->island_contacts; ++i) {
                trace->island_pairs[2 * i] = C[i].a;
                trace->island_pairs[2 * i + 1] = C[i].b;
            }
            for (uint32_t b = 0; b < 64; ++b) trace->island_of[b] = 0xffffffffu;
            for (uint32_t b = 0; b < nb && b < 64; ++b) {
                int r = (int)b;
                while (parent[r] != r) r = parent[r];
                trace->island_of[b] = island_of_root[r];
            }
        }
        /* Jacobi sweeps; sweep -1 applies the warm start. */
        const int iters = (int)s->iters + (final_substep ? (int)s->final_iters : 0);
        for (int it = -1; it < iters && !status; ++it) {
            if (it >= 0) {
                for (uint32_t i = 0; i < total; ++i) {
                    SCon* c = &C[i];
                    const v3 va = rn3(vadd(st->lin[c->a], rn3(vcross(st->ang[c->a], c->ra))));
                    const v3 vb = c->b >= 0 ? rn3(vadd(st->lin[c->b], rn3(vcross(st->ang[c->b], c->rb)))) : V(0, 0, 0);
                    const v3 dv = vsub(vb, va);
                    const double r0 = rn(c->target[0] - vdot(dv, c->n) - c->reg * c->lambda[0]);
                    const double r1 = rn(c->target[1] - vdot(dv, c->t));
                    const double r2 = rn(c->target[2] - vdot(dv, c->bt));
                    double prop[3], proj[3];
                    for (int k = 0; k < 3; ++k) prop[k] = c->lambda[k] + c->P[3 * k] * r0 + c->P[3 * k + 1] * r1 + c->P[3 * k + 2] * r2;
                    oracle_project_cone(prop, c->mu, c->mu, proj);
                    for (int k = 0; k < 3; ++k) c->delta[k] = rn(c->relax * (proj[k] - c->lambda[k]));
                    int finite = 1;
                    for (int k = 0; k < 3; ++k) finite &= isfinite(c->lambda[k] + c->delta[k]) && isfinite(c->delta[k]);
                    if (!finite) { status = MR_STEP_NONFINITE_RESULT; fail_index = i; break; }
                    for (int k = 0; k < 3; ++k) c->lambda[k] += c->delta[k];
                }
                if (status) break;
            }
            for (uint32_t b = 0; b < nb; ++b) {
                v3 dl = V(0, 0, 0), dw = V(0, 0, 0);
                for (uint32_t i = 0; i < total; ++i) {
                    const SCon* c = &C[i];
                    for (int side = 0; side < 2; ++side) {
                        if ((side ? c->b : c->a) != (int)b) continue;
                        const v3 imp = vadd(vadd(vmul(c->n, c->delta[0]), vmul(c->t, c->delta[1])), vmul(c->bt, c->delta[2]));
                        const v3 f = side ? imp : vmul(imp, -1.0);
                        dl = rn3(vadd(dl, f));
                        dw = rn3(vadd(dw, vcross(side ? c->rb : c->ra, f)));
                    }
                }
                st->lin[b] = rn3(vadd(st->lin[b], vmul(dl, s->inv_mass[b])));
                st->ang[b] = rn3(vadd(st->ang[b], sym3_apply(st->iiw[b], dw)));
            }
        }
        if (status) break;
        for (uint32_t i = 0; i < total; ++i)
            for (int k = 0; k < 3; ++k) cur[C[i].slot].m.points[C[i].point].impulses[k] = C[i].lambda[k];
        for (uint32_t b = 0; b < nb; ++b) {
            v3 lin = st->lin[b], ang = st->ang[b];
            const double ls = vlen(lin), ws = vlen(ang);
            if (s->max_lin[b] > 0.0 && ls > s->max_lin[b]) lin = vmul(lin, s->max_lin[b] / ls);
            if (s->max_ang[b] > 0.0 && ws > s->max_ang[b]) ang = vmul(ang, s->max_ang[b] / ws);
            const v3 c = rn3(vadd(st->pos[b], vmul(lin, h)));
            q4 qn = qmul(so3_increment(vmul(ang, h), 0), st->rot[b]);
            const double qq = qdot(qn, qn);
            if (!qfinite(qn) || !(qq > 1e-12) || !vfinite(c)) { status = MR_STEP_NONFINITE_RESULT; fail_index = b; break; }
            const double inv = 1.0 / sqrt(qq);
            st->rot[b] = Q(rn(qn.x * inv), rn(qn.y * inv), rn(qn.z * inv), rn(qn.w * inv));
            st->pos[b] = c;
            st->lin[b] = lin;
            st->ang[b] = ang;
        }
    }
    trace->status = status;
    trace->failing_index = fail_index;
    trace->band_decisions = g_band;
    trace->min_decision_margin = g_margin;
    g_band_width = kBand;
    if (status == MR_STEP_SUCCESS) {
        for (uint32_t b = 0; b < nb; ++b) {
            vst(q + 7 * b, st->pos[b]);
            q[7 * b + 3] = st->rot[b].x;
            q[7 * b + 4] = st->rot[b].y;
            q[7 * b + 5] = st->rot[b].z;
            q[7 * b + 6] = st->rot[b].w;
            vst(v + 6 * b, st->lin[b]);
            vst(v + 6 * b + 3, st->ang[b]);
        }
        memcpy(table, cur, mcount * sizeof(OracleSceneSlot));
        *count = mcount;
    }
    free(st);
    free(cur);
    free(nxt);
    free(C);
    return status;
}

uint32_t oracle_scene_collide(const OracleScene* s, const double* q, OracleSceneSlot* table, uint32_t* count, double* raw_out,
                              uint32_t raw_cap, uint32_t* raw_count) {
    g_band = 0;
    g_margin = INFINITY;
    SState* st = (SState*)calloc(1, sizeof(SState));
    OracleSceneSlot* nxt = (OracleSceneSlot*)calloc(SMAN, sizeof(OracleSceneSlot));
    uint32_t status = MR_STEP_SUCCESS, ncount = 0, nraw = 0;
    for (uint32_t b = 0; b < s->nb; ++b) {
        st->pos[b] = vld(q + 7 * b);
        if (!qnormalize(Q(q[7 * b + 3], q[7 * b + 4], q[7 * b + 5], q[7 * b + 6]), &st->rot[b], 1)) status = MR_STEP_NONFINITE_INPUT;
    }
    for (uint32_t p = 0; p < s->np && status == MR_STEP_SUCCESS; ++p) {
        const uint32_t a = s->pa[p], b = s->pb[p], key = a * 65u + b;
        const OracleManifold* old = NULL;
        for (uint32_t m = 0; m < *count; ++m)
            if (table[m].key == key) old = &table[m].m;
        SCol A, B;
        scol(s, st, a, &A);
        scol(s, st, b, &B);
        const double acc = A.offset + B.offset + (fmax(scol_scale(&A), scol_scale(&B)) + 1.0) * kPad;
        SRaw raw;
        const v3 n = snarrow(&A, &B, s->pc[p], a, b, acc, &raw);
        if (raw.status) { status = raw.status; break; }
        for (int i = 0; i < raw.n && nraw < raw_cap; ++i, ++nraw) {
            double* o = raw_out + 16 * nraw;
            o[0] = a;
            o[1] = b;
            vst(o + 2, n);
            o[5] = raw.sep[i];
            vst(o + 6, raw.pa[i]);
            vst(o + 9, raw.pb[i]);
            o[12] = raw.fa[i];
            o[13] = raw.fb[i];
            o[14] = o[15] = 0.0;
        }
        OracleManifold built;
        const int np_ = sbuild(s, old, &raw, n, &built, A.bpos, A.brot, B.bpos, B.brot);
        if (np_ < 0) { status = MR_STEP_NONFINITE_RESULT; break; }
        if (np_ > 0) {
            if (ncount >= SMAN) { status = MR_STEP_MANIFOLD_CAPACITY_OVERFLOW; break; }
            nxt[ncount].key = key;
            nxt[ncount].m = built;
            ++ncount;
        }
    }
    if (status == MR_STEP_SUCCESS) {
        memcpy(table, nxt, ncount * sizeof(OracleSceneSlot));
        *count = ncount;
        *raw_count = nraw;
    }
    free(st);
    free(nxt);
    return status;
}
