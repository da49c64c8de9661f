// Free-body control step on B200 -- device code shared by the per-world
// kernel (scene_step.cu) and the heterogeneous batch kernel (mix_step.cu):
// piles of spheres, capsules, boxes and cylinders on a ground plane
// (numi-lab's scene bodies).  One warp per environment for a whole
// control step; lanes own bodies (two per lane), compiled pairs, candidate
// pairs, manifolds and contacts in turn.
//
// Stage order per substep follows the reference's MetalWorld graph for scene
// bodies: prediction (mr_world_predict_scene, MetalWorldContact.metal:
// 2509-2570: exponential damping and gravity, no gyroscopic term),
// collider projection with the speculative sweep (Collision.metal:
// 5960-6030), pair flags over the compiled all-pairs list (Collision.metal:
// 7905-8180), analytic narrowphase (Collision.cpp:1106-2175 restated:
// sphere-sphere, sphere-box witness, box-box separating axes with vertex
// clipping, sphere/box vs plane), persistent manifolds keyed by collider
// pair, ConstraintIR evaluation, islands (min-root union find,
// ConstraintSolver.cpp:848-900), the temporalCone block-Jacobi solve with
// free-body responses, speed clamps and integration, and the per-environment
// latch: a failed control step publishes nothing, so the environment keeps
// its step-start state.
#pragma once

#include "audit.cuh"
#include "contact.cuh"
#include "dmath.cuh"
#include "numi_b200.h"
#include "scene.h"

#include <cstdint>

namespace numi {
namespace {

constexpr float kQueryPadS = 0.00000762939453125f;  // MR_COLLISION_QUERY_RELATIVE_PAD
constexpr float kAabbPadS = 0.00000762939453125f;   // MR_COLLISION_AABB_RELATIVE_PAD
constexpr float kTinyS = 1.0e-14f;  // Collision.metal:10
constexpr float kTieRel = 1.0e-5f;
constexpr float kTieAbs = 1.0e-12f;
constexpr int kRawCap = 8;
// Box-box separating axes, FP32 rules of the GPU collision
// (Collision.metal:1600-1650): edge pairs closer to parallel than
// |sin| = 1e-6 give no axis, and separations within a relative 1e-7 tie
// (the first axis wins).  The FP64 CPU collision uses 1e-24 and 1e-12.
constexpr float kParallelEdges = 1.0e-12f;
constexpr float kAxisTie = 1.0e-7f;
constexpr int kRecWords = 16;                                   // candidate record
constexpr int kLaneScratch = (4 + kRawCap) * kRecWords + 4;  // records, candidate ids
constexpr int kCw = 40;                                          // contact record words

// Shared-memory layout of one environment (floats): body state, swept
// bounds, candidate pairs and per-body contact lists -- about 9 KB, so that
// registers, not shared memory, bound the resident warps.
constexpr int kOffPos = 0;
constexpr int kOffQuat = kOffPos + kSceneMaxBodies * 3;
constexpr int kOffLin = kOffQuat + kSceneMaxBodies * 4;
constexpr int kOffAng = kOffLin + kSceneMaxBodies * 3;
constexpr int kOffIiw = kOffAng + kSceneMaxBodies * 3;   // world inverse inertia, sym 6
constexpr int kOffLo = kOffIiw + kSceneMaxBodies * 6;
constexpr int kOffHi = kOffLo + kSceneMaxBodies * 3;
constexpr int kOffMargin = kOffHi + kSceneMaxBodies * 3;
// Candidate pairs (u16) live only until the narrowphase has consumed them;
// the per-body contact list entries (u16) reuse their words afterwards.
constexpr int kOffCand = kOffMargin + kSceneMaxBodies;
constexpr int kOffEntries = kOffCand;
constexpr int kCandWords = (kSceneCandidates > 2 * kSceneContacts ? kSceneCandidates : 2 * kSceneContacts) / 2;
constexpr int kOffLists = kOffCand + kCandWords;  // start[65], fill[65] (ints)
constexpr int kOffKeys = kOffLists + 2 * (kSceneMaxBodies + 1);  // pair keys of the two tables (u32)
constexpr int kOffFirst = kOffKeys + 2 * kSceneManifolds;  // first contact of each manifold (u16, +1)
constexpr int kOffMisc = kOffFirst + (kSceneManifolds + 2) / 2;
constexpr int kSceneSmemWords = kOffMisc + 32;
// Compensated precision only, past the FP32 layout: compensation terms of
// the body positions' running sums (persistent, [env][body][7] entries 0-2
// in HBM) and of the substep's velocity sums over the Jacobi sweeps.
constexpr int kOffPosComp = kSceneSmemWords;
constexpr int kOffLinComp = kOffPosComp + kSceneMaxBodies * 3;
constexpr int kOffAngComp = kOffLinComp + kSceneMaxBodies * 3;
constexpr int kSceneSmemWordsComp = kOffAngComp + kSceneMaxBodies * 3;

// Global workspace of one environment (floats, L2-resident while the
// environment runs): two substep manifold tables, the contact records and
// one narrowphase scratch block per lane.
constexpr int kTableWords = kSceneManifolds * kSceneSlotWords;
constexpr int kWsTable0 = 0;
constexpr int kWsTable1 = kWsTable0 + kTableWords;
constexpr int kWsContacts = kWsTable1 + kTableWords;
constexpr int kWsLanes = kWsContacts + kSceneContacts * kCw;
constexpr int kWsWords = (kWsLanes + 32 * kLaneScratch + 31) / 32 * 32;

enum SceneMisc : int { kSmStatus = 0, kSmFail = 1, kSmContacts = 2, kSmManifolds = 3, kSmRaw = 4, kSmCand = 5, kSmIslands = 6 };
enum SceneCw : int {
    kScA = 0, kScB = 1, kScRa = 2, kScRb = 5, kScN = 8, kScT = 11, kScBt = 14, kScTarget = 17, kScReg = 20, kScMu = 21,
    kScLambda = 22, kScPre = 25, kScRelax = 34, kScDelta = 35, kScSlot = 38, kScFlags = 39
};
enum CandWord : int { kCdLaS = 0, kCdLbS = 3, kCdFaS = 6, kCdFbS = 7, kCdWpS = 8, kCdSepS = 11, kCdLifeS = 12, kCdImpS = 13 };

__device__ __forceinline__ int ai(float f) { return __float_as_int(f); }
__device__ __forceinline__ float af(int i) { return __int_as_float(i); }

// One contact record.  Records are stored word-major ([word][contact]), so
// the lanes of a warp reading one word of consecutive contacts touch one
// cache line.
struct Rec {
    float* p;
    __device__ __forceinline__ float& operator[](int w) const { return p[w * kSceneContacts]; }
    __device__ __forceinline__ float3 v3(int w) const {
        return f3(p[w * kSceneContacts], p[(w + 1) * kSceneContacts], p[(w + 2) * kSceneContacts]);
    }
    __device__ __forceinline__ void set3(int w, float3 v) const {
        p[w * kSceneContacts] = v.x;
        p[(w + 1) * kSceneContacts] = v.y;
        p[(w + 2) * kSceneContacts] = v.z;
    }
};
__device__ __forceinline__ Rec rec(float* C, int c) { return Rec{C + c}; }

__device__ __forceinline__ void fail(float* misc, unsigned code, unsigned index) {
    if (ai(misc[kSmStatus]) == MR_STEP_SUCCESS) {
        misc[kSmStatus] = af(static_cast<int>(code));
        misc[kSmFail] = af(static_cast<int>(index));
    }
}
__device__ __forceinline__ bool ok(const float* misc) {
    __syncwarp();
    return ai(misc[kSmStatus]) == MR_STEP_SUCCESS;
}

// World collider of a body or of the ground plane (index nb).
struct Collider {
    int type;
    float3 c;        // centre (= body position; colliders sit at the COM)
    float4 r;        // orientation
    float3 half;     // box half extents
    float radius;
    float offset;    // contact offset incl. speculative margin
    float3 lo, hi;   // swept, inflated bounds (finite shapes)
    float3 e0, e1;   // capsule segment endpoints (local -Y / +Y ends)
    float3 axis, bx, bz;  // cylinder axis (local +Y) and disk basis
    float hl;        // cylinder half length
    float3 normal;   // plane normal
    float3 bpos;     // pose of the collider's body: the frame of its
    float4 brot;     // manifold anchors (the ground body for the plane)
    const float4* hull;  // convex: scaled local hull vertices
    int hull_count;
};

__device__ void load_collider(const SceneModel& M, const float* s, int b, Collider& o) {
    if (b >= M.nb) {
        o.type = MR_SHAPE_PLANE;
        o.c = xyz(M.plane_position);
        o.r = M.plane_rotation;
        const float3 n = qrot(o.r, f3(0.0f, 1.0f, 0.0f));
        o.normal = n * rsqrtf(dot3(n, n));
        o.half = f3(0.0f, 0.0f, 0.0f);
        o.radius = 0.0f;
        o.offset = M.plane_offsets.x;
        o.lo = o.hi = f3(0.0f, 0.0f, 0.0f);
        o.axis = o.bx = o.bz = f3(0.0f, 0.0f, 0.0f);
        o.hl = 0.0f;
        o.bpos = xyz(M.ground_position);
        o.brot = M.ground_rotation;
        o.hull = nullptr;
        o.hull_count = 0;
        return;
    }
    o.type = M.shape_type[b];
    o.c = ld3(s + kOffPos + b * 3);
    o.r = ld4(s + kOffQuat + b * 4);
    const float4 d = M.dims[b];
    o.half = xyz(d);
    o.radius = d.x;
    o.offset = M.offsets[b].x + s[kOffMargin + b];
    o.lo = ld3(s + kOffLo + b * 3);
    o.hi = ld3(s + kOffHi + b * 3);
    if (o.type == MR_SHAPE_CAPSULE) {
        const float3 axis = qrot(o.r, f3(0.0f, d.y, 0.0f));
        o.e0 = o.c - axis;
        o.e1 = o.c + axis;
    } else {
        o.e0 = o.e1 = o.c;
    }
    o.hl = d.y;
    if (o.type == MR_SHAPE_CYLINDER) {
        // Collision.metal:759-784: unit axis, disk basis X orthogonalised
        // against it, Z = X x axis.
        float3 ax = qrot(o.r, f3(0.0f, 1.0f, 0.0f));
        ax = ax * rsqrtf(dot3(ax, ax));
        float3 bx = qrot(o.r, f3(1.0f, 0.0f, 0.0f));
        bx = bx - ax * dot3(ax, bx);
        bx = bx * rsqrtf(dot3(bx, bx));
        float3 bz = cross3(bx, ax);
        o.axis = ax;
        o.bx = bx;
        o.bz = bz * rsqrtf(dot3(bz, bz));
    } else {
        o.axis = o.bx = o.bz = f3(0.0f, 0.0f, 0.0f);
    }
    o.normal = f3(0.0f, 0.0f, 0.0f);
    o.bpos = o.c;
    o.brot = o.r;
    o.hull = M.hull_vertices + M.hull_first[b];
    o.hull_count = o.type == MR_SHAPE_CONVEX ? M.hull_count[b] : 0;
}

__device__ __forceinline__ float collider_scale(const Collider& k) {
    return fmaxf(fmaxf(maxabs3(k.c), maxabs3(k.half)), fmaxf(fabsf(k.radius), fmaxf(fabsf(k.offset),
                 fmaxf(maxabs3(k.lo), maxabs3(k.hi)))));
}

__device__ __forceinline__ float3 box_axis(const Collider& b, int axis) {
    return qrot(b.r, f3(axis == 0 ? 1.0f : 0.0f, axis == 1 ? 1.0f : 0.0f, axis == 2 ? 1.0f : 0.0f));
}
__device__ __forceinline__ float box_radius(const Collider& b, float3 axis) {
    return fabsf(dot3(axis, box_axis(b, 0))) * b.half.x + fabsf(dot3(axis, box_axis(b, 1))) * b.half.y +
           fabsf(dot3(axis, box_axis(b, 2))) * b.half.z;
}
__device__ __forceinline__ float3 box_vertex(const Collider& b, int v) {
    return b.c + qrot(b.r, f3((v & 1) ? b.half.x : -b.half.x, (v & 2) ? b.half.y : -b.half.y, (v & 4) ? b.half.z : -b.half.z));
}
__device__ __forceinline__ bool inside_inflated(float3 p, const Collider& b, float inflation) {
    const float3 l = qrotinv(b.r, p - b.c);
    return fabsf(l.x) <= b.half.x + inflation && fabsf(l.y) <= b.half.y + inflation && fabsf(l.z) <= b.half.z + inflation;
}
__device__ __forceinline__ float3 box_support(const Collider& b, float3 d) {
    float3 out = b.c;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float3 ax = box_axis(b, a);
        const float he = a == 0 ? b.half.x : (a == 1 ? b.half.y : b.half.z);
        out = out + ax * (dot3(d, ax) >= 0.0f ? he : -he);
    }
    return out;
}
__device__ __forceinline__ float3 coincident_normal(unsigned a, unsigned b) {
    const unsigned hsh = a * 73856093u ^ b * 19349663u;
    const unsigned axis = hsh % 3u;
    const float sign = (hsh & 4u) == 0u ? 1.0f : -1.0f;
    return f3(axis == 0u ? sign : 0.0f, axis == 1u ? sign : 0.0f, axis == 2u ? sign : 0.0f);
}

// Segment helpers of the capsule classes (Collision.metal:965-1125,
// Collision.cpp:1169-1336, restated).
__device__ __forceinline__ unsigned capsule_feature(float t) { return t <= 0.0f ? 0u : (t >= 1.0f ? 1u : 2u); }

__device__ float3 stable_segment_normal(float3 da, float3 db, unsigned ia, unsigned ib) {
    const float3 cr = cross3(da, db);
    if (dot3(cr, cr) > kTinyS) return cr * rsqrtf(dot3(cr, cr));
    float3 dir;
    if (dot3(da, da) > kTinyS) dir = da * rsqrtf(dot3(da, da));
    else if (dot3(db, db) > kTinyS) dir = db * rsqrtf(dot3(db, db));
    else return coincident_normal(ia, ib);
    const float ax = fabsf(dir.x), ay = fabsf(dir.y), az = fabsf(dir.z);
    const float3 ref = (ax <= ay && ax <= az) ? f3(1.0f, 0.0f, 0.0f) : (ay <= az ? f3(0.0f, 1.0f, 0.0f) : f3(0.0f, 0.0f, 1.0f));
    float3 out = cross3(dir, ref);
    out = out * rsqrtf(dot3(out, out));
    return ((ia * 73856093u) ^ (ib * 19349663u)) & 4u ? -out : out;
}

__device__ __forceinline__ float3 closest_on_segment(float3 x, float3 e0, float3 e1, float& t) {
    const float3 seg = e1 - e0;
    const float sq = dot3(seg, seg);
    if (!(sq > kTinyS)) {
        t = 0.0f;
        return e0;
    }
    t = fminf(fmaxf(dot3(x - e0, seg) / sq, 0.0f), 1.0f);
    return e0 + seg * t;
}

__device__ void closest_segments(float3 a0, float3 a1, float3 b0, float3 b1, float3& pa, float3& pb, float& ta, float& tb) {
    const float3 da = a1 - a0, db = b1 - b0, off = a0 - b0;
    const float sa = dot3(da, da), sb = dot3(db, db), pa_ = dot3(da, off), pb_ = dot3(db, off);
    ta = 0.0f;
    tb = 0.0f;
    if (!(sa > kTinyS) && !(sb > kTinyS)) {
        pa = a0;
        pb = b0;
        return;
    }
    if (!(sa > kTinyS)) {
        tb = fminf(fmaxf(pb_ / sb, 0.0f), 1.0f);
    } else {
        const float cp = dot3(da, db);
        if (!(sb > kTinyS)) {
            ta = fminf(fmaxf(-pa_ / sa, 0.0f), 1.0f);
        } else {
            const float den = sa * sb - cp * cp;
            if (den > kTinyS * sa * sb) ta = fminf(fmaxf((cp * pb_ - pa_ * sb) / den, 0.0f), 1.0f);
            tb = (cp * ta + pb_) / sb;
            if (tb < 0.0f) {
                tb = 0.0f;
                ta = fminf(fmaxf(-pa_ / sa, 0.0f), 1.0f);
            } else if (tb > 1.0f) {
                tb = 1.0f;
                ta = fminf(fmaxf((cp - pa_) / sa, 0.0f), 1.0f);
            }
        }
    }
    pa = a0 + da * ta;
    pb = b0 + db * tb;
}

// Capsule-box witness in the box frame (Collision.metal:1241,
// Collision.cpp:1462): the segment's deepest point when it pierces the box,
// else the closest of the two clamped endpoints and the twelve edges.
// Normal from the capsule to the box, world frame.
struct CapsuleBoxWitness {
    float3 normal, cap_point, box_point;
    float sep, t_cap;
    unsigned box_feature;
};

__device__ __forceinline__ CapsuleBoxWitness capsule_box_witness(float3 ce0, float3 ce1, float cap_radius, float3 bc, float4 br,
                                                             float3 half, unsigned ic, unsigned ib) {
    CapsuleBoxWitness w;
    const float3 s0 = qrotinv(br, ce0 - bc), s1 = qrotinv(br, ce1 - bc);
    const float3 dir = s1 - s0;
    const float he[3] = {half.x, half.y, half.z};
    const float st[3] = {s0.x, s0.y, s0.z}, dd[3] = {dir.x, dir.y, dir.z};
    float enter = 0.0f, exit = 1.0f;
    bool inside = true;
    for (int a = 0; a < 3; ++a) {
        if (fabsf(dd[a]) <= kTinyS) {
            if (st[a] < -he[a] || st[a] > he[a]) inside = false;
            continue;
        }
        float t0 = (-he[a] - st[a]) / dd[a], t1 = (he[a] - st[a]) / dd[a];
        if (t0 > t1) { const float t = t0; t0 = t1; t1 = t; }
        enter = fmaxf(enter, t0);
        exit = fminf(exit, t1);
        if (enter > exit) inside = false;
    }
    if (inside) {
        const float t_cap = fminf(fmaxf(0.5f * (enter + exit), 0.0f), 1.0f);
        const float3 core = s0 + dir * t_cap;
        const float cc[3] = {core.x, core.y, core.z};
        const float dist[3] = {he[0] - fabsf(cc[0]), he[1] - fabsf(cc[1]), he[2] - fabsf(cc[2])};
        int axis = 0;
        if (dist[1] < dist[axis]) axis = 1;
        if (dist[2] < dist[axis]) axis = 2;
        const float sign = cc[axis] >= 0.0f ? 1.0f : -1.0f;
        const float3 outward = f3(axis == 0 ? sign : 0.0f, axis == 1 ? sign : 0.0f, axis == 2 ? sign : 0.0f);
        float3 lbox = core;
        if (axis == 0) lbox.x = sign * he[0];
        else if (axis == 1) lbox.y = sign * he[1];
        else lbox.z = sign * he[2];
        const float3 ln = -outward;
        w.normal = qrot(br, ln);
        w.cap_point = bc + qrot(br, core + ln * cap_radius);
        w.box_point = bc + qrot(br, lbox);
        w.sep = -dist[axis] - cap_radius;
        w.t_cap = t_cap;
        w.box_feature = 27u + 2u * static_cast<unsigned>(axis) + (sign > 0.0f ? 1u : 0u);
        return w;
    }
    float best = INFINITY, best_t = 0.0f;
    float3 best_seg = s0, best_box = s0;
    unsigned best_f = 0xffffffffu;
    auto consider = [&](float3 sp, float3 bp, float t, unsigned f) {
        const float3 d = bp - sp;
        const float sq = dot3(d, d);
        const float tol = 1.0e-12f * (1.0f + fmaxf(best, sq));
        if (!isfinite(best) || sq < best - tol || (fabsf(sq - best) <= tol && f < best_f)) {
            best = sq;
            best_seg = sp;
            best_box = bp;
            best_t = t;
            best_f = f;
        }
    };
    for (int e = 0; e < 2; ++e) {
        const float3 sp = e == 0 ? s0 : s1;
        consider(sp, f3(fminf(fmaxf(sp.x, -he[0]), he[0]), fminf(fmaxf(sp.y, -he[1]), he[1]), fminf(fmaxf(sp.z, -he[2]), he[2])),
                 static_cast<float>(e), static_cast<unsigned>(e));
    }
    unsigned feature = 2u;
    for (int va = 0; va < 3; ++va) {
        const int f0 = (va + 1) % 3, f1 = (va + 2) % 3;
        for (int sg = 0; sg < 4; ++sg) {
            float c0[3], c1[3];
            c0[va] = -he[va];
            c1[va] = he[va];
            c0[f0] = c1[f0] = ((sg & 1) ? 1.0f : -1.0f) * he[f0];
            c0[f1] = c1[f1] = ((sg & 2) ? 1.0f : -1.0f) * he[f1];
            float3 pa, pb;
            float ta, tb;
            closest_segments(s0, s1, f3(c0[0], c0[1], c0[2]), f3(c1[0], c1[1], c1[2]), pa, pb, ta, tb);
            consider(pa, pb, ta, feature);
            ++feature;
        }
    }
    const float dist = sqrtf(fmaxf(best, 0.0f));
    const float3 ln = dist > kTinyS ? (best_box - best_seg) * (1.0f / dist) : qrotinv(br, coincident_normal(ic, ib));
    w.normal = qrot(br, ln);
    w.cap_point = bc + qrot(br, best_seg + ln * cap_radius);
    w.box_point = bc + qrot(br, best_box);
    w.sep = dist - cap_radius;
    w.t_cap = best_t;
    w.box_feature = 64u + best_f;
    return w;
}

// Raw contacts of one pair into candidate records (anchors in the bodies'
// frames, features, world midpoint, separation); returns the count and the
// pair's normal (A -> B).  Collision.cpp generateContacts, restated.
struct RawSink {
    float* rec;
    int count;
    float3 posA, posB;
    float4 rotA, rotB;
    __device__ void add(float3 pa, float3 pb, float sep, unsigned fa, unsigned fb) {
        if (count >= kRawCap) return;
        float* r = rec + count * kRecWords;
        st3(r + kCdLaS, qrotinv(rotA, pa - posA));
        st3(r + kCdLbS, qrotinv(rotB, pb - posB));
        r[kCdFaS] = af(static_cast<int>(fa));
        r[kCdFbS] = af(static_cast<int>(fb));
        st3(r + kCdWpS, 0.5f * (pa + pb));
        r[kCdSepS] = sep;
        ++count;
    }
};

// ---------------------------------------------------------------------------
// Support-mapped narrowphase: cylinder pairs (the reference's primitive-GJK
// class, MR_WORLD_WORK_PRIMITIVE_GJK): GJK distance (Collision.metal:
// 2298-2427), on overlap EPA (2511-2783) with MPR as the fallback
// (2786-3193), then the cylinder's contact patch (3327-3432).  One lane runs
// one pair; the simplex, the EPA polytope and the MPR portal are per-thread
// local arrays (about 6 KB, in the interleaved local space).  Two choices
// differ from the reference's text, in the device and the oracle alike:
// EPA orients a face against an interior point of the polytope rather than
// the origin (the same unless the origin lies on the face plane, where the
// origin test is ambiguous), and EPA reports the closest face's outward
// normal -- the A -> B normal of every other class -- where the reference
// writes its negation.  No query cache warm-starts GJK.
// ---------------------------------------------------------------------------
constexpr int kGjkIterations = 32;  // MR_GJK_MAX_ITERATIONS
constexpr int kEpaIterations = 48;  // MR_EPA_MAX_ITERATIONS
constexpr int kEpaVertices = 64;    // MR_EPA_VERTEX_CAPACITY
constexpr int kEpaFaces = 128;      // MR_EPA_FACE_CAPACITY
constexpr float kCylAlign = 1.0e-6f;  // Collision.metal:21
enum : unsigned { kCylNegRing = 0u, kCylPosRing = 4u, kCylNegSide = 8u, kCylPosSide = 9u, kCylNegRim = 10u, kCylPosRim = 11u };
constexpr float kFltEps = 1.1920929e-7f;

struct Sup {
    float3 w, pa, pb;  // Minkowski point A - B and its supports
    unsigned fa, fb;
};

struct SmQuery {
    float3 normal, pa, pb;
    float sep;
    unsigned fa, fb;
};

__device__ __forceinline__ float3 deterministic_direction(unsigned key) {
    const unsigned axis = key % 3u;
    const float sign = (key & 4u) == 0u ? 1.0f : -1.0f;
    return f3(axis == 0u ? sign : 0.0f, axis == 1u ? sign : 0.0f, axis == 2u ? sign : 0.0f);
}

__device__ float3 shape_support(const Collider& k, unsigned index, float3 d, unsigned& feat) {
    const float dd = dot3(d, d);
    d = (!(dd > kTinyS) || !isfinite(dd)) ? deterministic_direction(index) : d * rsqrtf(dd);
    if (k.type == MR_SHAPE_SPHERE) {
        feat = feature_key(MR_SHAPE_SPHERE, 0u);
        return k.c + d * k.radius;
    }
    if (k.type == MR_SHAPE_CAPSULE) {
        const bool pos = dot3(d, k.e1 - k.e0) >= 0.0f;
        feat = feature_key(MR_SHAPE_CAPSULE, pos ? 1u : 0u);
        return (pos ? k.e1 : k.e0) + d * k.radius;
    }
    if (k.type == MR_SHAPE_BOX) {
        const float3 l = qrotinv(k.r, d);
        unsigned v = 0u;
        float3 p = f3(-k.half.x, -k.half.y, -k.half.z);
        if (l.x >= 0.0f) { v |= 1u; p.x = k.half.x; }
        if (l.y >= 0.0f) { v |= 2u; p.y = k.half.y; }
        if (l.z >= 0.0f) { v |= 4u; p.z = k.half.z; }
        feat = feature_key(MR_SHAPE_BOX, v);
        return k.c + qrot(k.r, p);
    }
    if (k.type == MR_SHAPE_CONVEX) {
        // The vertex of largest projection, the lowest index on a tie
        // (Collision.metal:1899-1936).
        const float3 l = qrotinv(k.r, d);
        float best = -INFINITY;
        int bi = 0;
        for (int i = 0; i < k.hull_count; ++i) {
            const float4 v = k.hull[i];
            const float pr = dot3(f3(v.x, v.y, v.z), l);
            if (pr > best) {
                best = pr;
                bi = i;
            }
        }
        feat = feature_key(MR_SHAPE_CONVEX, static_cast<unsigned>(bi));
        const float4 v = k.hull[bi];
        return k.c + qrot(k.r, f3(v.x, v.y, v.z));
    }
    // cylinder
    const float axial = dot3(d, k.axis);
    const float3 radial = d - k.axis * axial;
    const float rsq = dot3(radial, radial);
    const float3 rdir = rsq > kTinyS ? radial * rsqrtf(rsq) : k.bx;
    const bool pos = axial >= 0.0f;
    unsigned local = pos ? kCylPosRim : kCylNegRim;
    if (fabsf(axial) <= kCylAlign) {
        const float x = dot3(rdir, k.bx), z = dot3(rdir, k.bz);
        local = 32u + (fabsf(x) >= fabsf(z) ? (x >= 0.0f ? 0u : 1u) : (z >= 0.0f ? 2u : 3u));
    } else if (rsq <= kTinyS) {
        local = pos ? 17u : 16u;
    }
    feat = feature_key(MR_SHAPE_CYLINDER, local);
    return k.c + k.axis * (pos ? k.hl : -k.hl) + rdir * k.radius;
}

__device__ __forceinline__ void minkowski(const Collider& A, const Collider& B, unsigned ia, unsigned ib, float3 d, Sup& o) {
    o.pa = shape_support(A, ia, d, o.fa);
    o.pb = shape_support(B, ib, -d, o.fb);
    o.w = o.pa - o.pb;
}

// Closest point to the origin on triangle abc with barycentric weights
// (the Voronoi-region walk of Ericson, Real-Time Collision Detection 5.1.5).
__device__ float3 closest_triangle(float3 a, float3 b, float3 c, float* wt) {
    const float3 ab = b - a, ac = c - a, ap = -a;
    const float d1 = dot3(ab, ap), d2 = dot3(ac, ap);
    if (d1 <= 0.0f && d2 <= 0.0f) { wt[0] = 1.0f; wt[1] = 0.0f; wt[2] = 0.0f; return a; }
    const float3 bp = -b;
    const float d3 = dot3(ab, bp), d4 = dot3(ac, bp);
    if (d3 >= 0.0f && d4 <= d3) { wt[0] = 0.0f; wt[1] = 1.0f; wt[2] = 0.0f; return b; }
    const float vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) {
        const float den = d1 - d3, v = den > kTinyS ? d1 / den : 0.0f;
        wt[0] = 1.0f - v; wt[1] = v; wt[2] = 0.0f;
        return a + ab * v;
    }
    const float3 cp = -c;
    const float d5 = dot3(ab, cp), d6 = dot3(ac, cp);
    if (d6 >= 0.0f && d5 <= d6) { wt[0] = 0.0f; wt[1] = 0.0f; wt[2] = 1.0f; return c; }
    const float vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) {
        const float den = d2 - d6, w = den > kTinyS ? d2 / den : 0.0f;
        wt[0] = 1.0f - w; wt[1] = 0.0f; wt[2] = w;
        return a + ac * w;
    }
    const float va = d3 * d6 - d5 * d4;
    if (va <= 0.0f && (d4 - d3) >= 0.0f && (d5 - d6) >= 0.0f) {
        const float den = (d4 - d3) + (d5 - d6), w = den > kTinyS ? (d4 - d3) / den : 0.0f;
        wt[0] = 0.0f; wt[1] = 1.0f - w; wt[2] = w;
        return b + (c - b) * w;
    }
    const float den = va + vb + vc;
    if (!(fabsf(den) > kTinyS) || !isfinite(den)) { wt[0] = 1.0f; wt[1] = 0.0f; wt[2] = 0.0f; return a; }
    const float v = vb / den, w = vc / den;
    wt[0] = 1.0f - v - w; wt[1] = v; wt[2] = w;
    return a + ab * v + ac * w;
}

// a . (b x c) with error-free products and sums (the FMA two-product and
// Knuth's two-sum of Ogita, Rump and Oishi, "Accurate sum and dot product",
// 2005): the tetrahedron containment test of near-degenerate simplices.
__device__ __forceinline__ void two_sum(float a, float b, float& s, float& e) {
    s = a + b;
    const float bb = s - a;
    e = (a - (s - bb)) + (b - bb);
}
__device__ float accurate_triple(float3 a, float3 b, float3 c) {
    // cross components as (value, error) from two products each
    auto cross_comp = [](float p, float q, float r, float s, float& v, float& e) {
        const float x = p * q, ex = __fmaf_rn(p, q, -x);
        const float y = r * s, ey = __fmaf_rn(r, s, -y);
        float d, ed;
        two_sum(x, -y, d, ed);
        v = d;
        e = ed + (ex - ey);
    };
    float cx, ecx, cy, ecy, cz, ecz;
    cross_comp(b.y, c.z, b.z, c.y, cx, ecx);
    cross_comp(b.z, c.x, b.x, c.z, cy, ecy);
    cross_comp(b.x, c.y, b.y, c.x, cz, ecz);
    const float tx = a.x * cx, etx = __fmaf_rn(a.x, cx, -tx) + a.x * ecx;
    const float ty = a.y * cy, ety = __fmaf_rn(a.y, cy, -ty) + a.y * ecy;
    const float tz = a.z * cz, etz = __fmaf_rn(a.z, cz, -tz) + a.z * ecz;
    float s1, e1, s2, e2;
    two_sum(tx, ty, s1, e1);
    two_sum(s1, tz, s2, e2);
    return s2 + (e1 + e2 + etx + ety + etz);
}

__device__ void compress_simplex(Sup* sx, int& n, float* wt) {
    Sup keep[4];
    float kw[4];
    int m = 0, best = 0;
    for (int i = 1; i < n; ++i)
        if (wt[i] > wt[best]) best = i;
    for (int i = 0; i < n; ++i)
        if (wt[i] > 1.0e-7f) { keep[m] = sx[i]; kw[m] = wt[i]; ++m; }
    if (m == 0) { keep[0] = sx[best]; kw[0] = 1.0f; m = 1; }
    float tot = 0.0f;
    for (int i = 0; i < m; ++i) tot += kw[i];
    const float inv = tot > kTinyS ? 1.0f / tot : 1.0f;
    for (int i = 0; i < m; ++i) { sx[i] = keep[i]; wt[i] = kw[i] * inv; }
    n = m;
}

__device__ bool closest_simplex(Sup* sx, int& n, float* wt, float3& closest) {
    if (n == 1) { wt[0] = 1.0f; closest = sx[0].w; return false; }
    if (n == 2) {
        const float3 a = sx[0].w, e = sx[1].w - a;
        const float den = dot3(e, e);
        const float t = den > kTinyS ? fminf(fmaxf(-dot3(a, e) / den, 0.0f), 1.0f) : 0.0f;
        wt[0] = 1.0f - t;
        wt[1] = t;
        closest = a + e * t;
        compress_simplex(sx, n, wt);
        return false;
    }
    if (n == 3) {
        closest = closest_triangle(sx[0].w, sx[1].w, sx[2].w, wt);
        compress_simplex(sx, n, wt);
        return false;
    }
    const float3 a = sx[0].w, ab = sx[1].w - a, ac = sx[2].w - a, ad = sx[3].w - a;
    const float det = accurate_triple(ab, ac, ad);
    if (fabsf(det) > kTinyS && isfinite(det)) {
        const float inv = 1.0f / det;
        const float u = accurate_triple(-a, ac, ad) * inv, v = accurate_triple(ab, -a, ad) * inv,
                    w = accurate_triple(ab, ac, -a) * inv;
        const float base = 1.0f - u - v - w, tol = -2.0e-6f;
        if (base >= tol && u >= tol && v >= tol && w >= tol) {
            wt[0] = base; wt[1] = u; wt[2] = v; wt[3] = w;
            closest = f3(0.0f, 0.0f, 0.0f);
            return true;
        }
    }
    const int faces[4][3] = {{0, 1, 2}, {0, 3, 1}, {0, 2, 3}, {1, 3, 2}};
    float best = INFINITY, bw[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    float3 bp = f3(0.0f, 0.0f, 0.0f);
    for (int f = 0; f < 4; ++f) {
        float tw[3];
        const float3 p = closest_triangle(sx[faces[f][0]].w, sx[faces[f][1]].w, sx[faces[f][2]].w, tw);
        const float dist = dot3(p, p);
        if (dist < best) {
            best = dist;
            bp = p;
            bw[0] = bw[1] = bw[2] = bw[3] = 0.0f;
            for (int k = 0; k < 3; ++k) bw[faces[f][k]] = tw[k];
        }
    }
    closest = bp;
    for (int i = 0; i < 4; ++i) wt[i] = bw[i];
    compress_simplex(sx, n, wt);
    return false;
}

// GJK distance: returns 1 on overlap (the simplex seeds EPA), 0 apart (q
// holds the witness), -1 without convergence.
__device__ int gjk(const Collider& A, const Collider& B, unsigned ia, unsigned ib, float scale, Sup* sx, int& n, float* wt,
                   SmQuery& q) {
    const float tol = 32.0f * kFltEps * scale;
    float3 d = B.c - A.c;
    if (dot3(d, d) <= kTinyS) d = deterministic_direction(ia * 65537u + ib);
    n = 1;
    minkowski(A, B, ia, ib, d, sx[0]);
    wt[0] = 1.0f;
    float3 closest = sx[0].w;
    float prev = INFINITY;
    for (int it = 0; it < kGjkIterations; ++it) {
        if (dot3(closest, closest) <= tol * tol) return 1;
        d = -closest;
        Sup cand;
        minkowski(A, B, ia, ib, d, cand);
        bool dup = false;
        for (int i = 0; i < n; ++i) {
            const float3 e = cand.w - sx[i].w;
            dup = dup || dot3(e, e) <= tol * tol;
        }
        // Stop once the support advances less than tol along the UNIT
        // direction.  (The reference measures it along the unnormalised
        // direction, which below 1 m lets the reported distance exceed the
        // true one by tol / distance -- millimetres near contact, enough to
        // report a 0.7 mm capsule-box overlap as 1.6 mm apart.)
        const float advance = dot3(cand.w, d) - dot3(closest, d);
        bool done = dup || advance <= tol * len3(d);
        if (!done) {
            sx[n++] = cand;
            if (closest_simplex(sx, n, wt, closest)) return 1;
            const float upd = dot3(closest, closest);
            done = prev < INFINITY && prev - upd <= tol * tol;
            prev = upd;
        }
        if (done) {
            q.pa = q.pb = f3(0.0f, 0.0f, 0.0f);
            int best = 0;
            for (int i = 0; i < n; ++i) {
                q.pa = q.pa + sx[i].pa * wt[i];
                q.pb = q.pb + sx[i].pb * wt[i];
                if (wt[i] > wt[best]) best = i;
            }
            q.fa = sx[best].fa;
            q.fb = sx[best].fb;
            const float3 delta = q.pb - q.pa;
            const float dist = len3(delta);
            q.normal = dist > tol ? delta * (1.0f / dist) : d * rsqrtf(dot3(d, d));
            q.sep = dist;
            return 0;
        }
    }
    return -1;
}

struct EpaFace {
    int a, b, c, active;
    float3 n;
    float dist;
};

// Outward unit normal against `inside` (a point interior to the polytope)
// and the origin's distance to the face plane.
__device__ bool make_face(const Sup* vx, int a, int b, int c, float3 inside, EpaFace& f) {
    float3 n = cross3(vx[b].w - vx[a].w, vx[c].w - vx[a].w);
    const float nn = dot3(n, n);
    if (!(nn > kTinyS) || !isfinite(nn)) return false;
    n = n * rsqrtf(nn);
    int second = b, third = c;
    if (dot3(n, vx[a].w - inside) < 0.0f) { n = -n; second = c; third = b; }
    f.a = a; f.b = second; f.c = third; f.active = 1; f.n = n; f.dist = dot3(n, vx[a].w);
    return isfinite(f.dist);
}

__device__ __forceinline__ void horizon_edge(unsigned short* edges, int& ne, int a, int b) {
    const unsigned short fwd = static_cast<unsigned short>(a | (b << 8)), rev = static_cast<unsigned short>(b | (a << 8));
    for (int e = 0; e < ne; ++e)
        if (edges[e] == rev) {
            edges[e] = edges[--ne];
            return;
        }
    if (ne < 3 * kEpaFaces) edges[ne++] = fwd;
}

__device__ bool epa(const Collider& A, const Collider& B, unsigned ia, unsigned ib, float scale, const Sup* seed, int nseed,
                    SmQuery& q) {
    Sup vx[kEpaVertices];
    EpaFace fc[kEpaFaces];
    unsigned short edges[3 * kEpaFaces];
    int nv = nseed;
    for (int i = 0; i < nseed; ++i) vx[i] = seed[i];
    for (int k = 0; nv < 4 && k < 6; ++k) {
        const float s = k < 3 ? 1.0f : -1.0f;
        const int ax = k % 3;
        Sup cand;
        minkowski(A, B, ia, ib, f3(ax == 0 ? s : 0.0f, ax == 1 ? s : 0.0f, ax == 2 ? s : 0.0f), cand);
        bool dup = false;
        for (int i = 0; i < nv; ++i) {
            const float3 e = cand.w - vx[i].w;
            dup = dup || dot3(e, e) <= 1.0e-12f;
        }
        if (!dup) vx[nv++] = cand;
    }
    if (nv < 4) return false;
    for (int f = 0; f < kEpaFaces; ++f) fc[f].active = 0;
    const float3 inside = 0.25f * ((vx[0].w + vx[1].w) + (vx[2].w + vx[3].w));
    const int init[4][3] = {{0, 1, 2}, {0, 3, 1}, {0, 2, 3}, {1, 3, 2}};
    int nf = 0;
    for (int f = 0; f < 4; ++f)
        if (make_face(vx, init[f][0], init[f][1], init[f][2], inside, fc[nf])) ++nf;
    if (nf < 4) return false;
    const float tol = 64.0f * kFltEps * scale;
    for (int it = 0; it < kEpaIterations; ++it) {
        int best = -1;
        float bd = INFINITY;
        for (int f = 0; f < nf; ++f)
            if (fc[f].active && fc[f].dist < bd) { bd = fc[f].dist; best = f; }
        if (best < 0) return false;
        Sup cand;
        minkowski(A, B, ia, ib, fc[best].n, cand);
        const float sd = dot3(fc[best].n, cand.w);
        bool dup = false;
        for (int i = 0; i < nv; ++i) {
            const float3 e = cand.w - vx[i].w;
            dup = dup || dot3(e, e) <= tol * tol;
        }
        if (dup || sd - bd <= tol) {
            const EpaFace F = fc[best];
            float bc[3];
            closest_triangle(vx[F.a].w, vx[F.b].w, vx[F.c].w, bc);
            q.pa = vx[F.a].pa * bc[0] + vx[F.b].pa * bc[1] + vx[F.c].pa * bc[2];
            q.pb = vx[F.a].pb * bc[0] + vx[F.b].pb * bc[1] + vx[F.c].pb * bc[2];
            int fv = F.a;
            float fw = bc[0];
            if (bc[1] > fw) { fv = F.b; fw = bc[1]; }
            if (bc[2] > fw) fv = F.c;
            q.fa = vx[fv].fa;
            q.fb = vx[fv].fb;
            q.normal = F.n;
            q.sep = -bd;
            return finite3(q.pa) && finite3(q.pb) && finite3(q.normal) && isfinite(q.sep);
        }
        if (nv >= kEpaVertices) return false;
        const int nvx = nv++;
        vx[nvx] = cand;
        int ne = 0;
        for (int f = 0; f < nf; ++f) {
            if (!fc[f].active || dot3(fc[f].n, cand.w - vx[fc[f].a].w) <= tol) continue;
            horizon_edge(edges, ne, fc[f].a, fc[f].b);
            horizon_edge(edges, ne, fc[f].b, fc[f].c);
            horizon_edge(edges, ne, fc[f].c, fc[f].a);
            fc[f].active = 0;
        }
        if (ne == 0) return false;
        for (int e = 0; e < ne; ++e) {
            int dst = -1;
            for (int f = 0; f < nf; ++f)
                if (!fc[f].active) { dst = f; break; }
            if (dst < 0) {
                if (nf >= kEpaFaces) return false;
                dst = nf++;
            }
            if (!make_face(vx, edges[e] & 0xff, edges[e] >> 8, nvx, inside, fc[dst])) fc[dst].active = 0;
        }
    }
    return false;
}

__device__ bool mpr_witness(const Collider& A, const Collider& B, unsigned ia, unsigned ib, const Sup* portal, SmQuery& q) {
    float wt[3];
    const float3 closest = closest_triangle(portal[1].w, portal[2].w, portal[3].w, wt);
    q.pa = portal[1].pa * wt[0] + portal[2].pa * wt[1] + portal[3].pa * wt[2];
    q.pb = portal[1].pb * wt[0] + portal[2].pb * wt[1] + portal[3].pb * wt[2];
    int fv = 1;
    float fw = wt[0];
    if (wt[1] > fw) { fv = 2; fw = wt[1]; }
    if (wt[2] > fw) fv = 3;
    q.fa = portal[fv].fa;
    q.fb = portal[fv].fb;
    float3 d = closest;
    float dist = len3(d);
    const float3 centres = B.c - A.c;
    if (!(dist > kTinyS)) { d = centres; dist = len3(d); }
    d = !(dist > kTinyS) ? deterministic_direction(ia * 65537u + ib) : d * (1.0f / dist);
    if (dot3(d, centres) < 0.0f) d = -d;
    float sep = dot3(q.pb - q.pa, d);
    if (sep > 0.0f) { d = -d; sep = -sep; }
    q.normal = d;
    q.sep = fminf(sep, -0.0f);
    return finite3(q.pa) && finite3(q.pb) && finite3(q.normal) && isfinite(q.sep);
}

__device__ bool mpr(const Collider& A, const Collider& B, unsigned ia, unsigned ib, float scale, SmQuery& q) {
    Sup portal[4];
    portal[0].pa = A.c;
    portal[0].pb = B.c;
    portal[0].w = A.c - B.c;
    portal[0].fa = portal[0].fb = 0u;
    const float tol = 64.0f * kFltEps * scale;
    if (dot3(portal[0].w, portal[0].w) <= tol * tol) portal[0].w = portal[0].w + deterministic_direction(ia * 65537u + ib) * tol;
    float3 d = -portal[0].w;
    d = d * rsqrtf(dot3(d, d));
    minkowski(A, B, ia, ib, d, portal[1]);
    if (dot3(portal[1].w, d) < -tol) return false;
    d = cross3(portal[0].w, portal[1].w);
    float dd = dot3(d, d);
    if (!(dd > tol * tol)) { portal[2] = portal[3] = portal[1]; return mpr_witness(A, B, ia, ib, portal, q); }
    d = d * rsqrtf(dd);
    minkowski(A, B, ia, ib, d, portal[2]);
    if (dot3(portal[2].w, d) < -tol) return false;
    d = cross3(portal[1].w - portal[0].w, portal[2].w - portal[0].w);
    dd = dot3(d, d);
    if (!(dd > tol * tol)) { portal[3] = portal[2]; return mpr_witness(A, B, ia, ib, portal, q); }
    d = d * rsqrtf(dd);
    if (dot3(d, portal[0].w) > 0.0f) {
        const Sup t = portal[1];
        portal[1] = portal[2];
        portal[2] = t;
        d = -d;
    }
    bool found = false;
    for (int it = 0; it < kGjkIterations; ++it) {
        minkowski(A, B, ia, ib, d, portal[3]);
        if (dot3(portal[3].w, d) < -tol) return false;
        if (dot3(cross3(portal[1].w, portal[3].w), portal[0].w) < -tol) {
            portal[2] = portal[3];
        } else if (dot3(cross3(portal[3].w, portal[2].w), portal[0].w) < -tol) {
            portal[1] = portal[3];
        } else {
            found = true;
            break;
        }
        d = cross3(portal[1].w - portal[0].w, portal[2].w - portal[0].w);
        dd = dot3(d, d);
        if (!(dd > tol * tol)) { portal[3] = portal[2]; return mpr_witness(A, B, ia, ib, portal, q); }
        d = d * rsqrtf(dd);
    }
    if (!found) return false;
    for (int it = 0; it < kEpaIterations; ++it) {
        d = cross3(portal[2].w - portal[1].w, portal[3].w - portal[1].w);
        dd = dot3(d, d);
        if (!(dd > kTinyS) || !isfinite(dd)) return mpr_witness(A, B, ia, ib, portal, q);
        d = d * rsqrtf(dd);
        Sup cand;
        minkowski(A, B, ia, ib, d, cand);
        const float cp = dot3(cand.w, d);
        const float pp = fminf(dot3(portal[1].w, d), fminf(dot3(portal[2].w, d), dot3(portal[3].w, d)));
        if (cp - pp <= tol || it + 1 == kEpaIterations) return mpr_witness(A, B, ia, ib, portal, q);
        const float3 cc = cross3(cand.w, portal[0].w);
        if (dot3(portal[1].w, cc) > 0.0f) {
            if (dot3(portal[2].w, cc) > 0.0f) portal[1] = cand;
            else portal[3] = cand;
        } else if (dot3(portal[3].w, cc) > 0.0f) {
            portal[2] = cand;
        } else {
            portal[1] = cand;
        }
    }
    return false;
}

// Penetration witness of the hull path (Collision.metal:3129-3260, the
// reference's replacement for EPA when a hull is involved): among the
// centre-to-centre direction and the three local axes of each collider,
// oriented from A towards B, the axis of largest separation
// dot(support_B(-axis) - support_A(axis), axis).  (The reference also
// tries the previous substep's query normal; no query cache is kept here.)
__device__ bool support_axis_witness(const Collider& A, const Collider& B, unsigned ia, unsigned ib, SmQuery& q) {
    const float3 delta = B.c - A.c;
    bool found = false;
    auto update = [&](float3 axis) {
        const float a2 = dot3(axis, axis);
        if (!(a2 > kTinyS) || !isfinite(a2)) return true;
        axis = axis * rsqrtf(a2);
        if (dot3(delta, delta) > kTinyS && dot3(axis, delta) < 0.0f) axis = -axis;
        unsigned fa, fb;
        const float3 pa = shape_support(A, ia, axis, fa);
        const float3 pb = shape_support(B, ib, -axis, fb);
        const float sep = dot3(pb - pa, axis);
        if (!isfinite(sep)) return false;
        if (!found || sep > q.sep) {
            found = true;
            q.normal = axis;
            q.sep = sep;
            q.pa = pa;
            q.pb = pb;
            q.fa = fa;
            q.fb = fb;
        }
        return true;
    };
    if (!update(delta)) return false;
    for (int axis = 0; axis < 3; ++axis) {
        const float3 e = f3(axis == 0 ? 1.0f : 0.0f, axis == 1 ? 1.0f : 0.0f, axis == 2 ? 1.0f : 0.0f);
        if (!update(qrot(A.r, e)) || !update(qrot(B.r, e))) return false;
    }
    if (!found) return false;
    q.sep = fminf(q.sep, -0.0f);
    return finite3(q.pa) && finite3(q.pb) && finite3(q.normal) && isfinite(q.sep);
}

// Contacts of a support-mapped pair into `sink`; the pair's normal (A -> B)
// in `normal`.  Returns MR_STEP_SUCCESS or MR_STEP_DID_NOT_CONVERGE.
// Cylinder pairs resolve an overlap by EPA, then MPR (the primitive-GJK
// class); pairs with a hull by the support-axis witness (the hull class,
// Collision.metal:3623-3720), and a hull on the plane by its deepest vertex.
__device__ __noinline__ unsigned support_mapped_contacts(const Collider& A, const Collider& B, unsigned ia, unsigned ib, float accepted,
                                                         RawSink& sink, float3& normal) {
    if (B.type == MR_SHAPE_PLANE) {
        // The deepest vertex against the plane (the plane is always B here).
        unsigned f;
        const float3 p = shape_support(A, ia, -B.normal, f);
        const float sep = dot3(B.normal, p - B.c);
        normal = -B.normal;
        if (sep <= accepted) sink.add(p, p - B.normal * sep, sep, f, feature_key(MR_SHAPE_PLANE, 0u));
        return MR_STEP_SUCCESS;
    }
    const bool hull = A.type == MR_SHAPE_CONVEX || B.type == MR_SHAPE_CONVEX;
    const float scale = fmaxf(collider_scale(A), collider_scale(B)) + 1.0f;
    Sup sx[4];
    float wt[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    int n = 0;
    SmQuery q;
    q.normal = f3(0.0f, 0.0f, 1.0f);
    const int g = gjk(A, B, ia, ib, scale, sx, n, wt, q);
    if (hull) {
        if (g != 0 && !support_axis_witness(A, B, ia, ib, q)) return MR_STEP_DID_NOT_CONVERGE;
    } else if (g == 1) {
        // Primitive pairs resolve with EPA first, MPR second (Collision.metal:3518-3560).
        if (!epa(A, B, ia, ib, scale, sx, n, q) && !mpr(A, B, ia, ib, scale, q)) return MR_STEP_DID_NOT_CONVERGE;
    } else if (g < 0) {
        if (!mpr(A, B, ia, ib, scale, q)) return MR_STEP_DID_NOT_CONVERGE;
    }
    normal = q.normal;
    if (q.sep > accepted) return MR_STEP_SUCCESS;
    float3 wa[kRawCap], wb[kRawCap];
    int nw = 0;
    sink.add(q.pa, q.pb, q.sep, q.fa, q.fb);
    // Only cylinders and hulls have a contact patch; other support-mapped
    // pairs (a capsule against a box) keep the query's witness alone.
    const bool cyl_a = A.type == MR_SHAPE_CYLINDER, cyl_b = B.type == MR_SHAPE_CYLINDER;
    if (!cyl_a && !cyl_b && !hull) return MR_STEP_SUCCESS;
    wa[nw] = q.pa;
    wb[nw] = q.pb;
    ++nw;
    // Patch (Collision.metal:3327-3432): supports of the sampled shape -- a
    // cylinder, else a hull, A first -- along the normal tilted by 2e-4
    // towards the disk basis (cylinder cap contact), the axis (cylinder side
    // contact) or the contact plane's tangents (hull).
    const bool sample_a = cyl_a || (!cyl_b && A.type == MR_SHAPE_CONVEX);
    const Collider& k = sample_a ? A : B;
    const unsigned kidx = sample_a ? ia : ib;
    const float3 sn = sample_a ? q.normal : -q.normal;
    int nd = 0;
    float3 dirs[4];
    if (k.type == MR_SHAPE_CYLINDER) {
        const float align = fabsf(dot3(sn, k.axis));
        if (align >= 0.95f) {
            dirs[0] = k.bx; dirs[1] = -k.bx; dirs[2] = k.bz; dirs[3] = -k.bz;
            nd = 4;
        } else if (align <= 0.20f) {
            dirs[0] = k.axis; dirs[1] = -k.axis;
            nd = 2;
        }
    } else {
        // contactPatchTangent: the normal crossed with the world axis of its
        // smallest absolute component.
        const float3 an = f3(fabsf(q.normal.x), fabsf(q.normal.y), fabsf(q.normal.z));
        const float3 ref = an.x <= an.y && an.x <= an.z ? f3(1.0f, 0.0f, 0.0f) : (an.y <= an.z ? f3(0.0f, 1.0f, 0.0f) : f3(0.0f, 0.0f, 1.0f));
        float3 t = cross3(q.normal, ref);
        t = t * rsqrtf(dot3(t, t));
        const float3 bt = cross3(q.normal, t);
        dirs[0] = t; dirs[1] = -t; dirs[2] = bt; dirs[3] = -bt;
        nd = 4;
    }
    const float dtol = 32.0f * kFltEps * scale;
    for (int i = 0; i < nd; ++i) {
        unsigned f;
        const float3 p = shape_support(k, kidx, sn + dirs[i] * 2.0e-4f, f);
        const float3 pa = sample_a ? p : p - q.normal * q.sep;
        const float3 pb = sample_a ? p + q.normal * q.sep : p;
        bool dup = false;
        for (int j = 0; j < nw; ++j) {
            const float3 da = wa[j] - pa, db = wb[j] - pb;
            dup = dup || (dot3(da, da) <= dtol * dtol && dot3(db, db) <= dtol * dtol);
        }
        if (dup || nw >= kRawCap) continue;
        sink.add(pa, pb, q.sep, sample_a ? f : q.fa, sample_a ? q.fb : f);
        wa[nw] = pa;
        wb[nw] = pb;
        ++nw;
    }
    return MR_STEP_SUCCESS;
}

// Returns MR_STEP_SUCCESS, or the code of a support-mapped query that did
// not resolve.
template <bool kConvex>
__device__ unsigned narrowphase(const Collider& A, const Collider& B, int cls, unsigned ia, unsigned ib, float accepted,
                                RawSink& sink, float3& normal) {
    if constexpr (kConvex) {
        if (cls == MR_COLLISION_PAIR_CONVEX) return support_mapped_contacts(A, B, ia, ib, accepted, sink, normal);
    }
    if (cls == MR_COLLISION_PAIR_SPHERE_SPHERE) {
        const float3 delta = B.c - A.c;
        const float d = len3(delta);
        normal = d > kTinyS ? delta * (1.0f / d) : coincident_normal(ia, ib);
        const float sep = d - A.radius - B.radius;
        if (sep <= accepted)
            sink.add(A.c + normal * A.radius, B.c - normal * B.radius, sep, feature_key(MR_SHAPE_SPHERE, 0u),
                     feature_key(MR_SHAPE_SPHERE, 0u));
        return MR_STEP_SUCCESS;
    }
    if (cls == MR_COLLISION_PAIR_SPHERE_BOX) {
        const bool sphere_a = A.type == MR_SHAPE_SPHERE;
        const Collider& sp = sphere_a ? A : B;
        const Collider& bx = sphere_a ? B : A;
        const float3 lc = qrotinv(bx.r, sp.c - bx.c);
        float3 cl = f3(fminf(fmaxf(lc.x, -bx.half.x), bx.half.x), fminf(fmaxf(lc.y, -bx.half.y), bx.half.y),
                       fminf(fmaxf(lc.z, -bx.half.z), bx.half.z));
        const float3 ld = cl - lc;
        const float dist = len3(ld);
        float3 n;
        float sep;
        unsigned feat;
        if (dist > kTinyS) {
            n = qrot(bx.r, ld * (1.0f / dist));
            sep = dist - sp.radius;
            auto region = [](float c, float he) { return c < -he ? 0u : (c > he ? 2u : 1u); };
            feat = region(lc.x, bx.half.x) + 3u * region(lc.y, bx.half.y) + 9u * region(lc.z, bx.half.z);
        } else {
            const float dx = bx.half.x - fabsf(lc.x), dy = bx.half.y - fabsf(lc.y), dz = bx.half.z - fabsf(lc.z);
            int axis = 0;
            float dm = dx;
            if (dy < dm) { axis = 1; dm = dy; }
            if (dz < dm) { axis = 2; dm = dz; }
            const float coord = axis == 0 ? lc.x : (axis == 1 ? lc.y : lc.z);
            const float sign = coord >= 0.0f ? 1.0f : -1.0f;
            const float3 outward = f3(axis == 0 ? sign : 0.0f, axis == 1 ? sign : 0.0f, axis == 2 ? sign : 0.0f);
            if (axis == 0) cl.x = sign * bx.half.x;
            else if (axis == 1) cl.y = sign * bx.half.y;
            else cl.z = sign * bx.half.z;
            n = qrot(bx.r, -outward);
            sep = -dm - sp.radius;
            feat = 27u + 2u * static_cast<unsigned>(axis) + (sign > 0.0f ? 1u : 0u);
        }
        const float3 box_point = bx.c + qrot(bx.r, cl);
        if (sep <= accepted) {
            const float3 sphere_point = sp.c + n * sp.radius;
            if (sphere_a)
                sink.add(sphere_point, box_point, sep, feature_key(MR_SHAPE_SPHERE, 0u), feature_key(MR_SHAPE_BOX, feat));
            else
                sink.add(box_point, sphere_point, sep, feature_key(MR_SHAPE_BOX, feat), feature_key(MR_SHAPE_SPHERE, 0u));
        }
        normal = sphere_a ? n : -n;
        return MR_STEP_SUCCESS;
    }
    if (cls == MR_COLLISION_PAIR_SPHERE_CAPSULE) {
        const bool sphere_a = A.type == MR_SHAPE_SPHERE;
        const Collider& sp = sphere_a ? A : B;
        const Collider& cp = sphere_a ? B : A;
        float t;
        const float3 on = closest_on_segment(sp.c, cp.e0, cp.e1, t);
        const float3 delta = on - sp.c;
        const float d = len3(delta);
        const float3 n = d > kTinyS ? delta * (1.0f / d)
                                    : stable_segment_normal(cp.e1 - cp.e0, f3(0.0f, 0.0f, 0.0f), sphere_a ? ia : ib, sphere_a ? ib : ia);
        const float sep = d - sp.radius - cp.radius;
        if (sep <= accepted) {
            const float3 ps = sp.c + n * sp.radius, pc = on - n * cp.radius;
            const unsigned fs = feature_key(MR_SHAPE_SPHERE, 0u), fc = feature_key(MR_SHAPE_CAPSULE, capsule_feature(t));
            if (sphere_a) sink.add(ps, pc, sep, fs, fc);
            else sink.add(pc, ps, sep, fc, fs);
        }
        normal = sphere_a ? n : -n;
        return MR_STEP_SUCCESS;
    }
    if (cls == MR_COLLISION_PAIR_CAPSULE_CAPSULE) {
        float3 pa, pb;
        float ta, tb;
        closest_segments(A.e0, A.e1, B.e0, B.e1, pa, pb, ta, tb);
        const float3 delta = pb - pa;
        const float d = len3(delta);
        normal = d > kTinyS ? delta * (1.0f / d) : stable_segment_normal(A.e1 - A.e0, B.e1 - B.e0, ia, ib);
        const float sep = d - A.radius - B.radius;
        if (sep <= accepted)
            sink.add(pa + normal * A.radius, pb - normal * B.radius, sep, feature_key(MR_SHAPE_CAPSULE, capsule_feature(ta)),
                     feature_key(MR_SHAPE_CAPSULE, capsule_feature(tb)));
        return MR_STEP_SUCCESS;
    }
    if (cls == MR_COLLISION_PAIR_CAPSULE_BOX) {
        const bool capsule_a = A.type == MR_SHAPE_CAPSULE;
        const Collider& cp = capsule_a ? A : B;
        const Collider& bx = capsule_a ? B : A;
        const CapsuleBoxWitness w =
            capsule_box_witness(cp.e0, cp.e1, cp.radius, bx.c, bx.r, bx.half, capsule_a ? ia : ib, capsule_a ? ib : ia);
        if (w.sep <= accepted) {
            const unsigned fc = feature_key(MR_SHAPE_CAPSULE, capsule_feature(w.t_cap)), fb = feature_key(MR_SHAPE_BOX, w.box_feature);
            if (capsule_a) sink.add(w.cap_point, w.box_point, w.sep, fc, fb);
            else sink.add(w.box_point, w.cap_point, w.sep, fb, fc);
        }
        normal = capsule_a ? w.normal : -w.normal;
        return MR_STEP_SUCCESS;
    }
    if (cls == MR_COLLISION_PAIR_BOX_BOX) {
        const float3 cd = B.c - A.c;
        float best_sep = -INFINITY;
        float3 best_n = coincident_normal(ia, ib);
        int best_axis = 0;
        // Axes are numbered in the list of accepted axes: a skipped
        // (parallel-edge) cross axis shifts the later indices, and the
        // index names the face feature (128 + index).
        int index = -1;
        for (int k = 0; k < 15; ++k) {
            float3 axis;
            if (k < 3) axis = box_axis(A, k);
            else if (k < 6) axis = box_axis(B, k - 3);
            else {
                const float3 cr = cross3(box_axis(A, (k - 6) / 3), box_axis(B, (k - 6) % 3));
                const float sq = dot3(cr, cr);
                if (!(sq > kParallelEdges)) continue;
                axis = cr * rsqrtf(sq);
            }
            ++index;
            const float proj = dot3(cd, axis);
            if (proj < 0.0f || (proj == 0.0f && dot3(axis, best_n) < 0.0f)) axis = -axis;
            const float sep = fabsf(proj) - box_radius(A, axis) - box_radius(B, axis);
            if (sep > accepted) {
                normal = axis;
                return MR_STEP_SUCCESS;  // separated: no contact
            }
            const float tol = kAxisTie * (1.0f + fmaxf(fabsf(best_sep), fabsf(sep)));
            if (!isfinite(best_sep) || sep > best_sep + tol || (fabsf(sep - best_sep) <= tol && index < best_axis)) {
                best_sep = sep;
                best_n = axis;
                best_axis = index;
            }
        }
        normal = best_n;
        const float near_b = dot3(B.c, best_n) - box_radius(B, best_n);
        const float far_a = dot3(A.c, best_n) + box_radius(A, best_n);
        for (int v = 0; v < 8; ++v) {
            const float3 pa = box_vertex(A, v);
            if (!inside_inflated(pa, B, accepted)) continue;
            const float sep = near_b - dot3(pa, best_n);
            if (sep <= accepted)
                sink.add(pa, pa + best_n * sep, sep, feature_key(MR_SHAPE_BOX, static_cast<unsigned>(v)),
                         feature_key(MR_SHAPE_BOX, 128u + static_cast<unsigned>(best_axis)));
        }
        for (int v = 0; v < 8; ++v) {
            const float3 pb = box_vertex(B, v);
            if (!inside_inflated(pb, A, accepted)) continue;
            const float sep = dot3(pb, best_n) - far_a;
            if (sep <= accepted)
                sink.add(pb - best_n * sep, pb, sep, feature_key(MR_SHAPE_BOX, 128u + static_cast<unsigned>(best_axis)),
                         feature_key(MR_SHAPE_BOX, static_cast<unsigned>(v)));
        }
        if (sink.count == 0) {
            const float3 pa = box_support(A, best_n);
            const float3 pb = box_support(B, -best_n);
            sink.add(pa, pb, dot3(pb - pa, best_n), feature_key(MR_SHAPE_BOX, 256u + static_cast<unsigned>(best_axis)),
                     feature_key(MR_SHAPE_BOX, 256u + static_cast<unsigned>(best_axis)));
        }
        return MR_STEP_SUCCESS;
    }
    // Finite shape (A) against the plane (B).
    const float3 pn = B.normal;
    normal = -pn;
    const unsigned plane_key = feature_key(MR_SHAPE_PLANE, 0u);
    if (cls == MR_COLLISION_PAIR_SPHERE_PLANE) {
        const float3 surface = A.c - pn * A.radius;
        const float sep = dot3(pn, surface - B.c);
        if (sep <= accepted) sink.add(surface, surface - pn * sep, sep, feature_key(MR_SHAPE_SPHERE, 0u), plane_key);
        return MR_STEP_SUCCESS;
    }
    if (cls == MR_COLLISION_PAIR_CAPSULE_PLANE) {
        for (int e = 0; e < 2; ++e) {
            const float3 surface = (e == 0 ? A.e0 : A.e1) - pn * A.radius;
            const float sep = dot3(pn, surface - B.c);
            if (sep <= accepted)
                sink.add(surface, surface - pn * sep, sep, feature_key(MR_SHAPE_CAPSULE, static_cast<unsigned>(e)), plane_key);
        }
        return MR_STEP_SUCCESS;
    }
    if (cls == MR_COLLISION_PAIR_BOX_PLANE) {
        for (int v = 0; v < 8; ++v) {
            const float3 w = box_vertex(A, v);
            const float sep = dot3(pn, w - B.c);
            if (sep <= accepted) sink.add(w, w - pn * sep, sep, feature_key(MR_SHAPE_BOX, static_cast<unsigned>(v)), plane_key);
        }
        return MR_STEP_SUCCESS;
    }
    if (cls == MR_COLLISION_PAIR_CYLINDER_PLANE) {
        // Collision.metal:4627-4800: a cap face parallel to the plane gives
        // its four-point ring plus the exact rim support, a side parallel to
        // it the two rim ends, any other pose the one extremal rim point.
        const float axial = dot3(pn, A.axis), rx = dot3(pn, A.bx), rz = dot3(pn, A.bz);
        const float3 rproj = A.bx * rx + A.bz * rz;
        const float rsq = fmaxf(0.0f, rx * rx + rz * rz);
        auto add = [&](float3 surface, unsigned local) {
            const float sep = dot3(pn, surface - B.c);
            if (sep <= accepted) sink.add(surface, surface - pn * sep, sep, feature_key(MR_SHAPE_CYLINDER, local), plane_key);
        };
        if (rsq <= kCylAlign * kCylAlign) {
            const bool pos = axial < 0.0f;
            const float3 cap = A.c + A.axis * (pos ? A.hl : -A.hl);
            const unsigned base = pos ? kCylPosRing : kCylNegRing;
            add(cap + A.bx * A.radius, base + 0u);
            add(cap - A.bx * A.radius, base + 1u);
            add(cap + A.bz * A.radius, base + 2u);
            add(cap - A.bz * A.radius, base + 3u);
            if (rsq > 0.0f) add(cap - rproj * (A.radius * rsqrtf(rsq)), pos ? kCylPosRim : kCylNegRim);
            return MR_STEP_SUCCESS;
        }
        const float3 rdir = -rproj * rsqrtf(rsq);
        if (fabsf(axial) <= kCylAlign) {
            add(A.c - A.axis * A.hl + rdir * A.radius, kCylNegSide);
            add(A.c + A.axis * A.hl + rdir * A.radius, kCylPosSide);
            return MR_STEP_SUCCESS;
        }
        const bool pos = axial < 0.0f;
        add(A.c + A.axis * (pos ? A.hl : -A.hl) + rdir * A.radius, pos ? kCylPosRim : kCylNegRim);
        return MR_STEP_SUCCESS;
    }
    return MR_STEP_SUCCESS;
}

// Persistent manifold of one pair from its raw records and old slot
// (buildPersistentWorldManifold): break thresholds, feature-then-proximity
// matching, greedy reduction to four with the precision-independent tie
// rule (scores within a relative 1e-5 go to the smaller feature key), then
// canonical feature order.  `scratch` holds four old records ahead of the
// raw records, and 16 candidate-id bytes after them.  Returns the point
// count, or -1 when non-finite.
__device__ __forceinline__ unsigned long long rkey(const float* r) {
    return (static_cast<unsigned long long>(static_cast<unsigned>(ai(r[kCdFaS]))) << 32) | static_cast<unsigned>(ai(r[kCdFbS]));
}

__device__ int build_manifold(const SceneModel& M, const float* old_slot, int nraw, float3 raw_normal, float* scratch,
                              float* out, float3 posA, float4 rotA, float3 posB, float4 rotB) {
    const float* raw = scratch + 4 * kRecWords;
    unsigned char* ids = reinterpret_cast<unsigned char*>(scratch + (4 + kRawCap) * kRecWords);
    if (nraw == 0) {
        for (int k = 0; k < 56; ++k) out[k] = 0.0f;
        return 0;
    }
    for (int i = 0; i < nraw; ++i) {
        const float* r = raw + i * kRecWords;
        if (!isfinite(r[kCdSepS]) || !finite3(ld3(r + kCdWpS)) || !finite3(ld3(r + kCdLaS)) || !finite3(ld3(r + kCdLbS)))
            return -1;
    }
    const float3 nw = raw_normal * (1.0f / len3(raw_normal));
    if (!finite3(nw) || dot3(nw, nw) < 0.9999f) return -1;
    const float4 thr = make_float4(M.thresholds[0], M.thresholds[1], M.thresholds[2], M.thresholds[3]);
    int nc = 0;
    bool old_ok = false;
    float3 transported = f3(0.0f, 0.0f, 0.0f);
    float old_age = 0.0f;
    const int old_count = old_slot ? ai(old_slot[7]) : 0;
    if (old_count > 0 && old_count <= 4) {
        float3 on = qrot(rotA, ld3(old_slot));
        on = on * (1.0f / len3(on));
        old_ok = finite3(on) && dot3(on, nw) >= thr.w;
        if (old_ok) {
            const float3 ot = qrot(rotA, ld3(old_slot + 4));
            transported = ot - nw * dot3(ot, nw);
            old_age = old_slot[3];
            for (int i = 0; i < old_count; ++i) {
                const float* op = old_slot + 8 + i * 12;
                const float3 pa = posA + qrot(rotA, ld3(op));
                const float3 pb = posB + qrot(rotB, ld3(op + 3));
                const float3 delta = pb - pa;
                const float sep = dot3(delta, nw);
                const float3 tan = delta - nw * sep;
                if (sep > thr.x || len3(tan) > thr.y) continue;
                float* rec = scratch + i * kRecWords;
                for (int k = 0; k < 8; ++k) rec[k] = op[k];
                const unsigned life = static_cast<unsigned>(ai(op[8]));
                rec[kCdLifeS] = af(static_cast<int>(life == 0xffffffffu ? 0xffffffffu : life + 1u));
                rec[kCdImpS + 0] = op[9];
                rec[kCdImpS + 1] = op[10];
                rec[kCdImpS + 2] = op[11];
                st3(rec + kCdWpS, 0.5f * (pa + pb));
                rec[kCdSepS] = sep;
                ids[nc++] = static_cast<unsigned char>((i << 4) | i);
            }
        }
    }
    const float merge2 = thr.z * thr.z;
    for (int r = 0; r < nraw; ++r) {
        const float* rr = raw + r * kRecWords;
        const float3 la = ld3(rr + kCdLaS), lb = ld3(rr + kCdLbS);
        const int fa = ai(rr[kCdFaS]), fb = ai(rr[kCdFbS]);
        int match = -1;
        for (int k = 0; k < nc && match < 0; ++k) {
            const float* g = scratch + (ids[k] & 15u) * kRecWords;
            if (ai(g[kCdFaS]) == fa && ai(g[kCdFbS]) == fb) match = k;
        }
        for (int k = 0; k < nc && match < 0; ++k) {
            const float* g = scratch + (ids[k] & 15u) * kRecWords;
            const float3 da = ld3(g + kCdLaS) - la, db = ld3(g + kCdLbS) - lb;
            if (dot3(da, da) + dot3(db, db) <= 2.0f * merge2) match = k;
        }
        if (match < 0) {
            if (nc >= 4 + kRawCap) return -1;
            ids[nc++] = static_cast<unsigned char>((15u << 4) | (4u + r));
        } else {
            ids[match] = static_cast<unsigned char>((ids[match] & 0xf0u) | (4u + r));
        }
    }
    if (nc > 4) {
        for (int i = 1; i < nc; ++i) {
            const unsigned char val = ids[i];
            const float* gv = scratch + (val & 15u) * kRecWords;
            const float sv = gv[kCdSepS];
            const unsigned long long kv = rkey(gv);
            int d = i;
            while (d > 0) {
                const float* gp = scratch + (ids[d - 1] & 15u) * kRecWords;
                const float sp = gp[kCdSepS];
                if (!(sv < sp || (sv == sp && kv < rkey(gp)))) break;
                ids[d] = ids[d - 1];
                --d;
            }
            ids[d] = val;
        }
        unsigned selected = 1u;
        unsigned chosen = 0u;
        int chosen_count = 1;
        const float3 w0 = ld3(scratch + (ids[0] & 15u) * kRecWords + kCdWpS);
        float3 w1 = w0;
        for (int stage = 1; stage < 4; ++stage) {
            int best = -1;
            float best_score = -1.0f;
            unsigned long long best_f = ~0ull;
            for (int i = 0; i < nc; ++i) {
                if (selected & (1u << i)) continue;
                const float* gi = scratch + (ids[i] & 15u) * kRecWords;
                const float3 wi = ld3(gi + kCdWpS);
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
                        const float3 dl = wi - ld3(scratch + (ids[ck] & 15u) * kRecWords + kCdWpS);
                        const float3 t = dl - nw * dot3(dl, nw);
                        score = fminf(score, dot3(t, t));
                    }
                }
                const unsigned long long f = rkey(gi);
                const float tol = fmaxf(kTieAbs, kTieRel * fmaxf(fabsf(score), fabsf(best_score)));
                if (score > best_score + tol || (fabsf(score - best_score) <= tol && f < best_f)) {
                    best = i;
                    best_score = score;
                    best_f = f;
                }
            }
            if (best >= 0) {
                chosen |= static_cast<unsigned>(best) << (8 * chosen_count);
                ++chosen_count;
                selected |= 1u << best;
                if (stage == 1) w1 = ld3(scratch + (ids[best] & 15u) * kRecWords + kCdWpS);
            }
        }
        unsigned packed = 0u;
        for (int k = 0; k < chosen_count; ++k) packed |= static_cast<unsigned>(ids[(chosen >> (8 * k)) & 0xffu]) << (8 * k);
        for (int k = 0; k < chosen_count; ++k) ids[k] = static_cast<unsigned char>((packed >> (8 * k)) & 0xffu);
        nc = chosen_count;
    }
    for (int i = 1; i < nc; ++i) {
        const unsigned char val = ids[i];
        const unsigned long long f = rkey(scratch + (val & 15u) * kRecWords);
        int d = i;
        while (d > 0 && f < rkey(scratch + (ids[d - 1] & 15u) * kRecWords)) {
            ids[d] = ids[d - 1];
            --d;
        }
        ids[d] = val;
    }
    float3 tw = transported;
    if (!old_ok || !finite3(tw) || dot3(tw, tw) <= 1.0e-12f) tw = stable_tangent(nw);
    else tw = tw * (1.0f / len3(tw));
    st3(out, qrotinv(rotA, nw));
    out[3] = old_ok ? fminf(old_age + 1.0f, 65535.0f) : 0.0f;
    st3(out + 4, qrotinv(rotA, tw));
    out[7] = af(nc);
    for (int i = 0; i < 4; ++i) {
        float* op = out + 8 + i * 12;
        if (i < nc) {
            const unsigned id = ids[i];
            const float* g = scratch + (id & 15u) * kRecWords;
            for (int k = 0; k < 8; ++k) op[k] = g[k];
            if ((id >> 4) == 15u) {
                op[8] = af(0);
                op[9] = op[10] = op[11] = 0.0f;
            } else {
                const float* hrec = scratch + (id >> 4) * kRecWords;
                op[8] = hrec[kCdLifeS];
                op[9] = hrec[kCdImpS + 0];
                op[10] = hrec[kCdImpS + 1];
                op[11] = hrec[kCdImpS + 2];
            }
        } else {
            for (int k = 0; k < 12; ++k) op[k] = 0.0f;
        }
    }
    return nc;
}

// World inverse inertia R diag(inv) R^T, packed (xx, yx, yy, zx, zy, zz).
__device__ __forceinline__ void world_inv_inertia(float4 q, float4 inv, float* out) {
    const float3 c0 = qrot(q, f3(1.0f, 0.0f, 0.0f)), c1 = qrot(q, f3(0.0f, 1.0f, 0.0f)), c2 = qrot(q, f3(0.0f, 0.0f, 1.0f));
    const float R[3][3] = {{c0.x, c1.x, c2.x}, {c0.y, c1.y, c2.y}, {c0.z, c1.z, c2.z}};
    const float d[3] = {inv.x, inv.y, inv.z};
    int k = 0;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j <= i; ++j) {
            float acc = 0.0f;
            for (int m = 0; m < 3; ++m) acc = fmaf(R[i][m] * d[m], R[j][m], acc);
            out[k++] = acc;
        }
}
__device__ __forceinline__ float3 sym3_mul(const float* S, float3 x) {
    return f3(S[0] * x.x + S[1] * x.y + S[3] * x.z, S[1] * x.x + S[2] * x.y + S[4] * x.z, S[3] * x.x + S[4] * x.y + S[5] * x.z);
}

// FP64 audit of one environment's bodies (audit.cuh), read from its
// resident q [body][7] and v [body][6]; run by its own kernel after the
// control step.
__device__ void audit_scene(const SceneModel& M, const float* q, const float* v, double* rec, bool reset, int lane) {
    AuditSum a{};
    for (int b = lane; b < M.nb; b += 32) {
        const float4 ii = M.inv_inertia[b];
        const float3 id = f3(ii.x > 0.0f ? 1.0f / ii.x : 0.0f, ii.y > 0.0f ? 1.0f / ii.y : 0.0f, ii.z > 0.0f ? 1.0f / ii.z : 0.0f);
        audit_body(a, M.mass[b].x, ld3(q + b * 7), ld4(q + b * 7 + 3), ld3(v + b * 6), ld3(v + b * 6 + 3), id, f3(0.0f, 0.0f, 0.0f),
                   M.gravity);
    }
    audit_commit(a, rec, reset, lane);
}

// kComp: compensated sums for positions (across control steps, through
// p.q_comp) and for the velocity increments of the sweeps.  kConvex: the
// world has support-mapped (cylinder) pairs.
//
// One warp advances work item `item` of environment slot `env` by one
// control step, with `s` the warp's scene_step_smem_bytes() of shared
// memory.  Only warp-level synchronisation is used.
template <bool kComp, bool kConvex>
__device__ __forceinline__ void scene_step_item(const SceneParams& p, float* s, int item, int env) {
    const int lane = threadIdx.x & 31;
    const SceneModel& M = *p.model;
    if (p.world_tag != 0u && M.world_tag != p.world_tag) {
        // The record behind p.model is not the world this launch was
        // enqueued for: its body count need not match the caller's buffers,
        // so touch none of them.
        if (lane == 0) {
            if (p.status_codes) p.status_codes[item] = MR_STEP_UNSUPPORTED;
            if (p.active_contacts) p.active_contacts[item] = 0u;
            atomicAdd(p.stats + 0, 1u);
            atomicMin(p.stats + 6, static_cast<unsigned>(env));
            atomicAdd(p.stats + 9, 1u);
        }
        return;
    }
    const int nb = M.nb;
    const int nq = nb * 7, nv = nb * 6;
    float* misc = s + kOffMisc;
    const float h = M.h;
    if (lane < 32) misc[lane] = 0.0f;
    const bool reset = p.reset_masks != nullptr && p.reset_masks[item] != 0u;
    const float* srcq = (reset ? p.reset_q : p.q) + static_cast<size_t>(env) * nq;
    const float* srcv = (reset ? p.reset_v : p.v) + static_cast<size_t>(env) * nv;
    for (int b = lane; b < nb; b += 32) {
        st3(s + kOffPos + b * 3, ld3(srcq + b * 7));
        st4(s + kOffQuat + b * 4, ld4(srcq + b * 7 + 3));
        st3(s + kOffLin + b * 3, ld3(srcv + b * 6));
        st3(s + kOffAng + b * 3, ld3(srcv + b * 6 + 3));
        if (kComp) st3(s + kOffPosComp + b * 3, reset ? f3(0.0f, 0.0f, 0.0f) : ld3(p.q_comp + static_cast<size_t>(env) * nq + b * 7));
    }
    // Manifold table (sorted by pair key); a reset clears it.  Substeps
    // alternate between the two workspace tables; the environment's own
    // table is read by the first substep and written only on success.
    float* ws = p.workspace + static_cast<size_t>(env) * kWsWords;
    float* persistent = p.manifolds + static_cast<size_t>(env) * kTableWords;
    const float* cur_table = persistent;
    int mcount = reset ? 0 : static_cast<int>(p.manifold_count[env]);
    // Shared copies of the current table's pair keys (binary search) and of
    // the next one's, built as the narrowphase writes it.
    std::uint32_t* keys_cur = reinterpret_cast<std::uint32_t*>(s + kOffKeys);
    std::uint32_t* keys_next = keys_cur + kSceneManifolds;
    for (int i = lane; i < mcount; i += 32) keys_cur[i] = static_cast<std::uint32_t>(ai(persistent[i * kSceneSlotWords + 56]));
    const float friction_scale = p.friction_scale[env];
    __syncwarp();

    for (int sub = 0; sub < p.substeps; ++sub) {
        const bool final_substep = sub + 1 == p.substeps;
        // Prediction, world inverse inertia, swept bounds.
        for (int b = lane; b < nb; b += 32) {
            const float4 m = M.mass[b];
            float3 lin = ld3(s + kOffLin + b * 3), ang = ld3(s + kOffAng + b * 3);
            lin = expf(-h * m.z) * lin + h * f3(M.gravity[0], M.gravity[1], M.gravity[2]);
            ang = expf(-h * m.w) * ang;
            if (!finite3(lin) || !finite3(ang)) fail(misc, MR_STEP_NONFINITE_RESULT, static_cast<unsigned>(b));
            st3(s + kOffLin + b * 3, lin);
            st3(s + kOffAng + b * 3, ang);
            float4 q = ld4(s + kOffQuat + b * 4);
            float4 qn;
            if (!qnormalize(q, qn, true)) {
                fail(misc, MR_STEP_NONFINITE_INPUT, static_cast<unsigned>(b));
                qn = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
            }
            const float3 c = ld3(s + kOffPos + b * 3);
            if (!finite3(c)) fail(misc, MR_STEP_NONFINITE_INPUT, static_cast<unsigned>(b));
            world_inv_inertia(qn, M.inv_inertia[b], s + kOffIiw + b * 6);
            // Speculative sweep over the substep (Collision.metal:5960-6030).
            const float4 off = M.offsets[b];
            const float3 fc = c + h * lin;
            float4 fr = qmul(so3_increment(h * ang, false), qn);
            fr = qscale(fr, rsqrtf(qdot(fr, fr)));
            // Chord of the sweep sphere: the reference's 2 r sqrt(1 - cos^2)
            // with cos = |q . q_next| is 2 r |sin(h |w| / 2)|; written so,
            // FP32 has no cancellation near rest (1 - cos^2 of a resting body
            // would otherwise carry a spurious ~1e-4 m margin).
            const float chord = 2.0f * off.z * fabsf(sinf(0.5f * h * len3(ang)));
            const float envelope = fminf(len3(fc - c) + chord, h * M.speed_envelope);
            const float margin = M.speculative_scale * envelope;
            s[kOffMargin + b] = margin;
            const float4 dm = M.dims[b];
            float3 e0, e1;
            if (M.shape_type[b] == MR_SHAPE_SPHERE) {
                e0 = e1 = f3(dm.x, dm.x, dm.x);
            } else if (M.shape_type[b] == MR_SHAPE_CAPSULE) {
                const float3 a0 = qrot(qn, f3(0.0f, dm.y, 0.0f)), a1 = qrot(fr, f3(0.0f, dm.y, 0.0f));
                e0 = f3(fabsf(a0.x) + dm.x, fabsf(a0.y) + dm.x, fabsf(a0.z) + dm.x);
                e1 = f3(fabsf(a1.x) + dm.x, fabsf(a1.y) + dm.x, fabsf(a1.z) + dm.x);
            } else if (M.shape_type[b] == MR_SHAPE_CYLINDER) {
                // Collision.cpp:719-740: per component |a_i| hl + sqrt(1 - a_i^2) r.
                auto ext = [&](float4 r) {
                    const float3 a = qrot(r, f3(0.0f, 1.0f, 0.0f));
                    return f3(fabsf(a.x) * dm.y + sqrtf(fmaxf(0.0f, 1.0f - a.x * a.x)) * dm.x,
                              fabsf(a.y) * dm.y + sqrtf(fmaxf(0.0f, 1.0f - a.y * a.y)) * dm.x,
                              fabsf(a.z) * dm.y + sqrtf(fmaxf(0.0f, 1.0f - a.z * a.z)) * dm.x);
                };
                e0 = ext(qn);
                e1 = ext(fr);
            } else {
                auto ext = [&](float4 r) {
                    const float3 bx = qrot(r, f3(1.0f, 0.0f, 0.0f)), by = qrot(r, f3(0.0f, 1.0f, 0.0f)), bz = qrot(r, f3(0.0f, 0.0f, 1.0f));
                    return f3(fabsf(bx.x), fabsf(bx.y), fabsf(bx.z)) * dm.x + f3(fabsf(by.x), fabsf(by.y), fabsf(by.z)) * dm.y +
                           f3(fabsf(bz.x), fabsf(bz.y), fabsf(bz.z)) * dm.z;
                };
                e0 = ext(qn);
                e1 = ext(fr);
            }
            const float3 oo = f3(off.x, off.x, off.x);
            float3 lo = f3(fminf(c.x - e0.x, fc.x - e1.x), fminf(c.y - e0.y, fc.y - e1.y), fminf(c.z - e0.z, fc.z - e1.z)) - oo;
            float3 hi = f3(fmaxf(c.x + e0.x, fc.x + e1.x), fmaxf(c.y + e0.y, fc.y + e1.y), fmaxf(c.z + e0.z, fc.z + e1.z)) + oo;
            const float3 sc = f3(fmaxf(fabsf(lo.x), fabsf(hi.x)) + 1.0f, fmaxf(fabsf(lo.y), fabsf(hi.y)) + 1.0f,
                                 fmaxf(fabsf(lo.z), fabsf(hi.z)) + 1.0f);
            lo = lo - sc * kAabbPadS - f3(margin, margin, margin);
            hi = hi + sc * kAabbPadS + f3(margin, margin, margin);
            st3(s + kOffLo + b * 3, lo);
            st3(s + kOffHi + b * 3, hi);
            st4(s + kOffQuat + b * 4, qn);
        }
        if (!ok(misc)) break;

        // Pair flags over the compiled list, compacted in pair order.
        std::uint16_t* cand = reinterpret_cast<std::uint16_t*>(s + kOffCand);
        int ncand = 0;
        bool overflow = false;
        for (int base = 0; base < M.np; base += 32) {
            const int pi = base + lane;
            bool flag = false;
            if (pi < M.np) {
                const int a = M.pair_a[pi], b = M.pair_b[pi];
                const float3 la = ld3(s + kOffLo + a * 3), ha = ld3(s + kOffHi + a * 3);
                if (b >= nb) {
                    const float3 pn = qrot(M.plane_rotation, f3(0.0f, 1.0f, 0.0f));
                    const float3 n = pn * rsqrtf(dot3(pn, pn));
                    const float3 center = 0.5f * (la + ha), halfx = 0.5f * (ha - la);
                    const float off = M.offsets[a].x + s[kOffMargin + a];
                    const float scale = fmaxf(fmaxf(maxabs3(xyz(M.plane_position)), maxabs3(la)),
                                              fmaxf(maxabs3(ha), fmaxf(fabsf(M.plane_offsets.x), fabsf(off))));
                    const float3 an = f3(fabsf(n.x), fabsf(n.y), fabsf(n.z));
                    flag = dot3(n, center - xyz(M.plane_position)) - dot3(an, halfx) <= M.plane_offsets.x + (scale + 1.0f) * kQueryPadS;
                } else {
                    const float3 lb = ld3(s + kOffLo + b * 3), hb = ld3(s + kOffHi + b * 3);
                    flag = la.x <= hb.x && lb.x <= ha.x && la.y <= hb.y && lb.y <= ha.y && la.z <= hb.z && lb.z <= ha.z;
                }
            }
            const unsigned m = __ballot_sync(0xffffffffu, flag);
            const int at = ncand + __popc(m & ((1u << lane) - 1u));
            if (flag) {
                if (at < kSceneCandidates) cand[at] = static_cast<std::uint16_t>(pi);
                else overflow = true;
            }
            ncand += __popc(m);
        }
        if (__any_sync(0xffffffffu, overflow)) {
            if (lane == 0) fail(misc, MR_STEP_PAIR_CAPACITY_OVERFLOW, static_cast<unsigned>(ncand));
            __syncwarp();
            break;
        }
        if (lane == 0) misc[kSmCand] = af(max(ai(misc[kSmCand]), ncand));
        __syncwarp();

        // Narrowphase + manifolds, 32 candidates at a time.  A pair with raw
        // contacts always yields a manifold, so its table position is known
        // before the manifold is built, and it is built in place.
        const float* old_table = cur_table;
        float* new_table = ws + ((sub & 1) ? kWsTable1 : kWsTable0);
        float* scratch = ws + kWsLanes + lane * kLaneScratch;
        int ncount = 0, raw_total = 0;
        bool bad = false, mover = false, unresolved = false;
        for (int base = 0; base < ncand; base += 32) {
            const int ci = base + lane;
            int nraw = 0;
            unsigned key = 0u;
            const float* old_slot = nullptr;
            float3 normal = f3(0.0f, 0.0f, 1.0f);
            float3 posA = f3(0.0f, 0.0f, 0.0f), posB = posA;
            float4 rotA = make_float4(0.0f, 0.0f, 0.0f, 1.0f), rotB = rotA;
            if (ci < ncand) {
                const int pi = cand[ci];
                const int a = M.pair_a[pi], b = M.pair_b[pi];
                key = static_cast<unsigned>(a * (kSceneMaxBodies + 1) + b);
                // Old manifold of this pair (keys ascending).
                int lo_i = 0, hi_i = mcount - 1;
                while (lo_i <= hi_i) {
                    const int mid = (lo_i + hi_i) >> 1;
                    const unsigned mk = keys_cur[mid];
                    if (mk == key) { old_slot = old_table + mid * kSceneSlotWords; break; }
                    if (mk < key) lo_i = mid + 1;
                    else hi_i = mid - 1;
                }
                Collider A, B;
                load_collider(M, s, a, A);
                load_collider(M, s, b, B);
                const float accepted = A.offset + B.offset + (fmaxf(collider_scale(A), collider_scale(B)) + 1.0f) * kQueryPadS;
                RawSink sink{scratch + 4 * kRecWords, 0, A.bpos, B.bpos, A.brot, B.brot};
                if (narrowphase<kConvex>(A, B, M.pair_class[pi], static_cast<unsigned>(a), static_cast<unsigned>(b), accepted, sink,
                                         normal) != MR_STEP_SUCCESS)
                    unresolved = true;
                nraw = sink.count;
                posA = A.bpos;
                rotA = A.brot;
                posB = B.bpos;
                rotB = B.brot;
            }
            raw_total += nraw;
            const unsigned m = __ballot_sync(0xffffffffu, nraw > 0);
            const int at = ncount + __popc(m & ((1u << lane) - 1u));
            if (nraw > 0) {
                if (at < kSceneManifolds) {
                    float* dst = new_table + at * kSceneSlotWords;
                    if (build_manifold(M, old_slot, nraw, normal, scratch, dst, posA, rotA, posB, rotB) <= 0) bad = true;
                    dst[56] = af(static_cast<int>(key));
                    keys_next[at] = key;
                } else {
                    mover = true;
                }
            }
            ncount += __popc(m);
        }
        raw_total = __reduce_add_sync(0xffffffffu, raw_total);
        if (__any_sync(0xffffffffu, unresolved)) {
            if (lane == 0) fail(misc, MR_STEP_DID_NOT_CONVERGE, 0u);
            __syncwarp();
            break;
        }
        if (__any_sync(0xffffffffu, bad)) {
            if (lane == 0) fail(misc, MR_STEP_NONFINITE_RESULT, 0u);
            __syncwarp();
            break;
        }
        if (__any_sync(0xffffffffu, mover)) {
            if (lane == 0) fail(misc, MR_STEP_MANIFOLD_CAPACITY_OVERFLOW, static_cast<unsigned>(ncount));
            __syncwarp();
            break;
        }
        __syncwarp();
        cur_table = new_table;
        mcount = ncount;
        float* tab = new_table;
        {
            std::uint32_t* t = keys_cur;
            keys_cur = keys_next;
            keys_next = t;
        }
        if (lane == 0) {
            misc[kSmManifolds] = af(max(ai(misc[kSmManifolds]), mcount));
            misc[kSmRaw] = af(max(ai(misc[kSmRaw]), raw_total));
        }
        __syncwarp();

        // Contact records in manifold order (lane per manifold).
        float* C = ws + kWsContacts;
        std::uint16_t* mfirst = reinterpret_cast<std::uint16_t*>(s + kOffFirst);
        int total = 0;
        for (int base = 0; base < mcount; base += 32) {
            const int mi = base + lane;
            const int cnt = mi < mcount ? ai(tab[mi * kSceneSlotWords + 7]) : 0;
            int incl = cnt;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += t;
            }
            const int first = total + incl - cnt;
            total += __shfl_sync(0xffffffffu, incl, 31);
            if (mi < mcount) mfirst[mi] = static_cast<std::uint16_t>(min(first, kSceneContacts));
            if (cnt > 0 && first + cnt <= kSceneContacts) {
                const float* slot = tab + mi * kSceneSlotWords;
                const unsigned key = static_cast<unsigned>(ai(slot[56]));
                const int a = static_cast<int>(key / (kSceneMaxBodies + 1)), b = static_cast<int>(key % (kSceneMaxBodies + 1));
                const bool plane_b = b >= nb;
                const float3 posA = ld3(s + kOffPos + a * 3);
                const float4 rotA = ld4(s + kOffQuat + a * 4);
                const float3 posB = plane_b ? xyz(M.ground_position) : ld3(s + kOffPos + b * 3);
                const float4 rotB = plane_b ? M.ground_rotation : ld4(s + kOffQuat + b * 4);
                float3 nw = qrot(rotA, ld3(slot));
                nw = nw * (1.0f / len3(nw));
                float3 tw = qrot(rotA, ld3(slot + 4));
                tw = tw - nw * dot3(tw, nw);
                tw = dot3(tw, tw) > 1.0e-12f ? tw * (1.0f / len3(tw)) : stable_tangent(nw);
                const float3 bw = cross3(nw, tw);
                const int ma = M.material[a], mb = plane_b ? M.plane_material : M.material[b];
                const float4 fa = M.material_friction[ma], fb = M.material_friction[mb];
                const float mu_s = sqrtf(fmaxf(0.0f, fa.x * fb.x)) * friction_scale;
                const float mu_d = sqrtf(fmaxf(0.0f, fa.y * fb.y)) * friction_scale;
                const float4 ra = M.material_response[ma], rb = M.material_response[mb];
                const float rest = M.offsets[a].y + (plane_b ? M.plane_offsets.y : M.offsets[b].y);
                for (int i = 0; i < cnt; ++i) {
                    const float* op = slot + 8 + i * 12;
                    const Rec c = rec(C, first + i);
                    const float3 pa = posA + qrot(rotA, ld3(op));
                    const float3 pb = posB + qrot(rotB, ld3(op + 3));
                    const float3 pw = 0.5f * (pa + pb);
                    const float sep = dot3(pb - pa, nw) - rest;
                    c[kScA] = af(a);
                    c[kScB] = af(plane_b ? -1 : b);
                    c.set3(kScRa, pw - posA);
                    c.set3(kScRb, pw - posB);
                    c.set3(kScN, nw);
                    c.set3(kScT, tw);
                    c.set3(kScBt, bw);
                    const bool new_impact = static_cast<unsigned>(ai(op[8])) == 0u;
                    c[kScFlags] = af(new_impact ? 1 : 0);
                    c[kScSlot] = af(mi * 4 + i);
                    c[kScLambda + 0] = op[9];
                    c[kScLambda + 1] = op[10];
                    c[kScLambda + 2] = op[11];
                    c[kScTarget + 0] = sep > 0.0f ? -sep / h : 0.0f;
                    c[kScTarget + 1] = 0.0f;
                    c[kScTarget + 2] = 0.0f;
                    c[kScReg] = fmaxf((ra.z + rb.z) / (h * h) + (ra.w + rb.w) / h, 0.0f);
                    c[kScMu] = mu_s;
                    c[kScRelax] = fminf(fmaxf(fmaxf(ra.x, rb.x), 0.0f), 1.0f);  // restitution until evaluated
                    c[kScDelta + 0] = fmaxf(ra.y, rb.y);                          // restitution threshold
                    c[kScDelta + 1] = mu_d;
                    c[kScDelta + 2] = sep;
                }
            }
        }
        if (total > kSceneContacts) {
            if (lane == 0) fail(misc, MR_STEP_CONTACT_CAPACITY_OVERFLOW, static_cast<unsigned>(total));
            __syncwarp();
            break;
        }
        if (lane == 0) {
            misc[kSmContacts] = af(total);
            mfirst[mcount] = static_cast<std::uint16_t>(total);
        }
        __syncwarp();

        // Per-body contact lists (ascending contact index; side bit 1 = B),
        // walked manifold by manifold: a manifold's contacts are contiguous.
        int* start = reinterpret_cast<int*>(s + kOffLists);
        int* fill = start + kSceneMaxBodies + 1;
        std::uint16_t* entries = reinterpret_cast<std::uint16_t*>(s + kOffEntries);
        for (int b = lane; b < nb; b += 32) {
            int cnt = 0;
            for (int mi = 0; mi < mcount; ++mi) {
                const unsigned k = keys_cur[mi];
                if (static_cast<int>(k / (kSceneMaxBodies + 1)) == b || static_cast<int>(k % (kSceneMaxBodies + 1)) == b)
                    cnt += mfirst[mi + 1] - mfirst[mi];
            }
            fill[b] = cnt;
        }
        __syncwarp();
        if (lane == 0) {
            int acc = 0;
            for (int b = 0; b < nb; ++b) { start[b] = acc; acc += fill[b]; }
            start[nb] = acc;
        }
        __syncwarp();
        for (int b = lane; b < nb; b += 32) {
            int at = start[b];
            for (int mi = 0; mi < mcount; ++mi) {
                const unsigned k = keys_cur[mi];
                const int side = static_cast<int>(k / (kSceneMaxBodies + 1)) == b ? 0
                                 : (static_cast<int>(k % (kSceneMaxBodies + 1)) == b ? 1 : -1);
                if (side < 0) continue;
                for (int c = mfirst[mi]; c < mfirst[mi + 1]; ++c) entries[at++] = static_cast<std::uint16_t>((c << 1) | side);
            }
        }
        __syncwarp();

        // ConstraintIR evaluation at the predicted velocities, blocks,
        // preconditioners, relaxation and warm start (lane per contact).
        auto point_velocity = [&](int body, float3 r) {
            if (body < 0) return f3(0.0f, 0.0f, 0.0f);
            return ld3(s + kOffLin + body * 3) + cross3(ld3(s + kOffAng + body * 3), r);
        };
        for (int c = lane; c < total; c += 32) {
            const Rec cr = rec(C, c);
            const int a = ai(cr[kScA]), b = ai(cr[kScB]);
            const float3 ra = cr.v3(kScRa), rb = cr.v3(kScRb);
            const float3 dv = point_velocity(b, rb) - point_velocity(a, ra);
            const float3 dirs[3] = {cr.v3(kScN), cr.v3(kScT), cr.v3(kScBt)};
            const float rel[3] = {dot3(dv, dirs[0]), dot3(dv, dirs[1]), dot3(dv, dirs[2])};
            const float sep = cr[kScDelta + 2];
            const float tau_c = 2.0f * h;
            const float err = fminf(sep + M.slop, 0.0f);
            const float ratio = h / tau_c;
            float stab = -h * err / (tau_c * tau_c * (1.0f + 2.0f * ratio + ratio * ratio));
            stab = fminf(fmaxf(stab, 0.0f), M.max_depenetration);
            if (ai(cr[kScFlags]) & 1) {
                const float incoming = rel[0] - cr[kScTarget + 0];
                if (incoming < -cr[kScDelta + 0]) stab = fmaxf(stab, -cr[kScRelax] * incoming);
            }
            cr[kScTarget + 0] += stab;
            const float slip = sqrtf(rel[1] * rel[1] + rel[2] * rel[2]);
            if (!(slip <= 1.0e-3f)) cr[kScMu] = cr[kScDelta + 1];
            // W = sum over dynamic sides of m^-1 d_i.d_j + (r x d_i)^T I^-1 (r x d_j).
            float W[3][3];
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) W[i][j] = 0.0f;
            for (int side = 0; side < 2; ++side) {
                const int body = side ? b : a;
                if (body < 0) continue;
                const float3 r = side ? rb : ra;
                const float im = M.mass[body].y;
                const float* S = s + kOffIiw + body * 6;
                float3 rd[3], ird[3];
                for (int i = 0; i < 3; ++i) { rd[i] = cross3(r, dirs[i]); ird[i] = sym3_mul(S, rd[i]); }
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j) W[i][j] += im * dot3(dirs[i], dirs[j]) + dot3(rd[i], ird[j]);
            }
            // Row sum of normal couplings over contacts sharing a body.
            float rowsum = 0.0f;
            const float3 n_i = dirs[0];
            for (int side = 0; side < 2; ++side) {
                const int body = side ? b : a;
                if (body < 0) continue;
                for (int k = start[body]; k < start[body + 1]; ++k) {
                    const int cj = entries[k] >> 1, sj = entries[k] & 1;
                    const Rec crj = rec(C, cj);
                    const int oa = ai(crj[kScA]), ob = ai(crj[kScB]);
                    // Skip on the second body when the first one already counted j.
                    if (side == 1 && (oa == a || ob == a) && a >= 0) continue;
                    float w = 0.0f;
                    for (int t = 0; t < 2; ++t) {
                        const int bi = t ? b : a;
                        if (bi < 0) continue;
                        const int tj = (oa == bi) ? 0 : ((ob == bi) ? 1 : -1);
                        if (tj < 0) continue;
                        const float si = t ? 1.0f : -1.0f, sjn = tj ? 1.0f : -1.0f;
                        const float3 ri = t ? rb : ra, rj = crj.v3(tj ? kScRb : kScRa);
                        const float3 n_j = crj.v3(kScN);
                        const float3 rni = cross3(ri, n_i), rnj = cross3(rj, n_j);
                        w += si * sjn * (M.mass[bi].y * dot3(n_i, n_j) + dot3(rni, sym3_mul(s + kOffIiw + bi * 6, rnj)));
                    }
                    (void)sj;
                    rowsum += fabsf(w);
                }
            }
            const float reg[3] = {cr[kScReg], 0.0f, 0.0f};
            const float diag = fabsf(W[0][0]) + reg[0];
            for (int i = 0; i < 3; ++i) W[i][i] += reg[i];
            float inv[3][3];
            if (!invert3x3_reg(W, inv)) {
                fail(misc, MR_STEP_FACTORIZATION_FAILED, static_cast<unsigned>(c));
            } else {
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j) cr[kScPre + i * 3 + j] = inv[i][j];
            }
            cr[kScRelax] = rowsum > fmaxf(diag, kMatrixFloor) ? fminf(fmaxf(diag / rowsum, 1.0f / 32.0f), 1.0f) : 1.0f;
            const float3 warm = project_cone(cr.v3(kScLambda), cr[kScMu], cr[kScMu]);
            cr.set3(kScLambda, warm);
            cr.set3(kScDelta, warm);
            if (!isfinite(cr[kScTarget])) fail(misc, MR_STEP_NONFINITE_RESULT, static_cast<unsigned>(c));
        }
        if (!ok(misc)) break;
        // Islands: min-root union find over dynamic bodies joined by contacts.
        // The solve treats all contacts of an environment together (islands
        // do not interact in a Jacobi sweep), so islands are a diagnostic
        // here, counted on the final substep.
        if (lane == 0 && total > 0 && final_substep) {
            int* parent = reinterpret_cast<int*>(keys_next);  // the previous table's keys are dead by now
            for (int b = 0; b < nb; ++b) parent[b] = b;
            auto root = [&](int x) { while (parent[x] != x) x = parent[x] = parent[parent[x]]; return x; };
            unsigned touched[2] = {0u, 0u};
            for (int c = 0; c < total; ++c) {
                const int a = ai(rec(C, c)[kScA]), b = ai(rec(C, c)[kScB]);
                touched[a >> 5] |= 1u << (a & 31);
                if (b >= 0) {
                    touched[b >> 5] |= 1u << (b & 31);
                    const int x = root(a), y = root(b);
                    if (x != y) parent[max(x, y)] = min(x, y);
                }
            }
            int islands = 0;
            std::uint8_t* labels = p.island_labels ? p.island_labels + static_cast<size_t>(env) * kSceneMaxBodies : nullptr;
            for (int b = 0; b < nb; ++b) {
                // A root precedes every member of its set, so its island
                // index is known before any member asks for it.
                const int r = root(b);
                const bool island_root = ((touched[b >> 5] >> (b & 31)) & 1u) && r == b;
                if (labels) labels[b] = island_root ? static_cast<std::uint8_t>(islands) : (r == b ? 0xffu : labels[r]);
                if (island_root) ++islands;
            }
            misc[kSmIslands] = af(max(ai(misc[kSmIslands]), islands));
        } else if (lane == 0 && final_substep && p.island_labels) {
            for (int b = 0; b < nb; ++b) p.island_labels[static_cast<size_t>(env) * kSceneMaxBodies + b] = 0xffu;
        }
        __syncwarp();
        // Jacobi sweeps (sweep -1 applies the warm start).
        if (kComp) {
            for (int i = lane; i < nb * 3; i += 32) {
                s[kOffLinComp + i] = 0.0f;
                s[kOffAngComp + i] = 0.0f;
            }
        }
        const int iters = p.velocity_iterations + (final_substep ? p.final_velocity_iterations : 0);
        for (int it = -1; it < iters; ++it) {
            if (it >= 0) {
                for (int c = lane; c < total; c += 32) {
                    const Rec cr = rec(C, c);
                    const int a = ai(cr[kScA]), b = ai(cr[kScB]);
                    const float3 dv = point_velocity(b, cr.v3(kScRb)) - point_velocity(a, cr.v3(kScRa));
                    const float3 prev = cr.v3(kScLambda);
                    const float r0 = cr[kScTarget + 0] - dot3(dv, cr.v3(kScN)) - cr[kScReg] * prev.x;
                    const float r1 = cr[kScTarget + 1] - dot3(dv, cr.v3(kScT));
                    const float r2 = cr[kScTarget + 2] - dot3(dv, cr.v3(kScBt));
                    float3 prop = f3(prev.x + cr[kScPre + 0] * r0 + cr[kScPre + 1] * r1 + cr[kScPre + 2] * r2,
                                     prev.y + cr[kScPre + 3] * r0 + cr[kScPre + 4] * r1 + cr[kScPre + 5] * r2,
                                     prev.z + cr[kScPre + 6] * r0 + cr[kScPre + 7] * r1 + cr[kScPre + 8] * r2);
                    prop = project_cone(prop, cr[kScMu], cr[kScMu]);
                    const float3 delta = cr[kScRelax] * (prop - prev);
                    const float3 next = prev + delta;
                    if (!finite3(next) || !finite3(delta)) {
                        fail(misc, MR_STEP_NONFINITE_RESULT, static_cast<unsigned>(c));
                        cr.set3(kScDelta, f3(0.0f, 0.0f, 0.0f));
                    } else {
                        cr.set3(kScLambda, next);
                        cr.set3(kScDelta, delta);
                    }
                }
                __syncwarp();
            }
            for (int b = lane; b < nb; b += 32) {
                float3 dl = f3(0.0f, 0.0f, 0.0f), dw = f3(0.0f, 0.0f, 0.0f);
                for (int k = start[b]; k < start[b + 1]; ++k) {
                    const int c = entries[k] >> 1, side = entries[k] & 1;
                    const Rec cr = rec(C, c);
                    const float3 d = cr.v3(kScDelta);
                    const float3 imp = cr.v3(kScN) * d.x + cr.v3(kScT) * d.y + cr.v3(kScBt) * d.z;
                    const float3 f = side ? imp : -imp;
                    dl = dl + f;
                    dw = dw + cross3(cr.v3(side ? kScRb : kScRa), f);
                }
                const float im = M.mass[b].y;
                if (kComp) {
                    st3(s + kOffLin + b * 3, kahan_madd3(ld3(s + kOffLin + b * 3), im, dl, s + kOffLinComp + b * 3));
                    st3(s + kOffAng + b * 3,
                        kahan_madd3(ld3(s + kOffAng + b * 3), 1.0f, sym3_mul(s + kOffIiw + b * 6, dw), s + kOffAngComp + b * 3));
                } else {
                    st3(s + kOffLin + b * 3, ld3(s + kOffLin + b * 3) + im * dl);
                    st3(s + kOffAng + b * 3, ld3(s + kOffAng + b * 3) + sym3_mul(s + kOffIiw + b * 6, dw));
                }
            }
            __syncwarp();
        }
        if (!ok(misc)) break;
        // Impulses back into the manifold points.
        for (int c = lane; c < total; c += 32) {
            const Rec cr = rec(C, c);
            const int slot = ai(cr[kScSlot]);
            float* op = tab + (slot >> 2) * kSceneSlotWords + 8 + (slot & 3) * 12;
            op[9] = cr[kScLambda + 0];
            op[10] = cr[kScLambda + 1];
            op[11] = cr[kScLambda + 2];
        }
        // Speed clamps and integration (exponential map of the orientation).
        for (int b = lane; b < nb; b += 32) {
            float3 lin = ld3(s + kOffLin + b * 3), ang = ld3(s + kOffAng + b * 3);
            const float vmax = M.inv_inertia[b].w, wmax = M.offsets[b].w;
            const float ls = len3(lin), ws = len3(ang);
            if (vmax > 0.0f && ls > vmax) lin = lin * (vmax / ls);
            if (wmax > 0.0f && ws > wmax) ang = ang * (wmax / ws);
            const float3 c = kComp ? kahan_madd3(ld3(s + kOffPos + b * 3), h, lin, s + kOffPosComp + b * 3)
                                   : ld3(s + kOffPos + b * 3) + h * lin;
            float4 q = qmul(so3_increment(h * ang, false), ld4(s + kOffQuat + b * 4));
            const float qq = qdot(q, q);
            if (!finite4(q) || !(qq > 1.0e-12f) || !finite3(c) || !finite3(lin) || !finite3(ang)) {
                fail(misc, MR_STEP_NONFINITE_RESULT, static_cast<unsigned>(b));
            } else {
                q = qscale(q, rsqrtf(qq));
            }
            st3(s + kOffLin + b * 3, lin);
            st3(s + kOffAng + b * 3, ang);
            st3(s + kOffPos + b * 3, c);
            st4(s + kOffQuat + b * 4, q);
        }
        if (!ok(misc)) break;
    }

    // Commit: a failed control step publishes nothing (HBM keeps the
    // step-start state), except that a failed reset publishes the reset state.
    const unsigned code = static_cast<unsigned>(ai(misc[kSmStatus]));
    const bool success = code == MR_STEP_SUCCESS;
    float* qd = p.q + static_cast<size_t>(env) * nq;
    float* vd = p.v + static_cast<size_t>(env) * nv;
    float* obs = p.observations ? p.observations + static_cast<size_t>(item) * (nq + nv) : nullptr;
    if (success) {
        for (int b = lane; b < nb; b += 32) {
            st3(qd + b * 7, ld3(s + kOffPos + b * 3));
            st4(qd + b * 7 + 3, ld4(s + kOffQuat + b * 4));
            st3(vd + b * 6, ld3(s + kOffLin + b * 3));
            st3(vd + b * 6 + 3, ld3(s + kOffAng + b * 3));
            if (kComp) st3(p.q_comp + static_cast<size_t>(env) * nq + b * 7, ld3(s + kOffPosComp + b * 3));
        }
        if (cur_table != persistent)
            for (int i = lane; i < mcount * kSceneSlotWords; i += 32) persistent[i] = cur_table[i];
        if (lane == 0) {
            p.manifold_count[env] = static_cast<std::uint32_t>(mcount);
            // A zero point count ends the table for host readers.
            if (mcount < kSceneManifolds) persistent[mcount * kSceneSlotWords + 7] = af(0);
        }
    } else if (reset) {
        for (int i = lane; i < nq; i += 32) qd[i] = srcq[i];
        for (int i = lane; i < nv; i += 32) vd[i] = srcv[i];
        if (kComp)
            for (int b = lane; b < nb; b += 32) st3(p.q_comp + static_cast<size_t>(env) * nq + b * 7, f3(0.0f, 0.0f, 0.0f));
        if (lane == 0) {
            p.manifold_count[env] = 0u;
            p.manifolds[static_cast<size_t>(env) * kTableWords + 7] = af(0);
        }
    }
    __syncwarp();
    if (obs) {
        for (int i = lane; i < nq; i += 32) obs[i] = qd[i];
        for (int i = lane; i < nv; i += 32) obs[nq + i] = vd[i];
    }
    if (lane == 0) {
        const unsigned contacts = static_cast<unsigned>(ai(misc[kSmContacts]));
        if (p.status_codes) p.status_codes[item] = code;
        if (p.active_contacts) p.active_contacts[item] = success ? contacts : 0u;
        if (!success) {
            atomicAdd(p.stats + 0, 1u);
            atomicMin(p.stats + 6, static_cast<unsigned>(env));
        }
        if (reset) atomicAdd(p.stats + 8, 1u);
        atomicMax(p.stats + 1, contacts);
        atomicMax(p.stats + 2, static_cast<unsigned>(ai(misc[kSmManifolds])));
        atomicMax(p.stats + 3, static_cast<unsigned>(ai(misc[kSmRaw])));
        atomicMax(p.stats + 4, static_cast<unsigned>(ai(misc[kSmCand])));
        atomicMax(p.stats + 5, static_cast<unsigned>(ai(misc[kSmIslands])));
    }
}

}  // namespace
}  // namespace numi
