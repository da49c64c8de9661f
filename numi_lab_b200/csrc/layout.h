// Per-warp shared-memory carve-out of the microstep kernel.  Every section
// is sized from the compiled model, so a 7-DoF chain and a 29-DoF tree get
// exactly the scratch they need; sections start on 16-byte boundaries.
#pragma once

#include "device_model.h"

namespace numi {

// Words of one solver contact record in shared memory.
// Most environments (warps) one CTA of the FP32 temporalCone control-step
// kernel may carry; the other instances carry at most 4.
constexpr int kMaxStepWarpsPerBlock = 13;
constexpr int kContactWords = 45;  // 44 used; odd stride keeps lane-per-contact access conflict free
enum ContactWord : int {
    kCwPoint = 0,      // world contact point (3)
    kCwSeparation = 3,
    kCwNormal = 4,     // n, t, b directions (3 x 3)
    kCwTangent = 7,
    kCwBitangent = 10,
    kCwTarget = 13,    // evaluated target velocity per row (3)
    kCwReg = 16,       // regularisation per row (3)
    kCwMuU = 19,
    kCwMuV = 20,
    kCwLambda = 21,    // accumulated impulse (3)
    kCwPre = 24,       // 3x3 preconditioner, row-major (9)
    kCwRelax = 33,
    kCwDelta = 34,     // last impulse change (3)
    kCwBody = 37,      // articulated body (int bits)
    kCwFlags = 38,     // bit0 new impact, bit8 articulated side is B (int bits)
    kCwSlot = 39,      // pair * 4 + manifold point (int bits)
    kCwUfree = 40      // contact-frame relative velocity at v_free (3)
};

// Shared-memory strides (odd, so lane-per-body / per-DoF / per-pair access
// hits distinct banks).
constexpr int kPoseStride = 7;                    // COM position (3), orientation xyzw (4)
constexpr int kJStride = 7;                       // joint axis (3), origin (3), translation flag
constexpr int kSlotStride = kManifoldWords + 1;   // manifold slot

struct WarpLayout {
    int body_pose, dof_J;
    int q, qc, v, vc, vf, tau, qdd, tgt;
    int misc;
    int manifolds, contacts, G, L, z, margins, pair_stats;
    int narrow;  // narrowphase scratch; aliases the contact records and rows
    int qcomp;   // compensation terms of q's running sums (compensated precision only)
    int quality; // FP64 workspace of the quality solver (quality.cuh; quality-solver instances only)
    int total;   // floats per warp
};

__host__ __device__ inline int align4(int x) { return (x + 3) & ~3; }

// Narrowphase scratch of one pair: four kept old points and up to
// `max_raw` raw contacts, 16 words each, plus 16 candidate-id bytes.
constexpr int kCandidateWords = 16;
__host__ __device__ inline int pair_scratch_words(int max_raw) { return (4 + max_raw) * kCandidateWords + 4; }

// Most raw contacts one pair class can produce before manifold reduction.
__host__ __device__ inline int pair_max_raw(int pair_class) {
    return pair_class == MR_COLLISION_PAIR_BOX_PLANE ? 8 : (pair_class == MR_COLLISION_PAIR_CAPSULE_PLANE ? 2 : 1);
}

// `narrow_words` is the sum of pair_scratch_words over the compiled pairs.
// `compensated` appends the q compensation section and `quality_doubles`
// (quality_workspace_doubles, or 0) the quality solver's FP64 workspace;
// the other sections keep their offsets.
__host__ __device__ inline WarpLayout make_layout(int nb, int nv, int nq, int np, int ncap, int max_anc, int narrow_words,
                                                  bool contact, bool compensated = false, int quality_doubles = 0) {
    WarpLayout L{};
    int o = 0;
    auto take = [&o](int words) { const int at = o; o += align4(words); return at; };
    L.body_pose = take(nb * kPoseStride);
    L.dof_J = take(nv * kJStride);
    L.q = take(nq);
    L.qc = take(nq);
    L.v = take(nv);
    L.vc = take(nv);
    L.vf = take(nv);
    L.tau = take(nv);
    L.qdd = take(nv);
    L.tgt = take(nv);
    L.misc = take(32);
    L.z = take(nv);
    L.margins = take(32);
    if (contact) {
        L.manifolds = take(np * kSlotStride);
        L.pair_stats = take(32);
        // Factor rows; past the root block (24 words) they later hold the
        // per-DoF contact lists (nv x ncap u16).
        const int factor = nv * (nv + 1) / 2;
        const int lists = 24 + (nv * ncap + 1) / 2;
        L.L = take(factor > lists ? factor : lists);
        // Contact records and Jacobian rows are written only after the
        // narrowphase has finished with its scratch, so the three share words.
        L.contacts = take(ncap * kContactWords);
        const int rows = align4(ncap * 3 * (max_anc | 1));
        const int need = align4(narrow_words) - align4(ncap * kContactWords);
        L.G = take(rows > need ? rows : need);
        L.narrow = L.contacts;
    } else {
        L.manifolds = L.contacts = L.G = L.L = L.narrow = L.pair_stats = o;
    }
    L.qcomp = compensated ? take(nq) : o;
    L.quality = quality_doubles > 0 ? take(2 * quality_doubles) : o;
    L.total = align4(o);
    return L;
}

// misc words
enum MiscWord : int {
    kMiscP0 = 0,         // reference point (3)
    kMiscStatus = 4,     // step status code (int bits)
    kMiscFailIndex = 5,
    kMiscContactCount = 6,
    kMiscManifoldCount = 7,
    kMiscRawCount = 8,
    kMiscCandidatePairs = 9,
    kMiscIslands = 10,
    // Quality solver, over the control step's substeps: most Newton steps,
    // total line-search evaluations (int bits), largest scaled optimality,
    // cone violation and conic complementarity.
    kMiscQualityNewton = 16,
    kMiscQualityLineSearch = 17,
    kMiscQualityResidual = 18,
    kMiscQualityCone = 19,
    kMiscQualityComplementarity = 20
};

}  // namespace numi
