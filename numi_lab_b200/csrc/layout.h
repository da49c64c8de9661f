// Per-warp shared-memory carve-out of the microstep kernel.  Every section
// is sized from the compiled model, so a 7-DoF chain and a 29-DoF tree get
// exactly the scratch they need; sections start on 16-byte boundaries.
#pragma once

#include "device_model.h"

namespace numi {

// Words of one solver contact record in shared memory.
constexpr int kContactWords = 40;
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
    kCwSlot = 39       // pair * 4 + manifold point (int bits)
};

struct WarpLayout {
    int body_pose, body_V, body_CV, body_IA, body_PA, body_U, body_Du, body_A, body_r;
    int dof_S, dof_J;
    int q, qc, qn, v, vc, vf, tau, qdd, tgt;
    int misc;
    int manifolds, contacts, G, R, L;
    int rstride;
    int total;  // floats per warp
};

__host__ __device__ inline int align4(int x) { return (x + 3) & ~3; }

__host__ __device__ inline WarpLayout make_layout(int nb, int nv, int nq, int np, int ncap, int max_anc, bool contact) {
    WarpLayout L{};
    int o = 0;
    auto take = [&o](int words) { const int at = o; o += align4(words); return at; };
    L.body_pose = take(nb * 8);
    L.body_V = take(nb * 6);
    L.body_CV = take(nb * 6);
    L.body_IA = take(nb * 21);
    L.body_PA = take(nb * 6);
    L.body_U = take(nb * 6);
    L.body_Du = take(nb * 2);
    L.body_A = take(nb * 6);
    L.body_r = take(nb * 4);
    L.dof_S = take(nv * 6);
    L.dof_J = take(nv * 8);
    L.q = take(nq);
    L.qc = take(nq);
    L.qn = take(nq);
    L.v = take(nv);
    L.vc = take(nv);
    L.vf = take(nv);
    L.tau = take(nv);
    L.qdd = take(nv);
    L.tgt = take(nv);
    L.misc = take(32);
    L.rstride = nv | 1;  // odd column stride: lane-per-column access is bank-conflict free
    if (contact) {
        L.manifolds = take(np * kManifoldWords);
        L.contacts = take(ncap * kContactWords);
        L.G = take(ncap * 3 * max_anc);
        L.R = take(3 * ncap * L.rstride > 32 ? 3 * ncap * L.rstride : 32);  // also stages collider margins
        L.L = take(nv * (nv + 1) / 2);
    } else {
        L.manifolds = L.contacts = L.G = L.R = L.L = o;
    }
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
    kMiscPairBase = 12   // prefix offsets of pairs (up to 20 words here would overflow; pairs use manifold slots)
};

}  // namespace numi
