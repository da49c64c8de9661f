// Per-environment FP64 energy and momentum audit, shared by the articulated
// and free-body kernels.  After a successful control step each lane adds
// its bodies' kinetic energy (1/2 m |v|^2 + 1/2 w . R I R^T w), potential
// energy (-m g . c), linear momentum (m v) and angular momentum about the
// world origin (c x m v + R I R^T w) in FP64 from the committed FP32 state;
// the warp reduces them in FP64 and lane 0 updates the environment's
// resident audit record:
//   [0] kinetic  [1] potential  [2] total  [3] reference total (the first
//   audited step after enabling or after a reset)  [4] largest |total -
//   reference| so far  [5..7] linear momentum  [8..10] angular momentum
//   [11] audited control steps since the reference was taken.
#pragma once

#include <cuda_runtime.h>

namespace numi {

constexpr int kAuditWords = 12;

struct AuditSum {
    double v[8];  // kinetic, potential, p xyz, L xyz
};

// One body: mass m, COM c, orientation q (x, y, z, w), COM velocity v,
// angular velocity w (world), body-frame inertia diagonal id and products
// io (xy, xz, yz), gravity g.
__device__ __forceinline__ void audit_body(AuditSum& a, double m, const float3 c, const float4 q, const float3 v, const float3 w,
                                           const float3 id, const float3 io, const float* g) {
    const double x = q.x, y = q.y, z = q.z, s = q.w;
    const double R[3][3] = {{1.0 - 2.0 * (y * y + z * z), 2.0 * (x * y - z * s), 2.0 * (x * z + y * s)},
                            {2.0 * (x * y + z * s), 1.0 - 2.0 * (x * x + z * z), 2.0 * (y * z - x * s)},
                            {2.0 * (x * z - y * s), 2.0 * (y * z + x * s), 1.0 - 2.0 * (x * x + y * y)}};
    const double I[3][3] = {{id.x, io.x, io.y}, {io.x, id.y, io.z}, {io.y, io.z, id.z}};
    const double wv[3] = {w.x, w.y, w.z};
    // w in body axes, then I times it, then back to world axes.
    double wb[3], Ib[3], Iw[3];
    for (int i = 0; i < 3; ++i) wb[i] = R[0][i] * wv[0] + R[1][i] * wv[1] + R[2][i] * wv[2];
    for (int i = 0; i < 3; ++i) Ib[i] = I[i][0] * wb[0] + I[i][1] * wb[1] + I[i][2] * wb[2];
    for (int i = 0; i < 3; ++i) Iw[i] = R[i][0] * Ib[0] + R[i][1] * Ib[1] + R[i][2] * Ib[2];
    const double vv[3] = {v.x, v.y, v.z}, cc[3] = {c.x, c.y, c.z};
    a.v[0] += 0.5 * m * (vv[0] * vv[0] + vv[1] * vv[1] + vv[2] * vv[2]) + 0.5 * (wv[0] * Iw[0] + wv[1] * Iw[1] + wv[2] * Iw[2]);
    a.v[1] -= m * (static_cast<double>(g[0]) * cc[0] + static_cast<double>(g[1]) * cc[1] + static_cast<double>(g[2]) * cc[2]);
    for (int i = 0; i < 3; ++i) a.v[2 + i] += m * vv[i];
    a.v[5] += m * (cc[1] * vv[2] - cc[2] * vv[1]) + Iw[0];
    a.v[6] += m * (cc[2] * vv[0] - cc[0] * vv[2]) + Iw[1];
    a.v[7] += m * (cc[0] * vv[1] - cc[1] * vv[0]) + Iw[2];
}

// Warp reduction (fixed butterfly order: deterministic) and the record
// update by lane 0.  `reset`: this step began from the reset state.
__device__ __forceinline__ void audit_commit(AuditSum& a, double* rec, bool reset, int lane) {
#pragma unroll
    for (int i = 0; i < 8; ++i)
        for (int o = 16; o > 0; o >>= 1) a.v[i] += __shfl_xor_sync(0xffffffffu, a.v[i], o);
    if (lane != 0) return;
    const double total = a.v[0] + a.v[1];
    if (reset || rec[11] == 0.0) {
        rec[3] = total;
        rec[4] = 0.0;
        rec[11] = 0.0;
    }
    rec[0] = a.v[0];
    rec[1] = a.v[1];
    rec[2] = total;
    rec[4] = fmax(rec[4], fabs(total - rec[3]));
    for (int i = 0; i < 6; ++i) rec[5 + i] = a.v[2 + i];
    rec[11] += 1.0;
}

}  // namespace numi
