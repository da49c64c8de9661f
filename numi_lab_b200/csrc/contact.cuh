// Contact helpers shared by the articulated and the free-body microstep
// kernels: feature keys, the stable tangent of a contact frame, the
// regularised 3x3 block inverse and the elliptic friction-cone projection of
// the temporalCone iteration.
#pragma once

#include "dmath.cuh"

namespace numi {

constexpr float kContactCfm = 1.0e-2f;  // MetalWorldContact.metal:18
constexpr float kMatrixFloor = 1.0e-10f;

__device__ __forceinline__ unsigned feature_key(unsigned type, unsigned local) {
    return ((type & 0x0fu) << 28u) | (local & 0x0fffffffu);
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
__device__ inline bool invert3x3_reg(const float m[3][3], float inv[3][3]) {
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

}  // namespace numi
