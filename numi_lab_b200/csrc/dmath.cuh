// Small vector / quaternion / spatial-algebra helpers for the microstep
// kernels.  Quaternions are xyzw; spatial vectors are (angular, linear)
// about a common reference point in world axes.
#pragma once

#include <cuda_runtime.h>

namespace numi {

__device__ __forceinline__ float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 xyz(float4 a) { return make_float3(a.x, a.y, a.z); }
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator-(float3 a) { return f3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ float3 operator*(float s, float3 a) { return f3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ float3 operator*(float3 a, float s) { return f3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
    return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float len3(float3 a) { return sqrtf(dot3(a, a)); }
__device__ __forceinline__ float maxabs3(float3 a) { return fmaxf(fmaxf(fabsf(a.x), fabsf(a.y)), fabsf(a.z)); }
__device__ __forceinline__ bool finite3(float3 a) { return isfinite(a.x) && isfinite(a.y) && isfinite(a.z); }
__device__ __forceinline__ bool finite4(float4 a) {
    return isfinite(a.x) && isfinite(a.y) && isfinite(a.z) && isfinite(a.w);
}
__device__ __forceinline__ float3 ld3(const float* p) { return f3(p[0], p[1], p[2]); }
__device__ __forceinline__ void st3(float* p, float3 a) { p[0] = a.x; p[1] = a.y; p[2] = a.z; }
__device__ __forceinline__ float4 ld4(const float* p) { return make_float4(p[0], p[1], p[2], p[3]); }
__device__ __forceinline__ void st4(float* p, float4 a) { p[0] = a.x; p[1] = a.y; p[2] = a.z; p[3] = a.w; }

__device__ __forceinline__ float4 qconj(float4 q) { return make_float4(-q.x, -q.y, -q.z, q.w); }
__device__ __forceinline__ float4 qmul(float4 l, float4 r) {
    return make_float4(l.w * r.x + l.x * r.w + l.y * r.z - l.z * r.y,
                       l.w * r.y - l.x * r.z + l.y * r.w + l.z * r.x,
                       l.w * r.z + l.x * r.y - l.y * r.x + l.z * r.w,
                       l.w * r.w - l.x * r.x - l.y * r.y - l.z * r.z);
}
__device__ __forceinline__ float3 qrot(float4 q, float3 v) {
    const float3 u = xyz(q);
    const float3 t = 2.0f * cross3(u, v);
    return v + q.w * t + cross3(u, t);
}
__device__ __forceinline__ float3 qrotinv(float4 q, float3 v) { return qrot(qconj(q), v); }
__device__ __forceinline__ float qdot(float4 a, float4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
__device__ __forceinline__ float4 qscale(float4 q, float s) { return make_float4(q.x * s, q.y * s, q.z * s, q.w * s); }

// Normalises a quaternion; fails on non-finite input, a vanishing norm, or
// (require_unit) a norm further than 2e-5 from one.
__device__ __forceinline__ bool qnormalize(float4 in, float4& out, bool require_unit) {
    if (!finite4(in)) return false;
    const float n2 = qdot(in, in);
    if (!(n2 > 1.0e-12f) || !isfinite(n2)) return false;
    const float n = sqrtf(n2);
    if (require_unit && fabsf(n - 1.0f) > 2.0e-5f) return false;
    out = qscale(in, 1.0f / n);
    return finite4(out);
}

// Exponential-map increment for a world angular displacement h*omega,
// composed on the left: q' = normalize(exp(h w) * q).
__device__ __forceinline__ float4 so3_increment(float3 rv, bool reduce_angle) {
    const float angle = len3(rv);
    float half = 0.5f * angle;
    if (reduce_angle && angle > 6.28318530717958647692f) half = 0.5f * fmodf(angle, 6.28318530717958647692f);
    const float s = angle > 1.0e-6f ? sinf(half) / angle : 0.5f - angle * angle / 48.0f;
    return make_float4(rv.x * s, rv.y * s, rv.z * s, cosf(half));
}

// Packed symmetric 6x6 (lower triangle, row-major): index(i, j), i >= j.
__device__ __forceinline__ int sym6(int i, int j) { return i >= j ? i * (i + 1) / 2 + j : j * (j + 1) / 2 + i; }

// y = A x for packed symmetric 6x6 A (R = float or double).
template <typename R>
__device__ __forceinline__ void sym6_mul(const R* A, const float* x, R* y) {
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        R s = R(0);
#pragma unroll
        for (int j = 0; j < 6; ++j) s = fma(A[sym6(i, j)], static_cast<R>(x[j]), s);
        y[i] = s;
    }
}

__device__ __forceinline__ float dot6(const float* a, const float* b) {
    float s = 0.0f;
#pragma unroll
    for (int i = 0; i < 6; ++i) s = fmaf(a[i], b[i], s);
    return s;
}

__device__ __forceinline__ float warp_sum(float x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}
__device__ __forceinline__ float warp_max(float x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x = fmaxf(x, __shfl_xor_sync(0xffffffffu, x, o));
    return x;
}
__device__ __forceinline__ unsigned warp_umax(unsigned x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x = max(x, __shfl_xor_sync(0xffffffffu, x, o));
    return x;
}
__device__ __forceinline__ unsigned warp_umin(unsigned x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x = min(x, __shfl_xor_sync(0xffffffffu, x, o));
    return x;
}

// Compensated running sum x + a * b (Kahan's summation): `c` carries the
// low-order part that earlier additions to x rounded away; the product
// arrives with c subtracted in one rounding.  The explicit _rn intrinsics
// keep the correction from being contracted or reassociated.
__device__ __forceinline__ float kahan_madd(float x, float a, float b, float& c) {
    const float y = __fmaf_rn(a, b, -c);
    const float t = __fadd_rn(x, y);
    c = __fsub_rn(__fsub_rn(t, x), y);
    return t;
}
__device__ __forceinline__ float3 kahan_madd3(float3 x, float a, float3 b, float* c) {
    return f3(kahan_madd(x.x, a, b.x, c[0]), kahan_madd(x.y, a, b.y, c[1]), kahan_madd(x.z, a, b.z, c[2]));
}

}  // namespace numi
