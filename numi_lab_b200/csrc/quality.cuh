// Converged (quality) contact solve: one warp per problem, FP64 throughout.
//
// The problem is numi-lab's exact-cone contact QP (ReferenceConicSolver.hpp,
// QualityContactSolver.hpp:55-80):
//
//   min_lambda 0.5 lambda' (W + R) lambda + (u_free - u_target)' lambda
//   s.t. lambda_n >= 0, ||lambda_t|| <= mu lambda_n        (per contact)
//
// with W = G H^-1 G' the Delassus operator of joint-space inertia H and
// R > 0 diagonal.  The reference solves it on the GPU as a primal Newton
// iteration in generalized velocities (MetalUnifiedQualitySolver.metal:
// 1322-2263) and on the CPU as a dual semismooth Newton iteration
// (QualityContactSolver.cpp:1172).  This solver works in the factor space
// of the inertia instead.  With any factor Y (nv x 3n) of W = Y'Y (the
// kernels already hold Y = L^-T G' for H = L'L), the minimiser is the dual
// of
//
//   min_zeta f(zeta) = 0.5 ||zeta||^2 + sum_c psi_c(u_free_c + Y_c' zeta)
//   psi_c(u)  = -min_{lambda in K_c} (0.5 lambda' R_c lambda + (u - u_target,c)' lambda)
//
// whose gradient is zeta - Y lambda(zeta), lambda_c(u) the R_c-metric
// projection of -R_c^-1 (u - u_target,c) onto the friction cone.  f is
// convex and C^1 with a piecewise smooth gradient; its generalized Hessian
// I + sum_c Y_c D_c Y_c' (D_c = -d lambda_c / d u, PSD) is bounded below by
// the identity.  Each Newton direction (Cholesky solve of that nv x nv
// matrix) is followed by an exact line search: phi(t) = f(zeta + t d) has
// the monotone derivative
//   phi'(t) = d'zeta + t d'd - sum_c lambda_c(u_c + t w_c)' w_c,  w_c = Y_c' d,
// which costs O(contacts) per evaluation once the w_c are known, and its
// root is found by safeguarded Newton steps inside a bracket (the exact
// line search of MuJoCo's Newton solver, Todorov 2014, applied to this
// cone).  The iteration converges globally and, near the solution,
// superlinearly (semismooth Newton); a continuation on the regularisation
// (below) keeps the iterates near the solution's contact regions.  At the solution zeta = Y lambda, so
// the velocity change is H^-1 G' lambda = L^-1 zeta, and lambda is
// feasible by construction.
//
// The projection onto the cone {||l_t|| <= mu l_n} in the metric
// diag(r_n, r_t, r_t) is closed form: after the change of variables
// y_t = l_t / mu the cone is a unit Lorentz cone in the metric
// diag(D0, Dt, Dt), D0 = r_n, Dt = r_t mu^2, and a point b = (b0, b_t),
// s = ||b_t||, projects to
//   b                         if s <= b0            (sticking)
//   0                         if D0 b0 <= -Dt s     (separating)
//   rho (1, b_t / s),  rho = (D0 b0 + Dt s) / (D0 + Dt)   otherwise (sliding),
// the last from the KKT conditions of the metric projection.  Blocks whose
// two tangent regularisations differ are not supported (the callers
// reject them).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "device_model.h"

namespace numi {

enum QualityStatus : int {
    kQualityConverged = 0,
    kQualityNotConverged = 1,    // iteration or line-search budget exhausted
    kQualityFactorization = 2,   // Newton matrix not positive definite (non-finite data)
    kQualityNonfinite = 3
};

struct QualityOutcome {
    int status;
    int newton;          // Newton steps taken
    int line_search;     // line-search evaluations of phi', summed
    double residual;     // scaled optimality at exit
    double cone;         // largest cone violation of the impulses
    double complementarity;  // largest |lambda' (u - u_target + R lambda)|
    double objective;    // f at exit
};

// FP64 words of one contact in the workspace: the problem data (filled by
// the caller: free contact velocity, target velocity, regularisation with
// the floor applied, friction, warm impulse in kQuLambda), the solver's
// impulse and cone derivative (packed symmetric 00 01 02 11 12 22), and
// the line search's contact velocity and direction image w = Y_c' d.
enum QualityContactWord : int {
    kQuFree = 0,
    kQuTarget = 3,
    kQuReg = 6,
    kQuMu = 9,
    kQuLambda = 10,
    kQuD = 13,
    kQuU = 19,
    kQuW = 22,
    kQuWords = 25
};

// Workspace: zeta, gradient, direction (nv each), the packed lower Newton
// matrix, then the contact words.
__host__ __device__ inline int quality_contact_offset(int nv) { return 3 * nv + nv * (nv + 1) / 2; }
__host__ __device__ inline int quality_workspace_doubles(int nv, int nc) { return quality_contact_offset(nv) + nc * kQuWords; }

__device__ __forceinline__ double warp_sum_d(double x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}
__device__ __forceinline__ double warp_max_d(double x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x = fmax(x, __shfl_xor_sync(0xffffffffu, x, o));
    return x;
}
__device__ __forceinline__ int packed(int i, int j) { return i * (i + 1) / 2 + j; }  // row-major lower, j <= i

// Impulse, cone derivative and psi of one contact at contact velocity u,
// with the regularisation raised to at least `rho` (continuation stage).
__device__ __forceinline__ double quality_project(const double* k, const double u[3], double lam[3], double D[6], double rho) {
    const double e0 = u[0] - k[kQuTarget + 0], e1 = u[1] - k[kQuTarget + 1], e2 = u[2] - k[kQuTarget + 2];
    const double r0 = fmax(k[kQuReg + 0], rho), r1 = fmax(k[kQuReg + 1], rho), r2 = fmax(k[kQuReg + 2], rho);
    const double a0 = -e0 / r0, a1 = -e1 / r1, a2 = -e2 / r2;
    const double mu = k[kQuMu];
#pragma unroll
    for (int i = 0; i < 6; ++i) D[i] = 0.0;
    if (!(mu > 0.0)) {
        lam[0] = fmax(a0, 0.0);
        lam[1] = 0.0;
        lam[2] = 0.0;
        if (lam[0] > 0.0) D[0] = 1.0 / r0;
    } else {
        const double b1 = a1 / mu, b2 = a2 / mu;
        const double s = sqrt(b1 * b1 + b2 * b2);
        const double d0 = r0, dt = r1 * mu * mu;
        if (s <= a0) {
            lam[0] = a0;
            lam[1] = a1;
            lam[2] = a2;
            D[0] = 1.0 / r0;
            D[3] = 1.0 / r1;
            D[5] = 1.0 / r2;
        } else if (d0 * a0 <= -dt * s) {
            lam[0] = 0.0;
            lam[1] = 0.0;
            lam[2] = 0.0;
        } else {
            const double inv = 1.0 / (d0 + dt);
            const double rho = (d0 * a0 + dt * s) * inv;
            const double n1 = b1 / s, n2 = b2 / s;
            lam[0] = rho;
            lam[1] = mu * rho * n1;
            lam[2] = mu * rho * n2;
            // D = v v' / (D0 + Dt) + rho / (s r_t) (I - n n') on the tangent
            // block, v = (1, mu n).
            const double w = rho / (s * r1);
            D[0] = inv;
            D[1] = inv * mu * n1;
            D[2] = inv * mu * n2;
            D[3] = inv * mu * mu * n1 * n1 + w * (1.0 - n1 * n1);
            D[4] = inv * mu * mu * n1 * n2 - w * n1 * n2;
            D[5] = inv * mu * mu * n2 * n2 + w * (1.0 - n2 * n2);
        }
    }
    return -(0.5 * (r0 * lam[0] * lam[0] + r1 * lam[1] * lam[1] + r2 * lam[2] * lam[2]) + e0 * lam[0] + e1 * lam[1] +
             e2 * lam[2]);
}

// Warp-cooperative in-place Cholesky of the packed row-major lower matrix
// A (n x n, n <= 64) into its lower factor.  Returns false (uniformly) on a
// non-positive or non-finite pivot.
__device__ __forceinline__ bool warp_cholesky(double* A, int n, int lane) {
    for (int k = 0; k < n; ++k) {
        const double pivot = A[packed(k, k)];
        if (!(pivot > 0.0) || !isfinite(pivot)) return false;
        const double lkk = sqrt(pivot);
        __syncwarp();
        if (lane == 0) A[packed(k, k)] = lkk;
        for (int i = k + 1 + lane; i < n; i += 32) A[packed(i, k)] /= lkk;
        __syncwarp();
        for (int i = k + 1 + lane; i < n; i += 32) {
            const double lik = A[packed(i, k)];
            const int row = packed(i, 0);
            for (int j = k + 1; j <= i; ++j) A[row + j] -= lik * A[packed(j, k)];
        }
        __syncwarp();
    }
    return true;
}

// x = (L L')^-1 b for the packed lower factor L (n <= 64).  Row i of b and x
// lives in lane i % 32, register i / 32.
__device__ __forceinline__ void warp_factor_solve(const double* L, int n, int lane, double& x0, double& x1) {
    for (int k = 0; k < n; ++k) {
        const double own = k < 32 ? x0 : x1;
        const double yk = __shfl_sync(0xffffffffu, own, k & 31) / L[packed(k, k)];
        if (lane == (k & 31)) {
            if (k < 32) x0 = yk;
            else x1 = yk;
        }
        if (lane > k && lane < n) x0 -= L[packed(lane, k)] * yk;
        if (lane + 32 > k && lane + 32 < n) x1 -= L[packed(lane + 32, k)] * yk;
    }
    for (int k = n - 1; k >= 0; --k) {
        const double own = k < 32 ? x0 : x1;
        const double xk = __shfl_sync(0xffffffffu, own, k & 31) / L[packed(k, k)];
        if (lane == (k & 31)) {
            if (k < 32) x0 = xk;
            else x1 = xk;
        }
        const int row = packed(k, 0);
        if (lane < k) x0 -= L[row + lane] * xk;
        if (lane + 32 < k) x1 -= L[row + lane + 32] * xk;
    }
}

// x = L^-T b only (the backward half), same register convention.
__device__ __forceinline__ void warp_factor_solve_transposed(const double* L, int n, int lane, double& x0, double& x1) {
    for (int k = n - 1; k >= 0; --k) {
        const double own = k < 32 ? x0 : x1;
        const double xk = __shfl_sync(0xffffffffu, own, k & 31) / L[packed(k, k)];
        if (lane == (k & 31)) {
            if (k < 32) x0 = xk;
            else x1 = xk;
        }
        const int row = packed(k, 0);
        if (lane < k) x0 -= L[row + lane] * xk;
        if (lane + 32 < k) x1 -= L[row + lane + 32] * xk;
    }
}

// Rows: the factor Y, contact by contact.  Interface:
//   int count(c)             DoFs contact c reaches
//   int dof(c, k)            k-th of them
//   int pos(c, d)            position of DoF d in that list, or -1
//   double y(c, r, k)        entry of contact row r (normal, tangent, bitangent)
template <class Rows>
__device__ __forceinline__ double quality_y_dot(const Rows& Y, int c, int r, const double* x) {
    double acc = 0.0;
    const int n = Y.count(c);
    for (int k = 0; k < n; ++k) acc = fma(Y.y(c, r, k), x[Y.dof(c, k)], acc);
    return acc;
}

// (Y lambda)_d for DoF d from the impulses in the contact words.
template <class Rows>
__device__ __forceinline__ double quality_y_lambda(const Rows& Y, int nc, const double* K, int d) {
    double acc = 0.0;
    for (int c = 0; c < nc; ++c) {
        const int k = Y.pos(c, d);
        if (k < 0) continue;
        const double* kc = K + c * kQuWords + kQuLambda;
        acc = fma(Y.y(c, 0, k), kc[0], acc);
        acc = fma(Y.y(c, 1, k), kc[1], acc);
        acc = fma(Y.y(c, 2, k), kc[2], acc);
    }
    return acc;
}

// f at x (regularisation floor rho); with `commit` also the impulses and
// derivatives (contact words) and the gradient.  Every lane returns the
// same value.
template <class Rows>
__device__ double quality_eval(const Rows& Y, int nv, int nc, const double* x, double* K, double* grad, bool commit,
                               double rho, int lane) {
    double part = 0.0;
    for (int c = lane; c < nc; c += 32) {
        double* kc = K + c * kQuWords;
        double u[3];
#pragma unroll
        for (int r = 0; r < 3; ++r) u[r] = kc[kQuFree + r] + quality_y_dot(Y, c, r, x);
        double lam[3], D[6];
        part += quality_project(kc, u, lam, D, rho);
        if (commit) {
#pragma unroll
            for (int r = 0; r < 3; ++r) kc[kQuLambda + r] = lam[r];
#pragma unroll
            for (int i = 0; i < 6; ++i) kc[kQuD + i] = D[i];
        }
    }
    for (int d = lane; d < nv; d += 32) part += 0.5 * x[d] * x[d];
    const double f = warp_sum_d(part);
    if (commit) {
        __syncwarp();
        for (int d = lane; d < nv; d += 32) grad[d] = x[d] - quality_y_lambda(Y, nc, K, d);
        __syncwarp();
    }
    return f;
}

// Regularisation continuation: the solve runs first with every row's
// regularisation raised to kStageFloor0 and then kStageFloor1 times the
// configured floor, each stage to the scaled optimality kStageTolerance,
// and then with the problem's own regularisation to the configured
// tolerance, each stage warm-started by the last.  The raised floors smooth
// the kinks of the near-hard cone terms, so the Newton iterates find the
// contacts' sticking / sliding / separating regions on a smooth function
// and the final stage starts next to its solution.  Over 7,168 control
// steps of the 4096-environment tree29 world (1,024 environments x 7 steps,
// the largest Newton count of each step's four solves) the median / 99th
// percentile / maximum went from 27 / 67 / 124 Newton steps without the
// continuation to 13 / 21 / 31 with it.
constexpr double kStageFloor0 = 3000.0;
constexpr double kStageFloor1 = 30.0;
constexpr double kStageTolerance = 1.0e-3;

// Solves the problem whose contact words (kQuFree .. kQuMu and the warm
// impulse in kQuLambda) the caller filled.  On return the contact words hold
// the impulses and ws[0, nv) holds zeta = Y lambda (up to the tolerance).
template <class Rows>
__device__ QualityOutcome quality_solve(const Rows& Y, int nv, int nc, double* ws, const QualityConfig& cfg, int lane) {
    double* zeta = ws;
    double* grad = ws + nv;
    double* dir = ws + 2 * nv;
    double* H = ws + 3 * nv;
    double* K = ws + quality_contact_offset(nv);
    QualityOutcome out{};
    out.status = kQualityNotConverged;

    // Warm start: zeta = Y lambda_warm.
    for (int d = lane; d < nv; d += 32) zeta[d] = quality_y_lambda(Y, nc, K, d);
    __syncwarp();
    double f = 0.0, scaled = 0.0;
    bool broken = false;  // non-finite data or a failed factorization
    for (int stage = 0; stage < 3 && !broken; ++stage) {
        const double rho = (stage == 0 ? kStageFloor0 : stage == 1 ? kStageFloor1 : 0.0) * cfg.regularization_floor;
        const double tol = stage < 2 ? kStageTolerance : cfg.tolerance;
        f = quality_eval(Y, nv, nc, zeta, K, grad, true, rho, lane);
        for (;;) {
            double gm = 0.0, zm = 0.0, ym = 0.0;
            bool finite = true;
            for (int d = lane; d < nv; d += 32) {
                gm = fmax(gm, fabs(grad[d]));
                zm = fmax(zm, fabs(zeta[d]));
                ym = fmax(ym, fabs(zeta[d] - grad[d]));
                finite = finite && isfinite(grad[d]) && isfinite(zeta[d]);
            }
            gm = warp_max_d(gm);
            zm = warp_max_d(zm);
            ym = warp_max_d(ym);
            if (!__all_sync(0xffffffffu, finite) || !isfinite(f)) {
                out.status = kQualityNonfinite;
                broken = true;
                break;
            }
            scaled = gm / (1.0 + zm + ym);
            if (scaled <= tol) {
                if (stage == 2) out.status = kQualityConverged;
                break;
            }
            if (out.newton >= cfg.max_newton) {
                broken = true;
                break;
            }

            // Newton matrix I + sum_c Y_c D_c Y_c' (lane per column, rows >= column).
            for (int j = lane; j < nv; j += 32) {
                for (int i = j; i < nv; ++i) H[packed(i, j)] = i == j ? 1.0 : 0.0;
                for (int c = 0; c < nc; ++c) {
                    const int kj = Y.pos(c, j);
                    if (kj < 0) continue;
                    const double* D = K + c * kQuWords + kQuD;
                    const double y0 = Y.y(c, 0, kj), y1 = Y.y(c, 1, kj), y2 = Y.y(c, 2, kj);
                    const double e0 = D[0] * y0 + D[1] * y1 + D[2] * y2;
                    const double e1 = D[1] * y0 + D[3] * y1 + D[4] * y2;
                    const double e2 = D[2] * y0 + D[4] * y1 + D[5] * y2;
                    if (e0 == 0.0 && e1 == 0.0 && e2 == 0.0) continue;
                    const int n = Y.count(c);
                    for (int k = 0; k < n; ++k) {
                        const int i = Y.dof(c, k);
                        if (i < j) continue;
                        H[packed(i, j)] += Y.y(c, 0, k) * e0 + Y.y(c, 1, k) * e1 + Y.y(c, 2, k) * e2;
                    }
                }
            }
            __syncwarp();
            if (!warp_cholesky(H, nv, lane)) {
                out.status = kQualityFactorization;
                broken = true;
                break;
            }
            double x0 = lane < nv ? -grad[lane] : 0.0;
            double x1 = lane + 32 < nv ? -grad[lane + 32] : 0.0;
            warp_factor_solve(H, nv, lane, x0, x1);
            double sl = 0.0;
            if (lane < nv) sl += grad[lane] * x0;
            if (lane + 32 < nv) sl += grad[lane + 32] * x1;
            if (!(warp_sum_d(sl) < 0.0)) {
                // Rounding made the Newton direction useless: steepest descent.
                x0 = lane < nv ? -grad[lane] : 0.0;
                x1 = lane + 32 < nv ? -grad[lane + 32] : 0.0;
            }
            if (lane < nv) dir[lane] = x0;
            if (lane + 32 < nv) dir[lane + 32] = x1;
            __syncwarp();

            // Exact line search: the root of phi'(t) = a + t b - sum_c lambda_c' w_c.
            double pa = 0.0, pb = 0.0, pg = 0.0;
            for (int d = lane; d < nv; d += 32) {
                pa += dir[d] * zeta[d];
                pb += dir[d] * dir[d];
                pg += dir[d] * grad[d];
            }
            const double a = warp_sum_d(pa), b = warp_sum_d(pb), slope0 = warp_sum_d(pg);
            for (int c = lane; c < nc; c += 32) {
                double* kc = K + c * kQuWords;
#pragma unroll
                for (int r = 0; r < 3; ++r) {
                    kc[kQuU + r] = kc[kQuFree + r] + quality_y_dot(Y, c, r, zeta);
                    kc[kQuW + r] = quality_y_dot(Y, c, r, dir);
                }
            }
            double lo = 0.0, hi = INFINITY, t = 1.0, best = INFINITY, best_t = 1.0;
            for (int ls = 0; ls < cfg.max_line_search; ++ls) {
                double ps = 0.0, ph = 0.0;
                for (int c = lane; c < nc; c += 32) {
                    const double* kc = K + c * kQuWords;
                    double u[3], lam[3], D[6];
#pragma unroll
                    for (int r = 0; r < 3; ++r) u[r] = kc[kQuU + r] + t * kc[kQuW + r];
                    quality_project(kc, u, lam, D, rho);
                    const double w0 = kc[kQuW], w1 = kc[kQuW + 1], w2 = kc[kQuW + 2];
                    ps += lam[0] * w0 + lam[1] * w1 + lam[2] * w2;
                    ph += w0 * (D[0] * w0 + D[1] * w1 + D[2] * w2) + w1 * (D[1] * w0 + D[3] * w1 + D[4] * w2) +
                          w2 * (D[2] * w0 + D[4] * w1 + D[5] * w2);
                }
                const double dt = a + t * b - warp_sum_d(ps);
                const double h2 = b + warp_sum_d(ph);
                ++out.line_search;
                if (fabs(dt) < best) {
                    best = fabs(dt);
                    best_t = t;
                }
                if (fabs(dt) <= cfg.line_search_tolerance * fabs(slope0)) break;
                if (dt < 0.0) lo = t;
                else hi = t;
                double tn = t - dt / h2;
                if (!(tn > lo && tn < hi)) tn = isfinite(hi) ? 0.5 * (lo + hi) : 2.0 * t;
                if (isfinite(hi) && hi - lo <= 1.0e-14 * hi) break;
                t = tn;
            }
            for (int d = lane; d < nv; d += 32) zeta[d] += best_t * dir[d];
            __syncwarp();
            f = quality_eval(Y, nv, nc, zeta, K, grad, true, rho, lane);
            ++out.newton;
        }
    }
    out.residual = scaled;
    out.objective = f;

    // Certificates of the final impulses: cone feasibility and the conic
    // complementarity lambda' (u - u_target + R lambda).
    double cone = 0.0, comp = 0.0;
    for (int c = lane; c < nc; c += 32) {
        const double* kc = K + c * kQuWords;
        const double l0 = kc[kQuLambda], l1 = kc[kQuLambda + 1], l2 = kc[kQuLambda + 2];
        const double mu = kc[kQuMu];
        const double lt = sqrt(l1 * l1 + l2 * l2);
        cone = fmax(cone, fmax(-l0, mu > 0.0 ? lt - mu * l0 : lt));
        double w = 0.0;
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            const double u = kc[kQuFree + r] + quality_y_dot(Y, c, r, zeta);
            w += kc[kQuLambda + r] * (u - kc[kQuTarget + r] + kc[kQuReg + r] * kc[kQuLambda + r]);
        }
        comp = fmax(comp, fabs(w));
    }
    out.cone = warp_max_d(cone);
    out.complementarity = warp_max_d(comp);
    return out;
}

}  // namespace numi
