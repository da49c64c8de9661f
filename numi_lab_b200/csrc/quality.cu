// Batched converged contact solve of independent dense problems
// (mr_quality_solve_batch in numi_b200.h): one warp per problem factors the
// mass matrix H = L L', forms the factor rows Y = L^-1 G' of the Delassus
// operator W = G H^-1 G' = Y'Y, runs the FP64 solver of quality.cuh and
// returns v_free + L^-T (Y lambda).  The articulated control step runs the
// same solver on its tree-sparse factor rows.
#include "numi_b200.h"
#include "quality.cuh"
#include "runtime.h"

#include <cmath>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace numi {
namespace rt {

// MRQualitySolverConfigC with its defaults applied and checked.
QualityConfig quality_config(const MRQualitySolverConfigC* c) {
    QualityConfig q{};
    q.max_newton = c && c->maximum_newton_iterations ? static_cast<int>(c->maximum_newton_iterations) : 100;
    q.max_line_search = c && c->maximum_line_search_iterations ? static_cast<int>(c->maximum_line_search_iterations) : 50;
    q.tolerance = c && c->optimality_tolerance > 0.0 ? c->optimality_tolerance : 1.0e-9;
    q.line_search_tolerance = c && c->line_search_tolerance > 0.0 ? c->line_search_tolerance : 0.1;
    q.regularization_floor = c && c->regularization_floor > 0.0 ? c->regularization_floor : 1.0e-6;
    if (q.max_newton > 1000 || q.max_line_search > 200)
        throw std::invalid_argument("quality solver budgets are limited to 1000 Newton steps and 200 line-search evaluations");
    if (!std::isfinite(q.tolerance) || !std::isfinite(q.line_search_tolerance) || !std::isfinite(q.regularization_floor))
        throw std::invalid_argument("quality solver tolerances must be finite");
    return q;
}

}  // namespace rt

namespace {

struct DenseRows {
    const double* Y;  // [3 nc][nv]
    int nv;
    __device__ __forceinline__ int count(int) const { return nv; }
    __device__ __forceinline__ int dof(int, int k) const { return k; }
    __device__ __forceinline__ int pos(int, int d) const { return d; }
    __device__ __forceinline__ double y(int c, int r, int k) const { return Y[(3 * c + r) * nv + k]; }
};

struct BatchParams {
    int problems, nv, cap;
    const std::uint32_t* counts;
    const double* mass;
    const double* jacobian;
    const double* free_velocity;
    const double* target;
    const double* regularization;
    const double* friction;
    const double* warm;
    double* impulses;
    double* velocity;
    MRQualityResultC* results;
    double* scratch;
    size_t scratch_stride;  // doubles per problem
    QualityConfig cfg;
};

__host__ __device__ inline size_t batch_scratch_doubles(int nv, int cap) {
    return static_cast<size_t>(nv) * (nv + 1) / 2 + static_cast<size_t>(3 * cap) * nv + quality_workspace_doubles(nv, cap);
}

__global__ void __launch_bounds__(128) quality_batch_kernel(BatchParams P) {
    const int lane = threadIdx.x & 31;
    const int p = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (p >= P.problems) return;
    const int nv = P.nv, cap = P.cap;
    const int nc = P.counts ? static_cast<int>(P.counts[p]) : cap;
    double* Lf = P.scratch + static_cast<size_t>(p) * P.scratch_stride;
    double* Y = Lf + nv * (nv + 1) / 2;
    double* ws = Y + 3 * cap * nv;
    double* K = ws + quality_contact_offset(nv);
    const double* A = P.mass + static_cast<size_t>(p) * nv * nv;
    const double* G = P.jacobian + static_cast<size_t>(p) * 3 * cap * nv;
    const double* vf = P.free_velocity + static_cast<size_t>(p) * nv;
    const size_t row0 = static_cast<size_t>(p) * 3 * cap;
    MRQualityResultC res{};

    // The lower triangle of H (the mass matrix is read there only).
    for (int r = 0; r < nv; ++r)
        for (int j = lane; j <= r; j += 32) Lf[packed(r, j)] = A[r * nv + j];
    __syncwarp();
    bool ok = warp_cholesky(Lf, nv, lane);
    QualityOutcome o{};
    if (ok) {
        // Factor rows: L y = G_row' by forward substitution, lane per row.
        for (int row = lane; row < 3 * nc; row += 32) {
            const double* g = G + static_cast<size_t>(row) * nv;
            double* y = Y + static_cast<size_t>(row) * nv;
            for (int k = 0; k < nv; ++k) {
                double acc = g[k];
                const double* lk = Lf + packed(k, 0);
                for (int j = 0; j < k; ++j) acc -= lk[j] * y[j];
                y[k] = acc / lk[k];
            }
        }
        for (int c = lane; c < nc; c += 32) {
            double* k = K + c * kQuWords;
            for (int r = 0; r < 3; ++r) {
                const double* g = G + static_cast<size_t>(3 * c + r) * nv;
                double u = 0.0;
                for (int d = 0; d < nv; ++d) u = fma(g[d], vf[d], u);
                k[kQuFree + r] = u;
                k[kQuTarget + r] = P.target[row0 + 3 * c + r];
                k[kQuReg + r] = fmax(P.regularization[row0 + 3 * c + r], P.cfg.regularization_floor);
            }
            const double mu = P.friction[static_cast<size_t>(p) * cap + c];
            k[kQuMu] = mu;
            double l0 = 0.0, l1 = 0.0, l2 = 0.0;
            if (P.warm) {
                l0 = fmax(P.warm[row0 + 3 * c], 0.0);
                l1 = P.warm[row0 + 3 * c + 1];
                l2 = P.warm[row0 + 3 * c + 2];
                const double lt = sqrt(l1 * l1 + l2 * l2), cap_t = mu * l0;
                if (lt > cap_t) {
                    const double s = lt > 0.0 ? cap_t / lt : 0.0;
                    l1 *= s;
                    l2 *= s;
                }
            }
            k[kQuLambda + 0] = l0;
            k[kQuLambda + 1] = l1;
            k[kQuLambda + 2] = l2;
        }
        __syncwarp();
        const DenseRows rows{Y, nv};
        o = quality_solve(rows, nv, nc, ws, P.cfg, lane);
        // Velocity v_free + L^-T (Y lambda) and the dual objective
        // 0.5 ||Y lambda||^2 + sum_c (0.5 l' R l + (u_free - u_target)' l).
        double x0 = lane < nv ? quality_y_lambda(rows, nc, K, lane) : 0.0;
        double x1 = lane + 32 < nv ? quality_y_lambda(rows, nc, K, lane + 32) : 0.0;
        double part = 0.5 * (x0 * x0 + x1 * x1);
        for (int c = lane; c < nc; c += 32) {
            const double* k = K + c * kQuWords;
            for (int r = 0; r < 3; ++r) {
                const double l = k[kQuLambda + r];
                part += 0.5 * k[kQuReg + r] * l * l + (k[kQuFree + r] - k[kQuTarget + r]) * l;
            }
        }
        res.objective = warp_sum_d(part);
        warp_factor_solve_transposed(Lf, nv, lane, x0, x1);
        double* v = P.velocity + static_cast<size_t>(p) * nv;
        if (lane < nv) v[lane] = vf[lane] + x0;
        if (lane + 32 < nv) v[lane + 32] = vf[lane + 32] + x1;
    } else {
        double* v = P.velocity + static_cast<size_t>(p) * nv;
        for (int d = lane; d < nv; d += 32) v[d] = vf[d];
    }
    for (int i = lane; i < 3 * cap; i += 32) {
        const int c = i / 3;
        P.impulses[row0 + i] = ok && c < nc ? K[c * kQuWords + kQuLambda + (i - 3 * c)] : 0.0;
    }
    if (lane == 0) {
        if (!ok) {
            res.code = MR_STEP_FACTORIZATION_FAILED;
        } else {
            res.code = o.status == kQualityConverged       ? MR_STEP_SUCCESS
                       : o.status == kQualityFactorization ? MR_STEP_FACTORIZATION_FAILED
                       : o.status == kQualityNonfinite     ? MR_STEP_NONFINITE_RESULT
                                                           : MR_STEP_DID_NOT_CONVERGE;
            res.newton_iterations = static_cast<std::uint32_t>(o.newton);
            res.line_search_iterations = static_cast<std::uint32_t>(o.line_search);
            res.scaled_optimality = o.residual;
            res.cone_violation = o.cone;
            res.complementarity = o.complementarity;
        }
        P.results[p] = res;
    }
}

template <typename T>
T* upload(rt::DeviceBuffer<T>& buf, const T* host, size_t n) {
    if (!host) return nullptr;
    buf.resize(n);
    rt::check(cudaMemcpy(buf.ptr, host, n * sizeof(T), cudaMemcpyHostToDevice), "quality problem upload");
    return buf.ptr;
}

bool all_finite(const double* x, size_t n) {
    for (size_t i = 0; i < n; ++i)
        if (!std::isfinite(x[i])) return false;
    return true;
}

}  // namespace
}  // namespace numi

extern "C" {

MR_API int mr_quality_solve_batch(uint32_t problem_count, uint32_t nv, uint32_t contact_capacity, const uint32_t* contact_counts,
                                  const double* mass, const double* jacobian, const double* free_velocity,
                                  const double* target_velocity, const double* regularization, const double* friction,
                                  const double* warm_impulses, const MRQualitySolverConfigC* config, double* impulses,
                                  double* velocity, MRQualityResultC* results) {
    using numi::rt::check;
    return numi::rt::guarded([&] {
        if (problem_count == 0) throw std::invalid_argument("problem_count must be positive");
        if (nv == 0 || nv > 64) throw std::invalid_argument("nv must be in [1, 64]");
        if (contact_capacity == 0 || contact_capacity > 32) throw std::invalid_argument("contact_capacity must be in [1, 32]");
        if (!mass || !jacobian || !free_velocity || !target_velocity || !regularization || !friction || !impulses || !velocity ||
            !results)
            throw std::invalid_argument("problem arrays and outputs must be non-null (only contact_counts, warm_impulses and config may be null)");
        const numi::QualityConfig cfg = numi::rt::quality_config(config);
        const size_t P = problem_count, cap = contact_capacity, rows = 3 * cap;
        if (!numi::all_finite(mass, P * nv * nv) || !numi::all_finite(jacobian, P * rows * nv) ||
            !numi::all_finite(free_velocity, P * nv) || !numi::all_finite(target_velocity, P * rows) ||
            !numi::all_finite(regularization, P * rows) || !numi::all_finite(friction, P * cap) ||
            (warm_impulses && !numi::all_finite(warm_impulses, P * rows)))
            throw std::invalid_argument("problem data must be finite");
        for (size_t p = 0; p < P; ++p) {
            const size_t nc = contact_counts ? contact_counts[p] : cap;
            if (nc > cap) throw std::invalid_argument("contact_counts[" + std::to_string(p) + "] exceeds contact_capacity");
            for (size_t c = 0; c < nc; ++c) {
                const double mu = friction[p * cap + c];
                const double* r = regularization + p * rows + 3 * c;
                if (mu < 0.0 || r[0] < 0.0 || r[1] < 0.0 || r[2] < 0.0)
                    throw std::invalid_argument("friction and regularization must be non-negative");
                if (mu > 0.0 && std::fmax(r[1], cfg.regularization_floor) != std::fmax(r[2], cfg.regularization_floor))
                    throw std::invalid_argument("problem " + std::to_string(p) + " contact " + std::to_string(c) +
                                                ": the two tangent regularisations of a frictional contact must be equal");
            }
        }
        numi::rt::DeviceBuffer<std::uint32_t> d_counts;
        numi::rt::DeviceBuffer<double> d_mass, d_jac, d_vf, d_target, d_reg, d_mu, d_warm, d_imp, d_vel, d_scratch;
        numi::rt::DeviceBuffer<MRQualityResultC> d_res;
        numi::BatchParams bp{};
        bp.problems = static_cast<int>(problem_count);
        bp.nv = static_cast<int>(nv);
        bp.cap = static_cast<int>(contact_capacity);
        bp.counts = numi::upload(d_counts, contact_counts, P);
        bp.mass = numi::upload(d_mass, mass, P * nv * nv);
        bp.jacobian = numi::upload(d_jac, jacobian, P * rows * nv);
        bp.free_velocity = numi::upload(d_vf, free_velocity, P * nv);
        bp.target = numi::upload(d_target, target_velocity, P * rows);
        bp.regularization = numi::upload(d_reg, regularization, P * rows);
        bp.friction = numi::upload(d_mu, friction, P * cap);
        bp.warm = numi::upload(d_warm, warm_impulses, P * rows);
        d_imp.resize(P * rows);
        d_vel.resize(P * nv);
        d_res.resize(P);
        bp.scratch_stride = numi::batch_scratch_doubles(bp.nv, bp.cap);
        d_scratch.resize(P * bp.scratch_stride);
        bp.impulses = d_imp.ptr;
        bp.velocity = d_vel.ptr;
        bp.results = d_res.ptr;
        bp.scratch = d_scratch.ptr;
        bp.cfg = cfg;
        constexpr int kWarps = 4;
        const unsigned blocks = static_cast<unsigned>((P + kWarps - 1) / kWarps);
        numi::quality_batch_kernel<<<blocks, 32 * kWarps>>>(bp);
        check(cudaGetLastError(), "quality solve launch");
        check(cudaMemcpy(impulses, d_imp.ptr, P * rows * sizeof(double), cudaMemcpyDeviceToHost), "impulses D2H");
        check(cudaMemcpy(velocity, d_vel.ptr, P * nv * sizeof(double), cudaMemcpyDeviceToHost), "velocity D2H");
        check(cudaMemcpy(results, d_res.ptr, P * sizeof(MRQualityResultC), cudaMemcpyDeviceToHost), "results D2H");
    });
}

}  // extern "C"
