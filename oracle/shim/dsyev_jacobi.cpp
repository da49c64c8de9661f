// Eigenvalues of a real symmetric matrix by the cyclic Jacobi method
// (Golub & Van Loan, "Matrix Computations", 4th ed., Alg. 8.5.3), exposed
// under the LAPACK dsyev_ calling convention for JOBZ = 'N' only.
//
// Test infrastructure: it lets the reference's FP64 CPU core link on Linux
// (its QualityContactSolver.cpp calls dsyev_ for a minimum-eigenvalue check).
// Eigenvalues are returned in ascending order like LAPACK.

#include "Accelerate/Accelerate.h"

#include <algorithm>
#include <cmath>
#include <vector>

extern "C" void dsyev_(
    const char* jobz,
    const char* uplo,
    const __LAPACK_int* n,
    double* a,
    const __LAPACK_int* lda,
    double* w,
    double* work,
    const __LAPACK_int* lwork,
    __LAPACK_int* info
) {
    const __LAPACK_int order = *n;
    *info = 0;
    if (jobz == nullptr || (*jobz != 'N' && *jobz != 'n') || order < 0 ||
        *lda < std::max<__LAPACK_int>(1, order)) {
        *info = -1;
        return;
    }
    if (*lwork == -1) {
        work[0] = static_cast<double>(std::max<__LAPACK_int>(1, 3 * order));
        return;
    }
    if (order == 0) {
        return;
    }
    const bool upper = (*uplo == 'U' || *uplo == 'u');
    const std::size_t size = static_cast<std::size_t>(order);
    const std::size_t stride = static_cast<std::size_t>(*lda);
    // Column-major input; mirror the referenced triangle into a full matrix.
    std::vector<double> m(size * size);
    for (std::size_t column = 0; column < size; ++column) {
        for (std::size_t row = 0; row < size; ++row) {
            const bool stored = upper ? row <= column : row >= column;
            const double value = stored ? a[row + column * stride]
                                        : a[column + row * stride];
            m[row * size + column] = value;
        }
    }
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0;
        double scale = 0.0;
        for (std::size_t i = 0; i < size; ++i) {
            for (std::size_t j = 0; j < size; ++j) {
                const double v = m[i * size + j] * m[i * size + j];
                scale += v;
                if (i != j) {
                    off += v;
                }
            }
        }
        if (off <= 1.0e-30 * scale || off == 0.0) {
            break;
        }
        for (std::size_t p = 0; p + 1 < size; ++p) {
            for (std::size_t q = p + 1; q < size; ++q) {
                const double apq = m[p * size + q];
                if (apq == 0.0) {
                    continue;
                }
                const double app = m[p * size + p];
                const double aqq = m[q * size + q];
                const double tau = (aqq - app) / (2.0 * apq);
                const double t = (tau >= 0.0 ? 1.0 : -1.0) /
                    (std::fabs(tau) + std::sqrt(1.0 + tau * tau));
                const double c = 1.0 / std::sqrt(1.0 + t * t);
                const double s = t * c;
                for (std::size_t k = 0; k < size; ++k) {
                    const double mkp = m[k * size + p];
                    const double mkq = m[k * size + q];
                    m[k * size + p] = c * mkp - s * mkq;
                    m[k * size + q] = s * mkp + c * mkq;
                }
                for (std::size_t k = 0; k < size; ++k) {
                    const double mpk = m[p * size + k];
                    const double mqk = m[q * size + k];
                    m[p * size + k] = c * mpk - s * mqk;
                    m[q * size + k] = s * mpk + c * mqk;
                }
            }
        }
    }
    for (std::size_t i = 0; i < size; ++i) {
        w[i] = m[i * size + i];
    }
    std::sort(w, w + size);
    for (std::size_t column = 0; column < size; ++column) {
        for (std::size_t row = 0; row < size; ++row) {
            a[row + column * stride] = 0.0;
        }
    }
}
