// The dense symmetric eigensolvers of the modes' Rayleigh-Ritz step, on the host: the p x p
// projected problems of the subspace iteration are small (p = max(2 q, q + 8) for q modes), and
// the reference solves them the same way.
//
// eigen.rs:183-269: K q = lambda M q by a Cholesky factor of D M D (D = diag(M)^-1/2, a unit
// diagonal keeps the factor accurate when the columns differ in scale), C = L^-1 (D K D) L^-T
// made symmetric, its eigenpairs, Q = D L^-T V. eigen.rs:274-331: the cyclic Jacobi method
// (G. H. Golub and C. F. Van Loan, Matrix Computations, 4th ed., algorithm 8.5.1), sweeps until
// the off-diagonal norm is below 1e-15 of the norm, at most 100; the eigenvalues ascending
// (stable order on ties). The operations follow the reference's order and the unit is compiled
// with -ffp-contract=off, so the results equal the reference's bit for bit on the same input.
#include "dense_eigen.hpp"

#include <algorithm>
#include <cmath>
#include <numeric>

namespace femgpu {

void dense_jacobi(double* a, int n, double* values, double* vout) {
    const size_t nn = (size_t)n;
    std::vector<double> v(nn * nn, 0.0);
    for (size_t i = 0; i < nn; ++i) v[i * nn + i] = 1.0;
    double norm = 0.0;
    for (size_t k = 0; k < nn * nn; ++k) norm += a[k] * a[k];
    norm = std::sqrt(norm);
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0;
        for (size_t i = 0; i < nn; ++i)
            for (size_t j = 0; j < nn; ++j)
                if (j != i) off += a[i * nn + j] * a[i * nn + j];
        if (!(std::sqrt(off) > 1e-15 * norm)) break;
        for (size_t p = 0; p < nn; ++p)
            for (size_t q = p + 1; q < nn; ++q) {
                const double apq = a[p * nn + q];
                if (apq == 0.0) continue;
                const double tau = (a[q * nn + q] - a[p * nn + p]) / (2.0 * apq);
                const double t = tau >= 0.0 ? 1.0 / (tau + std::hypot(tau, 1.0))
                                            : -1.0 / (-tau + std::hypot(tau, 1.0));
                const double c = 1.0 / std::hypot(t, 1.0);
                const double s = t * c;
                for (size_t r = 0; r < nn; ++r) {  // columns p and q
                    const double x = a[r * nn + p], y = a[r * nn + q];
                    a[r * nn + p] = c * x - s * y;
                    a[r * nn + q] = s * x + c * y;
                }
                for (size_t r = 0; r < nn; ++r) {  // rows p and q
                    const double x = a[p * nn + r], y = a[q * nn + r];
                    a[p * nn + r] = c * x - s * y;
                    a[q * nn + r] = s * x + c * y;
                }
                for (size_t r = 0; r < nn; ++r) {  // the accumulated rotations
                    const double x = v[r * nn + p], y = v[r * nn + q];
                    v[r * nn + p] = c * x - s * y;
                    v[r * nn + q] = s * x + c * y;
                }
            }
    }
    std::vector<size_t> order(nn);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(),
                     [&](size_t i, size_t j) { return a[i * nn + i] < a[j * nn + j]; });
    for (size_t k = 0; k < nn; ++k) {
        values[k] = a[order[k] * nn + order[k]];
        for (size_t r = 0; r < nn; ++r) vout[r * nn + k] = v[r * nn + order[k]];
    }
}

bool dense_generalized(const double* k, const double* m, int n, double* values, double* q,
                       std::string* err) {
    const size_t nn = (size_t)n;
    std::vector<double> d(nn);
    for (size_t i = 0; i < nn; ++i) {
        if (!(m[i * nn + i] > 0.0)) {
            *err = "the projected mass matrix is not positive definite";
            return false;
        }
        d[i] = 1.0 / std::sqrt(m[i * nn + i]);
    }
    std::vector<double> l(nn * nn, 0.0);
    for (size_t j = 0; j < nn; ++j) {
        double s = m[j * nn + j] * d[j] * d[j];
        for (size_t c = 0; c < j; ++c) s -= l[j * nn + c] * l[j * nn + c];
        if (!(s > 1e-14)) {
            *err = "the projected mass matrix is singular: the subspace vectors are dependent";
            return false;
        }
        s = std::sqrt(s);
        l[j * nn + j] = s;
        for (size_t i = j + 1; i < nn; ++i) {
            double v = m[i * nn + j] * d[i] * d[j];
            for (size_t c = 0; c < j; ++c) v -= l[i * nn + c] * l[j * nn + c];
            l[i * nn + j] = v / s;
        }
    }
    auto lower_solve = [&](double* b) {
        for (size_t i = 0; i < nn; ++i) {
            double v = b[i];
            for (size_t c = 0; c < i; ++c) v -= l[i * nn + c] * b[c];
            b[i] = v / l[i * nn + i];
        }
    };
    std::vector<double> w(nn * nn), col(nn), c(nn * nn);
    for (size_t j = 0; j < nn; ++j) {  // W = L^-1 (D K D)
        for (size_t i = 0; i < nn; ++i) col[i] = k[i * nn + j] * d[i] * d[j];
        lower_solve(col.data());
        for (size_t i = 0; i < nn; ++i) w[i * nn + j] = col[i];
    }
    for (size_t j = 0; j < nn; ++j) {  // C = L^-1 W^T
        std::copy(w.begin() + j * nn, w.begin() + (j + 1) * nn, col.begin());
        lower_solve(col.data());
        for (size_t i = 0; i < nn; ++i) c[i * nn + j] = col[i];
    }
    for (size_t i = 0; i < nn; ++i)
        for (size_t j = 0; j < i; ++j) {
            const double v = 0.5 * (c[i * nn + j] + c[j * nn + i]);
            c[i * nn + j] = v;
            c[j * nn + i] = v;
        }
    std::vector<double> v(nn * nn);
    dense_jacobi(c.data(), n, values, v.data());
    for (size_t j = 0; j < nn; ++j)  // Q = D L^-T V
        for (size_t i = nn; i-- > 0;) {
            double s = v[i * nn + j];
            for (size_t r = i + 1; r < nn; ++r) s -= l[r * nn + i] * q[r * nn + j];
            q[i * nn + j] = s / l[i * nn + i];
        }
    for (size_t i = 0; i < nn; ++i)
        for (size_t j = 0; j < nn; ++j) q[i * nn + j] *= d[i];
    return true;
}

}  // namespace femgpu
