// Oracle (test infrastructure): the consistent mass of the 10-node tetrahedron
// (crates/fem/src/tet10.rs:173-212) and the dense symmetric eigensolvers of
// crates/fem/src/eigen.rs:183-331 (the generalized problem by a scaled Cholesky reduction, the
// standard problem by the cyclic Jacobi method of Golub and Van Loan, algorithm 8.5.1). The
// subspace iteration of eigen.rs:81-177 is restated in oracle/__init__.py over these.
#include <algorithm>
#include <cmath>
#include <numeric>
#include <string>

#include "oracle.hpp"

namespace orc {

namespace {
const int EDGE[6][2] = {{0, 1}, {1, 2}, {0, 2}, {0, 3}, {1, 3}, {2, 3}};  // tet10.rs:38
}

// tet10.rs:173-212
void tet10_mass(double volume, double density, double m[900]) {
    auto scalar = [](int i, int j) -> double {
        if (i < 4 && j < 4) return i == j ? 6.0 : 1.0;
        if (i < 4 || j < 4) {
            int c = i < 4 ? i : j, e = i < 4 ? j - 4 : i - 4;
            return (EDGE[e][0] == c || EDGE[e][1] == c) ? -4.0 : -6.0;
        }
        const int* a = EDGE[i - 4];
        const int* b = EDGE[j - 4];
        int shared = (a[0] == b[0] || a[0] == b[1]) + (a[1] == b[0] || a[1] == b[1]);
        return shared == 2 ? 32.0 : (shared == 1 ? 16.0 : 8.0);
    };
    double w = density * volume / 420.0;
    std::fill(m, m + 900, 0.0);
    for (int i = 0; i < 10; ++i)
        for (int j = 0; j < 10; ++j) {
            double v = w * scalar(i, j);
            for (int a = 0; a < 3; ++a) m[(3 * i + a) * 30 + 3 * j + a] = v;
        }
}

// eigen.rs:274-331
void dense_jacobi(double* a, int n, double* values, double* vout) {
    vector<double> v((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) v[(size_t)i * n + i] = 1.0;
    double norm = 0.0;
    for (size_t k = 0; k < (size_t)n * n; ++k) norm += a[k] * a[k];
    norm = std::sqrt(norm);
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0;
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j)
                if (j != i) off += a[(size_t)i * n + j] * a[(size_t)i * n + j];
        off = std::sqrt(off);
        if (!(off > 1e-15 * norm)) break;
        for (int p = 0; p < n; ++p)
            for (int q = p + 1; q < n; ++q) {
                double apq = a[(size_t)p * n + q];
                if (apq == 0.0) continue;
                double tau = (a[(size_t)q * n + q] - a[(size_t)p * n + p]) / (2.0 * apq);
                double t = tau >= 0.0 ? 1.0 / (tau + std::hypot(tau, 1.0))
                                      : -1.0 / (-tau + std::hypot(tau, 1.0));
                double c = 1.0 / std::hypot(t, 1.0);
                double s = t * c;
                for (int r = 0; r < n; ++r) {
                    double x = a[(size_t)r * n + p], y = a[(size_t)r * n + q];
                    a[(size_t)r * n + p] = c * x - s * y;
                    a[(size_t)r * n + q] = s * x + c * y;
                }
                for (int r = 0; r < n; ++r) {
                    double x = a[(size_t)p * n + r], y = a[(size_t)q * n + r];
                    a[(size_t)p * n + r] = c * x - s * y;
                    a[(size_t)q * n + r] = s * x + c * y;
                }
                for (int r = 0; r < n; ++r) {
                    double x = v[(size_t)r * n + p], y = v[(size_t)r * n + q];
                    v[(size_t)r * n + p] = c * x - s * y;
                    v[(size_t)r * n + q] = s * x + c * y;
                }
            }
    }
    vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int i, int j) {
        return a[(size_t)i * n + i] < a[(size_t)j * n + j];
    });
    for (int k = 0; k < n; ++k) {
        values[k] = a[(size_t)order[k] * n + order[k]];
        for (int r = 0; r < n; ++r) vout[(size_t)r * n + k] = v[(size_t)r * n + order[k]];
    }
}

// eigen.rs:183-269
bool dense_generalized(const double* k, const double* m, int n, double* values, double* q,
                       std::string* err) {
    vector<double> d(n);
    for (int i = 0; i < n; ++i) {
        if (!(m[(size_t)i * n + i] > 0.0)) {
            *err = "the projected mass matrix is not positive definite";
            return false;
        }
        d[i] = 1.0 / std::sqrt(m[(size_t)i * n + i]);
    }
    vector<double> l((size_t)n * n, 0.0);
    for (int j = 0; j < n; ++j) {
        double s = m[(size_t)j * n + j] * d[j] * d[j];
        for (int c = 0; c < j; ++c) s -= l[(size_t)j * n + c] * l[(size_t)j * n + c];
        if (!(s > 1e-14)) {
            *err = "the projected mass matrix is singular: the subspace vectors are dependent";
            return false;
        }
        s = std::sqrt(s);
        l[(size_t)j * n + j] = s;
        for (int i = j + 1; i < n; ++i) {
            double v = m[(size_t)i * n + j] * d[i] * d[j];
            for (int c = 0; c < j; ++c) v -= l[(size_t)i * n + c] * l[(size_t)j * n + c];
            l[(size_t)i * n + j] = v / s;
        }
    }
    auto lower_solve = [&](double* b) {
        for (int i = 0; i < n; ++i) {
            double v = b[i];
            for (int c = 0; c < i; ++c) v -= l[(size_t)i * n + c] * b[c];
            b[i] = v / l[(size_t)i * n + i];
        }
    };
    vector<double> w((size_t)n * n), col(n), c((size_t)n * n);
    for (int j = 0; j < n; ++j) {
        for (int i = 0; i < n; ++i) col[i] = k[(size_t)i * n + j] * d[i] * d[j];
        lower_solve(col.data());
        for (int i = 0; i < n; ++i) w[(size_t)i * n + j] = col[i];
    }
    for (int j = 0; j < n; ++j) {
        std::copy(w.begin() + (size_t)j * n, w.begin() + (size_t)(j + 1) * n, col.begin());
        lower_solve(col.data());
        for (int i = 0; i < n; ++i) c[(size_t)i * n + j] = col[i];
    }
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < i; ++j) {
            double v = 0.5 * (c[(size_t)i * n + j] + c[(size_t)j * n + i]);
            c[(size_t)i * n + j] = v;
            c[(size_t)j * n + i] = v;
        }
    vector<double> v((size_t)n * n);
    dense_jacobi(c.data(), n, values, v.data());
    for (int j = 0; j < n; ++j)
        for (int i = n - 1; i >= 0; --i) {
            double s = v[(size_t)i * n + j];
            for (int r = i + 1; r < n; ++r) s -= l[(size_t)r * n + i] * q[(size_t)r * n + j];
            q[(size_t)i * n + j] = s / l[(size_t)i * n + i];
        }
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) q[(size_t)i * n + j] *= d[i];
    return true;
}

}  // namespace orc
