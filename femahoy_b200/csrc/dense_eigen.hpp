// The dense symmetric eigensolvers of the modes (eigen.rs:183-331), host code.
#pragma once
#include <string>
#include <vector>

namespace femgpu {

// The standard problem of the symmetric n x n matrix `a` (row-major, overwritten): the
// eigenvalues ascending and the orthonormal eigenvectors as the columns of `v` (n x n).
void dense_jacobi(double* a, int n, double* values, double* v);
// K q = lambda M q (row-major n x n, M symmetric positive definite): the eigenvalues ascending and
// the vectors as the columns of `q`, with Q^T M Q = I. False, with the reference's text in `err`,
// when M is not positive definite.
bool dense_generalized(const double* k, const double* m, int n, double* values, double* q,
                       std::string* err);

}  // namespace femgpu
