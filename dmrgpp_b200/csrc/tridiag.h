// Symmetric tridiagonal eigensolver (tridiag.cpp).
#pragma once

namespace dmrgpp {

// Eigenvalues (ascending, into d) and optionally eigenvectors (z: n x n
// column-major, column i belongs to d[i]) of the symmetric tridiagonal
// matrix with diagonal d[0..n-1] and off-diagonal off[0..n-2].  Returns false
// if the iteration fails to converge.
bool tridiag_eigen(int n, double* d, const double* off, double* z);

} // namespace dmrgpp

namespace dmrgpp {

// Eigenvalues (ascending, w) and eigenvectors (v: n x n column-major) of the
// dense symmetric matrix a (n x n column-major) by cyclic Jacobi rotations.
bool sym_eigen(int n, const double* a, double* w, double* v);

} // namespace dmrgpp
