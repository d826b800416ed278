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

// Lowest eigenvalue w and its unit eigenvector v (n entries) of the dense
// symmetric matrix a (n x n column-major): Householder reduction to
// tridiagonal form, bisection for the eigenvalue, inverse iteration for the
// tridiagonal eigenvector, transformed back.  About (4/3) n^3 flops, against
// some 20 n^3 for the full Jacobi solve above.
bool sym_lowest(int n, const double* a, double* w, double* v);

} // namespace dmrgpp

namespace dmrgpp {

// k-th lowest eigenvalue (k >= 1) of the symmetric tridiagonal matrix
// (diagonal d[0..n-1], off-diagonal off[0..n-2]) by bisection on Sturm
// counts (the number of negative pivots of T - x I), to the last bit.
double tridiag_kth_lowest(int n, const double* d, const double* off, int k);

// Unit eigenvector z[0..n-1] for the eigenvalue theta of the same matrix by
// inverse iteration (Gaussian elimination with partial pivoting of
// T - theta I); the component of largest magnitude is made positive.
void tridiag_inverse_iteration(int n, const double* d, const double* off, double theta, double* z);

} // namespace dmrgpp
