// Host eigensolvers (tridiag.cpp): symmetric tridiagonal problems of the
// Lanczos and Davidson drivers, and the truncation's density-matrix groups.
#pragma once

#include <vector>

namespace dmrgpp {

// Eigenvalues (ascending, into d) and optionally eigenvectors (z: n x n
// column-major, column i belongs to d[i]) of the symmetric tridiagonal
// matrix with diagonal d[0..n-1] and off-diagonal off[0..n-2].  Returns false
// if the iteration fails to converge.
bool tridiag_eigen(int n, double* d, const double* off, double* z);

// Eigenvalues alone (ascending, into d) of the same tridiagonal matrix by
// the square-root-free QL iteration (rotations of tridiag_eigen where the
// squares would leave the exponent range or the iteration fails).  They
// agree with tridiag_eigen's to rounding (~1e-15 of the norm), not bit for
// bit.  Returns false if neither iteration converges.
bool tridiag_values(int n, double* d, const double* off);

// Unit eigenvectors z (n x k, column-major) of the symmetric tridiagonal
// matrix (d, off) for its eigenvalues w[0..k) (ascending, as computed by
// tridiag_eigen) by inverse iteration: for each, three solves with the LU of
// T - w_j I from a start vector seeded by j, each followed by Gram-Schmidt
// against the earlier vectors of its cluster (eigenvalues closer than
// 1e-3 |T|, the grouping of LAPACK's dstein); the largest component is made
// positive.
void tridiag_eigenvectors(int n, const double* d, const double* off, const double* w, int k, double* z);

// Vectors that start their cluster go four at a time through vector lanes
// (bitwise the one-at-a-time result); 0 turns that off, nonzero (the
// default) on.
void eigenvectors_set_batch(int on);

// Householder reduction T = Q^T A Q of the dense symmetric n x n matrix a
// (column-major, n >= 2), Q = P_0 ... P_{n-3}, P_k = I - beta_k h_k h_k^T
// acting on entries k+1..n-1 with h_k(0) = 1: diagonal d (n), off-diagonal
// off (n - 1), reflectors hv (n x n, column k holds h_k) and beta (n).
void householder_tridiag(int n, const double* a, std::vector<double>& d, std::vector<double>& off,
                         std::vector<double>& hv, std::vector<double>& beta);

// The same reduction by a team of `threads` host threads (the caller's
// thread included; below 64 rows or 2 threads, householder_tridiag).  The
// sums of the threads' parts make its rounding depend on the thread count.
void householder_tridiag_parallel(int n, const double* a, std::vector<double>& d, std::vector<double>& off,
                                  std::vector<double>& hv, std::vector<double>& beta, int threads);

// The instruction set of the reductions' passes over the trailing block:
// nonzero (the default) uses AVX2 where the host has it, 0 the baseline
// x86-64 build; both round identically (tests compare them).
void householder_set_isa(int avx2);

// One matrix's Householder reduction (the outputs of householder_tridiag;
// n = 1: d = {a}, off = {0}, no reflectors) and whether the QL iteration on
// it converged.  d and off are those of 2^shift A: a matrix whose largest
// entry lies outside [2^-64, 2^64] (a group of negligible weight, say) is
// reduced scaled by a power of two, exactly, which leaves the reflectors as
// they are.
struct GroupReduction {
	std::vector<double> d, off, hv, beta;
	std::vector<double> scaled_values; // shift != 0: the eigenvalues of 2^shift A
	int                 shift = 0;
	bool                ok    = true;
};

// Eigenvalues of ng dense symmetric matrices on `threads` host threads:
// a[g] (n[g] x n[g], column-major; symmetrised in place as (a + a^T) / 2)
// is reduced to tridiagonal form (red[g]) and its eigenvalues go, ascending,
// to w[g].  When the largest matrix is a large share of the work, a team of
// threads shares each of its Householder steps while the other threads take
// the remaining matrices one at a time, largest first; the team joins them
// when it is done.  w[g] holds the eigenvalues of a[g] itself (scaled back
// from 2^shift a[g]).  Returns false if an iteration did not converge (that
// group's ok is false).
bool group_eigenvalues(size_t ng, const size_t* n, double* const* a, double* const* w,
                       std::vector<GroupReduction>& red, int threads);

// tridiag_eigenvectors of the tridiagonals red[g] for k[g] eigenvalues
// w[g][0..k[g]) (of the unscaled matrices, as group_eigenvalues returns
// them: the group's largest; a scaled group uses its scaled_values instead)
// into z[g] (n[g] x k[g]), all groups on `threads` threads:
// the vectors of a group go in runs cut only where a cluster ends, so the
// result is the serial one whatever the thread count.
void group_eigenvectors(size_t ng, const size_t* n, const size_t* k, const GroupReduction* red,
                        const double* const* w, double* const* z, int threads);

// v (n x ncols, column-major) <- Q v for the reflectors of householder_tridiag.
void apply_q(int n, const std::vector<double>& hv, const std::vector<double>& beta, double* v, int ncols);

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

// All eigenvalues (ascending, w) and, when v != NULL, the eigenvectors (v:
// n x n column-major, column i belongs to w[i]) of the dense symmetric matrix
// a by Householder reduction and the implicit QL iteration of tridiag_eigen;
// about 6 n^3 flops.  Returns false if the QL iteration fails to converge.
bool sym_eigen_full(int n, const double* a, double* w, double* v);

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

// The lowest eigenpair of the symmetric tridiagonal (d, off): *theta the
// lowest of tridiag_eigen's eigenvalues (bitwise), z (n) its unit
// eigenvector by tridiag_inverse_iteration, O(n), when the next eigenvalue
// lies more than 1e-8 max(1, |T|) above it; otherwise (a near-degenerate
// pair, or copies of a converged value from a Lanczos run without
// reorthogonalisation) the first of tridiag_eigen's eigenvectors, O(n^3).
// Returns false if the QL iteration fails.
bool tridiag_lowest(int n, const double* d, const double* off, double* theta, double* z);

} // namespace dmrgpp
