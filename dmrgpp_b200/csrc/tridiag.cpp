// Host eigensolvers in FP64: the tridiagonal problems of the Lanczos and
// Davidson drivers, and the density-matrix groups of the truncation.
//
// The reference obtains the Ritz values of its Lanczos tridiagonal with
// LAPACK dstedc (PsimagLite/src/PsimagLite/TridiagonalMatrix.cpp:21) and the
// Ritz vectors from a dense symmetric eigensolve of the same matrix
// (LanczosSolver.h:76-84).  Here both come from one implementation of the
// implicit QL algorithm with shifts taken from the leading 2x2 block
// (Bowdler, Martin, Reinsch and Wilkinson, Numer. Math. 11 (1968) 293-306;
// Golub and Van Loan, Matrix Computations, section 8.3); the lowest Ritz
// vector alone by inverse iteration.  The truncation's groups (the
// reference's per-group SVD, DensityMatrixSvd.h:355-410) go through a
// Householder reduction to tridiagonal form (vectorised passes, a thread
// team for the largest group), the square-root-free QL for the eigenvalues
// and inverse iteration for the kept eigenvectors, spread over the host's
// threads.
#include "tridiag.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <random>
#include <atomic>
#include <thread>
#include <vector>

namespace dmrgpp {

namespace {

// The implicit QL iteration on (d, off); every plane rotation is passed to
// rot(i, c, s) in the order applied (it maps columns i, i+1 of the
// eigenvector matrix: z_{i+1} <- s z_i + c z_{i+1}, z_i <- c z_i - s z_{i+1}).
// d ends as the eigenvalues, unsorted.  Kept as a template so that the
// eigenvalue-only solve skips the vector update entirely.
// sqrt(a^2 + b^2), through std::hypot only where the squares could over- or
// underflow
inline double safe_hypot(double a, double b)
{
	const double s = a * a + b * b;
	return (s > 1e-280 && s < 1e280) ? std::sqrt(s) : std::hypot(a, b);
}

template <class Rot> bool ql_iterate(int n, double* d, const double* off, Rot rot)
{
	std::vector<double> e(size_t(n), 0.0);
	for (int i = 0; i + 1 < n; ++i)
		e[size_t(i)] = off[i];
	// an off-diagonal element is negligible against its two diagonal
	// neighbours or against the norm of the whole matrix (the norm-based test
	// of the EISPACK tql2 routine): eigenvalues far below the norm, as in a
	// density matrix of low rank, carry rounding noise of the order of
	// eps * norm and a purely local test would never accept them
	double anorm = 0.0;
	for (int i = 0; i < n; ++i)
		anorm = std::max(anorm, std::fabs(d[i]) + std::fabs(e[size_t(i)]));
	for (int l = 0; l < n; ++l) {
		int iter = 0;
		for (;;) {
			// smallest m >= l whose off-diagonal element is negligible
			int m = l;
			for (; m + 1 < n; ++m) {
				const double dd = std::fabs(d[m]) + std::fabs(d[m + 1]);
				const double em = std::fabs(e[size_t(m)]);
				if (em <= DBL_EPSILON * dd || em <= DBL_EPSILON * anorm)
					break;
			}
			if (m == l)
				break;
			if (++iter > 60)
				return false;
			// shift: eigenvalue of the leading 2x2 block closer to d[l]
			double g = (d[l + 1] - d[l]) / (2.0 * e[size_t(l)]);
			double r = safe_hypot(g, 1.0);
			g        = d[m] - d[l] + e[size_t(l)] / (g + std::copysign(r, g));
			double s = 1.0, c = 1.0, p = 0.0;
			bool   split = false;
			for (int i = m - 1; i >= l; --i) {
				const double f = s * e[size_t(i)];
				const double b = c * e[size_t(i)];
				r              = safe_hypot(f, g);
				e[size_t(i) + 1] = r;
				if (r == 0.0) { // underflow: the block splits, restart on it
					d[i + 1] -= p;
					e[size_t(m)] = 0.0;
					split        = true;
					break;
				}
				s        = f / r;
				c        = g / r;
				g        = d[i + 1] - p;
				r        = (d[i] - g) * s + 2.0 * c * b;
				p        = s * r;
				d[i + 1] = g + p;
				g        = c * r - b;
				rot(i, c, s);
			}
			if (split)
				continue;
			d[l] -= p;
			e[size_t(l)] = g;
			e[size_t(m)] = 0.0;
		}
	}
	return true;
}

// Eigenvalues alone by the square-root-free QL iteration of Pal, Walker and
// Kahan (B. N. Parlett, The Symmetric Eigenvalue Problem, section 8.15):
// the sweep runs on the squared off-diagonal elements e2 with the squared
// cosine and sine of each rotation, so a rotation costs divisions but no
// square root (one per sweep, for the shift).  Shifts and deflation tests
// are those of ql_iterate (squared).  Each step forms both p / r and r / p
// from the same operands, so the next p = gamma^2 / c^2 = gamma^2 (r / p)
// waits for one division instead of two.  The squares need the matrix norm
// well inside the exponent range (callers check).  d ends unsorted.
bool ql_values_rootfree(int n, double* d, const double* off, double anorm)
{
	std::vector<double> e2(size_t(n), 0.0);
	for (int i = 0; i + 1 < n; ++i)
		e2[size_t(i)] = off[i] * off[i];
	const double eps2 = DBL_EPSILON * DBL_EPSILON, tn = eps2 * anorm * anorm;
	for (int l = 0; l < n; ++l) {
		int iter = 0;
		for (;;) {
			int m = l;
			for (; m + 1 < n; ++m) {
				const double dd = std::fabs(d[m]) + std::fabs(d[m + 1]);
				if (e2[size_t(m)] <= eps2 * dd * dd || e2[size_t(m)] <= tn)
					break;
			}
			if (m == l)
				break;
			if (++iter > 60)
				return false;
			// shift: eigenvalue of the leading 2x2 block closer to d[l]
			const double el    = std::sqrt(e2[size_t(l)]);
			const double t     = (d[l + 1] - d[l]) / (2.0 * el);
			const double sigma = d[l] - el / (t + std::copysign(safe_hypot(t, 1.0), t));
			double       c2 = 1.0, s2 = 0.0, gamma = d[m] - sigma, p = gamma * gamma;
			for (int i = m - 1; i >= l; --i) {
				const double bb = e2[size_t(i)], r = p + bb;
				if (i != m - 1)
					e2[size_t(i) + 1] = s2 * r;
				const double oldc = c2, q = r / p;
				c2                = p / r;
				s2                = bb / r;
				const double oldg = gamma, alpha = d[i];
				gamma             = c2 * (alpha - sigma) - s2 * oldg;
				d[i + 1]          = oldg + (alpha - gamma);
				p                 = c2 != 0.0 ? gamma * gamma * q : oldc * bb;
			}
			e2[size_t(l)] = s2 * p;
			d[l]          = sigma + gamma;
		}
	}
	return true;
}

} // namespace

bool tridiag_values(int n, double* d, const double* off)
{
	if (n <= 0)
		return true;
	double anorm = 0.0;
	for (int i = 0; i < n; ++i)
		anorm = std::max(anorm, std::fabs(d[i]) + (i + 1 < n ? std::fabs(off[i]) : 0.0));
	std::vector<double> d0(d, d + n);
	if (!(anorm > 1e-100 && anorm < 1e100) || !ql_values_rootfree(n, d, off, anorm)) {
		// outside the range of the squares, or no convergence: the QL
		// iteration with rotations from the same input
		std::copy(d0.begin(), d0.end(), d);
		if (!ql_iterate(n, d, off, [](int, double, double) {}))
			return false;
	}
	std::sort(d, d + n);
	return true;
}

bool tridiag_eigen(int n, double* d, const double* off, double* z)
{
	if (n <= 0)
		return true;
	if (z) {
		std::fill(z, z + size_t(n) * size_t(n), 0.0);
		for (int i = 0; i < n; ++i)
			z[size_t(i) + size_t(i) * size_t(n)] = 1.0;
	}
	const bool ok = ql_iterate(n, d, off, [&](int i, double c, double s) {
		if (!z)
			return;
		double* zi  = z + size_t(i) * size_t(n);
		double* zi1 = zi + size_t(n);
		for (int k = 0; k < n; ++k) {
			const double t = zi1[k];
			zi1[k]         = s * zi[k] + c * t;
			zi[k]          = c * zi[k] - s * t;
		}
	});
	if (!ok)
		return false;
	// ascending order, vectors follow their values
	std::vector<int> order(static_cast<size_t>(n));
	std::iota(order.begin(), order.end(), 0);
	std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return d[a] < d[b]; });
	std::vector<double> dv(d, d + n);
	for (int i = 0; i < n; ++i)
		d[i] = dv[size_t(order[size_t(i)])];
	if (z) {
		std::vector<double> zv(z, z + size_t(n) * size_t(n));
		for (int i = 0; i < n; ++i)
			std::copy(zv.begin() + size_t(order[size_t(i)]) * size_t(n),
			          zv.begin() + size_t(order[size_t(i)] + 1) * size_t(n),
			          z + size_t(i) * size_t(n));
	}
	return true;
}

} // namespace dmrgpp

namespace dmrgpp {

bool sym_eigen(int n, const double* a, double* w, double* v)
{
	// cyclic Jacobi rotations (Golub and Van Loan, section 8.5): robust and
	// accurate for the small projected matrices of the Davidson solver
	std::vector<double> m(a, a + size_t(n) * size_t(n));
	for (int i = 0; i < n; ++i)
		for (int j = 0; j < n; ++j)
			v[size_t(i) + size_t(j) * size_t(n)] = (i == j) ? 1.0 : 0.0;
	auto M = [&](int i, int j) -> double& { return m[size_t(i) + size_t(j) * size_t(n)]; };
	auto V = [&](int i, int j) -> double& { return v[size_t(i) + size_t(j) * size_t(n)]; };
	for (int sweep = 0; sweep < 100; ++sweep) {
		double off = 0.0, tot = 0.0;
		for (int i = 0; i < n; ++i)
			for (int j = 0; j < n; ++j) {
				tot += M(i, j) * M(i, j);
				if (i != j)
					off += M(i, j) * M(i, j);
			}
		if (off <= 1e-30 * tot || off == 0.0)
			break;
		for (int p = 0; p < n - 1; ++p)
			for (int q = p + 1; q < n; ++q) {
				const double apq = M(p, q);
				if (apq == 0.0)
					continue;
				const double theta = (M(q, q) - M(p, p)) / (2.0 * apq);
				const double t     = std::copysign(1.0, theta) / (std::fabs(theta) + std::hypot(theta, 1.0));
				const double c     = 1.0 / std::hypot(t, 1.0);
				const double s     = t * c;
				for (int k = 0; k < n; ++k) { // columns p, q
					const double mkp = M(k, p), mkq = M(k, q);
					M(k, p)          = c * mkp - s * mkq;
					M(k, q)          = s * mkp + c * mkq;
				}
				for (int k = 0; k < n; ++k) { // rows p, q
					const double mpk = M(p, k), mqk = M(q, k);
					M(p, k)          = c * mpk - s * mqk;
					M(q, k)          = s * mpk + c * mqk;
				}
				for (int k = 0; k < n; ++k) {
					const double vkp = V(k, p), vkq = V(k, q);
					V(k, p)          = c * vkp - s * vkq;
					V(k, q)          = s * vkp + c * vkq;
				}
			}
	}
	std::vector<int> order(static_cast<size_t>(n));
	std::iota(order.begin(), order.end(), 0);
	std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return M(x, x) < M(y, y); });
	std::vector<double> vv(v, v + size_t(n) * size_t(n));
	for (int i = 0; i < n; ++i) {
		w[i] = M(order[size_t(i)], order[size_t(i)]);
		std::copy(vv.begin() + size_t(order[size_t(i)]) * size_t(n),
		          vv.begin() + size_t(order[size_t(i)] + 1) * size_t(n), v + size_t(i) * size_t(n));
	}
	return true;
}

} // namespace dmrgpp

namespace dmrgpp {

namespace {

// number of eigenvalues of T below x
int sturm_count(int n, const double* d, const double* off, double x, double tiny)
{
	int    count = 0;
	double q     = d[0] - x;
	for (int i = 0;; ++i) {
		if (q == 0.0)
			q = -tiny;
		if (q < 0.0)
			++count;
		if (i + 1 == n)
			break;
		q = d[i + 1] - x - off[i] * off[i] / q;
	}
	return count;
}

} // namespace

double tridiag_kth_lowest(int n, const double* d, const double* off, int k)
{
	if (n <= 0)
		return 0.0;
	double lo = d[0], hi = d[0], scale = 0.0;
	for (int i = 0; i < n; ++i) { // Gershgorin bounds
		const double r = (i > 0 ? std::fabs(off[i - 1]) : 0.0) + (i + 1 < n ? std::fabs(off[i]) : 0.0);
		lo             = std::min(lo, d[i] - r);
		hi             = std::max(hi, d[i] + r);
		scale          = std::max(scale, std::fabs(d[i]) + r);
	}
	const double tiny = std::max(scale, 1.0) * 1e-300;
	lo -= 1e-14 * std::max(scale, 1.0);
	hi += 1e-14 * std::max(scale, 1.0);
	for (int it = 0; it < 400; ++it) {
		const double mid = 0.5 * (lo + hi);
		if (mid <= lo || mid >= hi)
			break;
		if (sturm_count(n, d, off, mid, tiny) >= k)
			hi = mid;
		else
			lo = mid;
	}
	return 0.5 * (lo + hi);
}

void tridiag_inverse_iteration(int n, const double* d, const double* off, double theta, double* z)
{
	if (n == 1) {
		z[0] = 1.0;
		return;
	}
	double scale = 0.0;
	for (int i = 0; i < n; ++i)
		scale = std::max(scale, std::fabs(d[i] - theta) + (i + 1 < n ? std::fabs(off[i]) : 0.0));
	const double tiny = std::max(scale, 1e-300) * 1e-15;
	// LU of T - theta I with row interchanges: U row i = (u0, u1, u2) at
	// columns i, i+1, i+2; the multipliers and swaps replay on the rhs
	std::vector<double> u0(static_cast<size_t>(n)), u1(static_cast<size_t>(n), 0.0), u2(static_cast<size_t>(n), 0.0), m(static_cast<size_t>(n), 0.0);
	std::vector<char>   sw(size_t(n), 0);
	double              a = d[0] - theta, b = off[0];
	for (int i = 0; i + 1 < n; ++i) {
		const double l = off[i], dd = d[i + 1] - theta, u = i + 2 < n ? off[i + 1] : 0.0;
		if (std::fabs(a) >= std::fabs(l)) {
			if (a == 0.0)
				a = tiny;
			u0[size_t(i)] = a;
			u1[size_t(i)] = b;
			m[size_t(i)]  = l / a;
			a             = dd - m[size_t(i)] * b;
			b             = u;
		} else {
			u0[size_t(i)] = l;
			u1[size_t(i)] = dd;
			u2[size_t(i)] = u;
			m[size_t(i)]  = a / l;
			sw[size_t(i)] = 1;
			const double na = b - m[size_t(i)] * dd;
			b               = -m[size_t(i)] * u;
			a               = na;
		}
	}
	u0[size_t(n - 1)] = a == 0.0 ? tiny : a;
	for (int i = 0; i < n; ++i)
		z[i] = 1.0 / std::sqrt(double(n));
	for (int iter = 0; iter < 3; ++iter) {
		// forward: apply the swaps and multipliers to the rhs
		for (int i = 0; i + 1 < n; ++i) {
			if (sw[size_t(i)]) {
				const double t = z[i];
				z[i]           = z[i + 1];
				z[i + 1]       = t - m[size_t(i)] * z[i + 1];
			} else {
				z[i + 1] -= m[size_t(i)] * z[i];
			}
		}
		// back substitution
		for (int i = n - 1; i >= 0; --i) {
			double s = z[i];
			if (i + 1 < n)
				s -= u1[size_t(i)] * z[i + 1];
			if (i + 2 < n)
				s -= u2[size_t(i)] * z[i + 2];
			z[i] = s / u0[size_t(i)];
		}
		double nrm = 0.0, big = 0.0;
		int    arg = 0;
		for (int i = 0; i < n; ++i) {
			nrm += z[i] * z[i];
			if (std::fabs(z[i]) > big) {
				big = std::fabs(z[i]);
				arg = i;
			}
		}
		const double f = (z[arg] < 0.0 ? -1.0 : 1.0) / std::sqrt(nrm);
		for (int i = 0; i < n; ++i)
			z[i] *= f;
	}
}

bool tridiag_lowest(int n, const double* d, const double* off, double* theta, double* z)
{
	if (n <= 0)
		return true;
	std::vector<double> ev(d, d + n);
	if (!tridiag_eigen(n, ev.data(), off, nullptr))
		return false;
	*theta = ev[0];
	double norm = 0.0;
	for (double x : ev)
		norm = std::max(norm, std::fabs(x));
	if (n == 1 || ev[1] - ev[0] > 1e-8 * std::max(1.0, norm)) {
		tridiag_inverse_iteration(n, d, off, ev[0], z);
		return true;
	}
	// the two lowest coincide: every eigenvector by QL, the first one kept
	std::vector<double> dv(d, d + n), zz(size_t(n) * size_t(n));
	if (!tridiag_eigen(n, dv.data(), off, zz.data()))
		return false;
	std::copy(zz.begin(), zz.begin() + n, z);
	return true;
}

} // namespace dmrgpp

namespace dmrgpp {

namespace {

// Four doubles at any 8-byte alignment (GCC vector extension; SSE2 pairs in
// the baseline build, one AVX register in the AVX2 clone below).  The
// helpers taking and returning them are always inlined, so the note that
// their calling convention differs between the two builds does not apply.
#pragma GCC diagnostic ignored "-Wpsabi"
// They may alias plain doubles: scratch arrays of them live in
// std::vector<double> storage.
typedef double v4d __attribute__((vector_size(32), aligned(8), may_alias));

inline __attribute__((always_inline)) v4d load4(const double* x)
{
	v4d v;
	std::memcpy(&v, x, sizeof v);
	return v;
}
inline __attribute__((always_inline)) void store4(double* x, const v4d& v) { std::memcpy(x, &v, sizeof v); }
inline __attribute__((always_inline)) double hsum(const v4d& v) { return (v[0] + v[1]) + (v[2] + v[3]); }

// One pass of a Householder step over columns [c0, c1) of the lower triangle
// of the trailing block (len x len; column j at a + j * ld, rows i >= j).
// UPD: the previous step's rank-2 update, A(i, j) -= hp[i] qp[j] + qp[i] hp[j].
// PROD: then this step's product p += A h, from the lower triangle alone:
// p[i] += A(i, j) h[j] (i >= j) and p[j] += A(i, j) h[i] (i > j).
// Columns go in pairs that share the loads of hp, qp, h and p; the order of
// every sum is fixed, and neither target (baseline x86-64, AVX2 without
// FMA) has fused multiply-add instructions that GCC could contract the
// products and sums into, so both instruction-set builds round alike.
template <bool UPD, bool PROD>
inline __attribute__((always_inline)) void pass_cols(int len, double* a, size_t ld, int c0, int c1, const double* hp,
                                                     const double* qp, const double* h, double* p)
{
	int j = c0;
	for (; j + 1 < c1; j += 2) {
		double*      x0 = a + size_t(j) * ld;
		double*      x1 = x0 + ld;
		const double q0 = UPD ? qp[j] : 0.0, g0 = UPD ? hp[j] : 0.0;
		const double q1 = UPD ? qp[j + 1] : 0.0, g1 = UPD ? hp[j + 1] : 0.0;
		const double h0 = PROD ? h[j] : 0.0, h1 = PROD ? h[j + 1] : 0.0;
		if (UPD) {
			x0[j] -= hp[j] * q0 + qp[j] * g0;
			x0[j + 1] -= hp[j + 1] * q0 + qp[j + 1] * g0;
			x1[j + 1] -= hp[j + 1] * q1 + qp[j + 1] * g1;
		}
		double s0 = 0.0, s1 = 0.0;
		if (PROD) {
			s0 = x0[j] * h0 + x0[j + 1] * h1;
			s1 = x1[j + 1] * h1;
			p[j + 1] += x0[j + 1] * h0;
		}
		v4d vs0 = { 0.0, 0.0, 0.0, 0.0 }, vs1 = vs0;
		int i   = j + 2;
		for (; i + 4 <= len; i += 4) {
			v4d a0 = load4(x0 + i), a1 = load4(x1 + i);
			if (UPD) {
				const v4d vh = load4(hp + i), vq = load4(qp + i);
				a0 -= vh * q0 + vq * g0;
				a1 -= vh * q1 + vq * g1;
				store4(x0 + i, a0);
				store4(x1 + i, a1);
			}
			if (PROD) {
				const v4d vx = load4(h + i);
				vs0 += a0 * vx;
				vs1 += a1 * vx;
				store4(p + i, load4(p + i) + (a0 * h0 + a1 * h1));
			}
		}
		for (; i < len; ++i) {
			double a0 = x0[i], a1 = x1[i];
			if (UPD) {
				a0 -= hp[i] * q0 + qp[i] * g0;
				a1 -= hp[i] * q1 + qp[i] * g1;
				x0[i] = a0;
				x1[i] = a1;
			}
			if (PROD) {
				s0 += a0 * h[i];
				s1 += a1 * h[i];
				p[i] += a0 * h0 + a1 * h1;
			}
		}
		if (PROD) {
			p[j] += s0 + hsum(vs0);
			p[j + 1] += s1 + hsum(vs1);
		}
	}
	if (j < c1) { // an odd last column
		double*      x  = a + size_t(j) * ld;
		const double q0 = UPD ? qp[j] : 0.0, g0 = UPD ? hp[j] : 0.0, h0 = PROD ? h[j] : 0.0;
		double       s  = 0.0;
		for (int i = j; i < len; ++i) {
			double v = x[i];
			if (UPD) {
				v -= hp[i] * q0 + qp[i] * g0;
				x[i] = v;
			}
			if (PROD) {
				if (i > j) {
					s += v * h[i];
					p[i] += v * h0;
				} else {
					s += v * h0;
				}
			}
		}
		if (PROD)
			p[j] += s;
	}
}

template <class... Args> inline __attribute__((always_inline)) void pass_any(bool upd, bool prod, Args... args)
{
	if (upd && prod)
		pass_cols<true, true>(args...);
	else if (upd)
		pass_cols<true, false>(args...);
	else if (prod)
		pass_cols<false, true>(args...);
}

__attribute__((target("avx2"))) void pass_avx2(bool upd, bool prod, int len, double* a, size_t ld, int c0, int c1,
                                               const double* hp, const double* qp, const double* h, double* p)
{
	pass_any(upd, prod, len, a, ld, c0, c1, hp, qp, h, p);
}

void pass_base(bool upd, bool prod, int len, double* a, size_t ld, int c0, int c1, const double* hp,
               const double* qp, const double* h, double* p)
{
	pass_any(upd, prod, len, a, ld, c0, c1, hp, qp, h, p);
}

bool host_has_avx2()
{
	static const bool yes = [] {
		__builtin_cpu_init();
		return bool(__builtin_cpu_supports("avx2"));
	}();
	return yes;
}

// the instruction set of trailing_pass: AVX2 where the host has it (the two
// builds give identical results); 0 forces the baseline build
std::atomic<int> g_pass_isa { 1 };

void trailing_pass(bool upd, bool prod, int len, double* a, size_t ld, int c0, int c1, const double* hp,
                   const double* qp, const double* h, double* p)
{
	if (g_pass_isa.load(std::memory_order_relaxed) && host_has_avx2())
		pass_avx2(upd, prod, len, a, ld, c0, c1, hp, qp, h, p);
	else
		pass_base(upd, prod, len, a, ld, c0, c1, hp, qp, h, p);
}

} // namespace

void householder_set_isa(int avx2) { g_pass_isa.store(avx2 ? 1 : 0); }

// Householder reduction T = Q^T A Q of the dense symmetric n x n matrix a
// (column-major), Q = P_0 P_1 ... P_{n-3}, P_k = I - beta_k h_k h_k^T acting
// on rows / columns k+1..n-1 with h_k(0) = 1 (Golub and Van Loan, algorithms
// 5.1.1 and 8.3.1): diagonal d, off-diagonal off (n - 1), reflectors hv
// (column k holds h_k) and beta.  n >= 2.
void householder_tridiag(int n, const double* a, std::vector<double>& d, std::vector<double>& off,
                         std::vector<double>& hv, std::vector<double>& beta)
{
	// Only the lower triangle of the (symmetric) trailing block is kept, and
	// the rank-2 update of step k - 1 is applied in the same pass over it
	// that forms step k's product p = beta A22 h: one read and one write of
	// the lower triangle per step.
	const size_t        N = size_t(n);
	std::vector<double> m(a, a + N * N), p(N), q(N), qprev(N), hprev(N);
	d.assign(N, 0.0);
	off.assign(N - 1, 0.0);
	hv.assign(N * N, 0.0);
	beta.assign(N, 0.0);
	auto M       = [&](int i, int j) -> double& { return m[size_t(i) + size_t(j) * N]; };
	bool pending = false; // update A <- A - h' q'^T - q' h'^T on rows / columns >= k
	for (int k = 0; k + 2 < n; ++k) {
		const int len = n - k - 1;
		// bring column k (rows >= k) up to date; h', q' index 0 is row k
		if (pending) {
			const double hk = hprev[0], qk = qprev[0];
			for (int i = 0; i <= len; ++i)
				M(k + i, k) -= hprev[size_t(i)] * qk + qprev[size_t(i)] * hk;
		}
		double* h     = hv.data() + size_t(k) * N; // h[0..len)
		double  sigma = 0.0;
		for (int i = 1; i < len; ++i)
			sigma += M(k + 1 + i, k) * M(k + 1 + i, k);
		const double x0 = M(k + 1, k);
		d[size_t(k)]    = M(k, k);
		double b        = 0.0;
		if (sigma == 0.0) { // already tridiagonal in this column
			off[size_t(k)] = x0;
		} else {
			const double mu = std::sqrt(x0 * x0 + sigma);
			const double h0 = x0 <= 0.0 ? x0 - mu : -sigma / (x0 + mu);
			b               = 2.0 * h0 * h0 / (sigma + h0 * h0);
			beta[size_t(k)] = b;
			h[0]            = 1.0;
			for (int i = 1; i < len; ++i)
				h[i] = M(k + 1 + i, k) / h0;
			off[size_t(k)] = mu;
		}
		// one pass over the lower triangle of A22 (rows / columns >= k+1):
		// the pending update, then p += A22 h with the updated entries
		std::fill(p.begin(), p.begin() + len, 0.0);
		trailing_pass(pending, b != 0.0, len, &M(k + 1, k + 1), N, 0, len, hprev.data() + 1, qprev.data() + 1, h,
		              p.data());
		pending = b != 0.0;
		if (!pending)
			continue;
		// p = beta A22 h, w = p - (beta / 2)(p^T h) h: the update of this step
		double ph = 0.0;
		for (int i = 0; i < len; ++i) {
			p[size_t(i)] *= b;
			ph += p[size_t(i)] * h[i];
		}
		for (int i = 0; i < len; ++i) {
			qprev[size_t(i)] = p[size_t(i)] - 0.5 * b * ph * h[i];
			hprev[size_t(i)] = h[i];
		}
	}
	if (pending) { // the last update reaches the trailing 2 x 2 block
		const int k0 = n - 2; // hprev index 0 is row n - 2
		for (int j = 0; j < 2; ++j)
			for (int i = j; i < 2; ++i)
				M(k0 + i, k0 + j) -= hprev[size_t(i)] * qprev[size_t(j)] + qprev[size_t(i)] * hprev[size_t(j)];
	}
	d[N - 2]   = M(n - 2, n - 2);
	d[N - 1]   = M(n - 1, n - 1);
	off[N - 2] = M(n - 1, n - 2);
}

namespace {

// A sense-reversing spin barrier for a fixed team of threads (the parallel
// reduction below synchronises three times per Householder step, too often
// for a condition variable).
class SpinBarrier {
public:
	explicit SpinBarrier(int n)
	    : n_(n)
	{
	}
	void wait()
	{
		const int gen = gen_.load(std::memory_order_acquire);
		if (count_.fetch_add(1, std::memory_order_acq_rel) == n_ - 1) {
			count_.store(0, std::memory_order_relaxed);
			gen_.store(gen + 1, std::memory_order_release);
			return;
		}
		while (gen_.load(std::memory_order_acquire) == gen)
			std::this_thread::yield();
	}

private:
	const int        n_;
	std::atomic<int> count_ { 0 };
	std::atomic<int> gen_ { 0 };
};

} // namespace

void householder_tridiag_parallel(int n, const double* a, std::vector<double>& d, std::vector<double>& off,
                                  std::vector<double>& hv, std::vector<double>& beta, int threads)
{
	if (threads < 2 || n < 64) {
		householder_tridiag(n, a, d, off, hv, beta);
		return;
	}
	// householder_tridiag's one-pass scheme with the pass over the lower
	// triangle split by columns into equal areas; each thread accumulates its
	// own part of p, and the parts are summed in thread order
	const size_t                     N = size_t(n);
	const int                        T = threads;
	std::vector<double>              m(a, a + N * N), p(N), hprev(N), qprev(N);
	std::vector<std::vector<double>> part(static_cast<size_t>(T), std::vector<double>(N));
	d.assign(N, 0.0);
	off.assign(N - 1, 0.0);
	hv.assign(N * N, 0.0);
	beta.assign(N, 0.0);
	auto        M       = [&](int i, int j) -> double& { return m[size_t(i) + size_t(j) * N]; };
	bool        pending = false;
	double      b       = 0.0;
	SpinBarrier bar(T);
	// thread 0, between passes: the end of step k - 1 (its update vectors)
	// and the start of step k (column k brought up to date, reflector k)
	auto serial = [&](int k) {
		const int len = n - k - 1;
		if (pending) {
			const double hk = hprev[0], qk = qprev[0];
			for (int i = 0; i <= len; ++i)
				M(k + i, k) -= hprev[size_t(i)] * qk + qprev[size_t(i)] * hk;
		}
		double* h     = hv.data() + size_t(k) * N;
		double  sigma = 0.0;
		for (int i = 1; i < len; ++i)
			sigma += M(k + 1 + i, k) * M(k + 1 + i, k);
		const double x0 = M(k + 1, k);
		d[size_t(k)]    = M(k, k);
		b               = 0.0;
		if (sigma == 0.0) {
			off[size_t(k)] = x0;
		} else {
			const double mu = std::sqrt(x0 * x0 + sigma);
			const double h0 = x0 <= 0.0 ? x0 - mu : -sigma / (x0 + mu);
			b               = 2.0 * h0 * h0 / (sigma + h0 * h0);
			beta[size_t(k)] = b;
			h[0]            = 1.0;
			for (int i = 1; i < len; ++i)
				h[i] = M(k + 1 + i, k) / h0;
			off[size_t(k)] = mu;
		}
	};
	auto finish_step = [&](int k) { // thread 0, after the reduction of p
		const int     len = n - k - 1;
		const double* h   = hv.data() + size_t(k) * N;
		const bool    had = pending;
		pending           = b != 0.0;
		if (!pending)
			return had;
		double ph = 0.0;
		for (int i = 0; i < len; ++i) {
			p[size_t(i)] *= b;
			ph += p[size_t(i)] * h[i];
		}
		for (int i = 0; i < len; ++i) {
			qprev[size_t(i)] = p[size_t(i)] - 0.5 * b * ph * h[i];
			hprev[size_t(i)] = h[i];
		}
		return had;
	};
	auto worker = [&](int t) {
		for (int k = 0; k + 2 < n; ++k) {
			if (t == 0)
				serial(k);
			bar.wait();
			const int     len = n - k - 1;
			const double* h   = hv.data() + size_t(k) * N;
			const double* hp  = hprev.data() + 1;
			const double* qp  = qprev.data() + 1;
			// columns [c0, c1) of the trailing block: equal shares of its
			// lower-triangle area len (len + 1) / 2
			auto col_of = [&](int share) {
				if (share <= 0)
					return 0;
				if (share >= T)
					return len;
				const double target = double(share) / T * 0.5 * double(len) * double(len + 1);
				// area of columns [0, c) is c * len - c (c - 1) / 2
				const double L  = double(len) + 0.5;
				const double c  = L - std::sqrt(std::max(0.0, L * L - 2.0 * target));
				return std::min(len, std::max(0, int(c)));
			};
			const int c0 = col_of(t), c1 = col_of(t + 1);
			double*   pt = part[size_t(t)].data();
			std::fill(pt, pt + len, 0.0);
			trailing_pass(pending, b != 0.0, len, &M(k + 1, k + 1), N, c0, c1, hp, qp, h, pt);
			bar.wait();
			// p = sum of the parts, rows split among the threads
			const int r0 = int((long long)len * t / T), r1 = int((long long)len * (t + 1) / T);
			for (int i = r0; i < r1; ++i) {
				double sum = 0.0;
				for (int q = 0; q < T; ++q)
					sum += part[size_t(q)][size_t(i)];
				p[size_t(i)] = sum;
			}
			bar.wait();
			if (t == 0)
				finish_step(k);
		}
	};
	std::vector<std::thread> team;
	for (int t = 1; t < T; ++t)
		team.emplace_back(worker, t);
	worker(0);
	for (std::thread& th : team)
		th.join();
	if (pending) { // the last update reaches the trailing 2 x 2 block
		const int k0 = n - 2;
		for (int j = 0; j < 2; ++j)
			for (int i = j; i < 2; ++i)
				M(k0 + i, k0 + j) -= hprev[size_t(i)] * qprev[size_t(j)] + qprev[size_t(i)] * hprev[size_t(j)];
	}
	d[N - 2]   = M(n - 2, n - 2);
	d[N - 1]   = M(n - 1, n - 1);
	off[N - 2] = M(n - 1, n - 2);
}

namespace {

// the team that shares the Householder steps of the largest matrix: about
// twice its share of the flops (a team of T runs at roughly T / 2 times one
// thread), at most half the threads and at most 8 (three barriers per step
// cost more than a larger team saves); none below 128 rows
int team_size(size_t ng, const size_t* n, size_t big, int threads)
{
	if (threads < 4 || n[big] < 128)
		return 0;
	double all = 0.0;
	for (size_t g = 0; g < ng; ++g)
		all += double(n[g]) * double(n[g]) * double(n[g]);
	const double share = double(n[big]) * double(n[big]) * double(n[big]) / all;
	const int    t     = int(std::ceil(2.0 * share * threads));
	return std::max(2, std::min(std::min(threads / 2, 8), t));
}

} // namespace

bool group_eigenvalues(size_t ng, const size_t* n, double* const* a, double* const* w,
                       std::vector<GroupReduction>& red, int threads)
{
	red.assign(ng, GroupReduction {});
	threads = std::max(1, threads);
	std::vector<size_t> order(ng); // largest first
	std::iota(order.begin(), order.end(), size_t(0));
	std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) { return n[x] > n[y]; });
	// the reduction of one matrix (symmetrised first), by a team of `team`
	// threads when team > 1; then its eigenvalues
	auto reduce = [&](size_t g, int team) {
		const int       n_g = int(n[g]);
		GroupReduction& R   = red[g];
		double*         m   = a[g];
		for (int j = 0; j < n_g; ++j) // symmetrise the round-off of the two triangles
			for (int i = 0; i < j; ++i) {
				const size_t ij = size_t(i) + size_t(j) * size_t(n_g), ji = size_t(j) + size_t(i) * size_t(n_g);
				m[ij] = m[ji] = 0.5 * (m[ij] + m[ji]);
			}
		// largest entry outside [2^-64, 2^64]: reduce 2^shift m instead
		// (exact; the reflectors do not change), so that the squares of the
		// eigenvalue iteration and the growth of inverse iteration (up to
		// 1e15 / |T|) stay far inside the exponent range
		const size_t        nn   = size_t(n_g) * size_t(n_g);
		double              amax = 0.0;
		std::vector<double> scaled;
		for (size_t q = 0; q < nn; ++q)
			amax = std::max(amax, std::fabs(m[q]));
		R.shift = 0;
		if (amax > 0.0 && std::isfinite(amax) && (amax < 0x1p-64 || amax > 0x1p64)) {
			int e = 0;
			std::frexp(amax, &e);
			R.shift = -e;
			scaled.resize(nn);
			for (size_t q = 0; q < nn; ++q)
				scaled[q] = std::ldexp(m[q], R.shift);
			m = scaled.data();
		}
		if (n_g == 1) {
			R.d.assign(1, m[0]);
			R.off.assign(1, 0.0);
		} else if (team > 1) {
			householder_tridiag_parallel(n_g, m, R.d, R.off, R.hv, R.beta, team);
		} else {
			householder_tridiag(n_g, m, R.d, R.off, R.hv, R.beta);
		}
	};
	auto values = [&](size_t g) {
		GroupReduction& R = red[g];
		std::copy(R.d.begin(), R.d.end(), w[g]);
		R.ok = tridiag_values(int(n[g]), w[g], R.off.data()); // ascending
		if (R.shift) {
			R.scaled_values.assign(w[g], w[g] + n[g]);
			for (size_t i = 0; i < n[g]; ++i)
				w[g][i] = std::ldexp(w[g][i], -R.shift);
		}
	};
	const int    team  = ng ? team_size(ng, n, order[0], threads) : 0;
	const size_t first = team ? 1 : 0;
	// the other matrices, largest first, to whichever thread is free
	std::atomic<size_t> next { first };
	auto                drain = [&] {
		for (size_t q; (q = next.fetch_add(1)) < ng;)
			if (n[order[q]] > 0) {
				reduce(order[q], 1);
				values(order[q]);
			}
	};
	std::vector<std::thread> pool;
	for (int t = 0; t < threads - std::max(team, 1); ++t)
		pool.emplace_back(drain);
	if (team) {
		reduce(order[0], team);
		for (int t = 1; t < team; ++t) // the team's other threads take matrices now
			pool.emplace_back(drain);
		values(order[0]);
	}
	drain();
	for (std::thread& th : pool)
		th.join();
	bool ok = true;
	for (const GroupReduction& R : red)
		ok = ok && R.ok;
	return ok;
}

// v (n x ncols, column-major) <- Q v
void apply_q(int n, const std::vector<double>& hv, const std::vector<double>& beta, double* v, int ncols)
{
	const size_t N = size_t(n);
	for (int k = n - 3; k >= 0; --k) {
		if (beta[size_t(k)] == 0.0)
			continue;
		const double* h   = hv.data() + size_t(k) * N;
		const int     len = n - k - 1;
		for (int c = 0; c < ncols; ++c) {
			double* x = v + size_t(c) * N + size_t(k) + 1;
			double  s = 0.0;
			for (int i = 0; i < len; ++i)
				s += h[i] * x[i];
			s *= beta[size_t(k)];
			for (int i = 0; i < len; ++i)
				x[i] -= s * h[i];
		}
	}
}

bool sym_lowest(int n, const double* a, double* w, double* v)
{
	if (n <= 0)
		return false;
	if (n == 1) {
		*w   = a[0];
		v[0] = 1.0;
		return true;
	}
	std::vector<double> d, off, hv, beta;
	householder_tridiag(n, a, d, off, hv, beta);
	// lowest eigenpair of T, then v = Q z
	*w = tridiag_kth_lowest(n, d.data(), off.data(), 1);
	tridiag_inverse_iteration(n, d.data(), off.data(), *w, v);
	apply_q(n, hv, beta, v, 1);
	return true;
}

bool sym_eigen_full(int n, const double* a, double* w, double* v)
{
	if (n <= 0)
		return true;
	if (n == 1) {
		w[0] = a[0];
		if (v)
			v[0] = 1.0;
		return true;
	}
	std::vector<double> d, off, hv, beta;
	householder_tridiag(n, a, d, off, hv, beta);
	if (!tridiag_eigen(n, d.data(), off.data(), v))
		return false;
	std::copy(d.begin(), d.end(), w);
	if (v)
		apply_q(n, hv, beta, v, n);
	return true;
}

} // namespace dmrgpp

namespace dmrgpp {

namespace {

// uniform in [-1, 1) from (seed, index): the splitmix64 finaliser (Steele,
// Lea and Flood, OOPSLA 2014) of their combination, top 53 bits
inline double start_value(uint64_t seed, uint64_t i)
{
	uint64_t x = seed + 0x9e3779b97f4a7c15ULL * (i + 1);
	x          = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
	x          = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
	x ^= x >> 31;
	return double(x >> 11) * 0x1.0p-52 - 1.0;
}

// |T|_inf of the tridiagonal (d, off)
double tridiag_norm(int n, const double* d, const double* off)
{
	double norm = 0.0;
	for (int i = 0; i < n; ++i)
		norm = std::max(norm, std::fabs(d[i]) + (i > 0 ? std::fabs(off[i - 1]) : 0.0)
		                         + (i + 1 < n ? std::fabs(off[i]) : 0.0));
	return norm;
}

typedef long long v4l __attribute__((vector_size(32), aligned(8), may_alias));

// One vector by inverse iteration (n >= 2): the LU of T - w_j I with row
// interchanges (as tridiag_inverse_iteration), then from the start vector
// seeded by j three solves, each followed by Gram-Schmidt against the
// cluster's earlier vectors ys[0..ny) and a normalisation; the largest
// component made positive.  The arithmetic is written so that
// eigenvectors_batch4 repeats it operation for operation.
void eigenvector_one(int n, const double* d, const double* off, double wj, int j, double tiny, const double* const* ys,
                     int ny, double* x, double* rp, double* u1, double* u2, double* m, char* sw)
{
	const size_t N = size_t(n);
	double       a = d[0] - wj, b = off[0];
	for (int i = 0; i + 1 < n; ++i) {
		const double l = off[i], dd = d[i + 1] - wj, uu = i + 2 < n ? off[i + 1] : 0.0;
		if (std::fabs(a) >= std::fabs(l)) {
			if (a == 0.0)
				a = tiny;
			const double r = 1.0 / a;
			rp[i]          = r;
			u1[i]          = b;
			u2[i]          = 0.0;
			m[i]           = l * r;
			sw[i]          = 0;
			a              = dd - m[i] * b;
			b              = uu;
		} else {
			const double r  = 1.0 / l;
			rp[i]           = r;
			u1[i]           = dd;
			u2[i]           = uu;
			m[i]            = a * r;
			sw[i]           = 1;
			const double na = b - m[i] * dd;
			b               = -(m[i] * uu);
			a               = na;
		}
	}
	rp[N - 1] = 1.0 / (a == 0.0 ? tiny : a);
	for (int i = 0; i < n; ++i)
		x[i] = start_value(uint64_t(j), uint64_t(i));
	for (int iter = 0; iter < 3; ++iter) {
		for (int i = 0; i + 1 < n; ++i) {
			const double xi = x[i], xi1 = x[i + 1];
			if (sw[i]) {
				x[i]     = xi1;
				x[i + 1] = xi - m[i] * xi1;
			} else {
				x[i + 1] = xi1 - m[i] * xi;
			}
		}
		for (int i = n - 1; i >= 0; --i) {
			double s = x[i];
			if (i + 1 < n)
				s -= u1[i] * x[i + 1];
			if (i + 2 < n)
				s -= u2[i] * x[i + 2];
			x[i] = s * rp[i];
		}
		// Gram-Schmidt against the cluster's earlier vectors; after the last
		// solve twice, since the solve leaves x almost entirely in their span
		// and one pass keeps rounding errors of that size ("twice is enough")
		for (int pass = 0; pass < (iter == 2 ? 2 : 1); ++pass)
			for (int q = 0; q < ny; ++q) {
				const double* y = ys[q];
				double        p = 0.0;
				for (int i = 0; i < n; ++i)
					p += y[i] * x[i];
				for (int i = 0; i < n; ++i)
					x[i] -= p * y[i];
			}
		double nrm = 0.0;
		for (int i = 0; i < n; ++i)
			nrm += x[i] * x[i];
		nrm = std::sqrt(nrm);
		if (!(nrm > 0.0) || !std::isfinite(nrm)) { // start again from a unit vector
			std::fill(x, x + N, 0.0);
			x[j % n] = 1.0;
			continue;
		}
		const double r = 1.0 / nrm;
		for (int i = 0; i < n; ++i)
			x[i] *= r;
	}
	double big = 0.0;
	int    arg = 0;
	for (int i = 0; i < n; ++i)
		if (std::fabs(x[i]) > big) {
			big = std::fabs(x[i]);
			arg = i;
		}
	if (x[arg] < 0.0)
		for (int i = 0; i < n; ++i)
			x[i] = -x[i];
}

// Four vectors that need no Gram-Schmidt (each starts its cluster) at once,
// one per lane: eigenvector_one's operations with the pivot choice and the
// row interchanges as lane masks, so each lane's result is bitwise the one
// eigenvector_one gives.  xs[l]: the output columns; scratch X, RP, U1, U2,
// M (n each) and SW.
inline __attribute__((always_inline)) void batch4_body(int n, const double* d, const double* off, const double* wj,
                                                       const int* jj, double tiny, double* const* xs, v4d* X, v4d* RP,
                                                       v4d* U1, v4d* U2, v4d* M, v4l* SW)
{
	const size_t N    = size_t(n);
	const v4d    zero = { 0.0, 0.0, 0.0, 0.0 };
	const v4d    w    = { wj[0], wj[1], wj[2], wj[3] };
	v4d          a = d[0] - w, b = zero + off[0];
	for (int i = 0; i + 1 < n; ++i) {
		const double l = off[i], uu = i + 2 < n ? off[i + 1] : 0.0;
		const v4d    dd = d[i + 1] - w;
		const v4d    al = a < 0.0 ? -a : a;
		const v4l    keep = al >= std::fabs(l); // no interchange
		a                 = (keep & (a == 0.0)) ? zero + tiny : a;
		const v4d piv     = keep ? a : zero + l;
		const v4d r       = 1.0 / piv;
		RP[i]             = r;
		U1[i]             = keep ? b : dd;
		U2[i]             = keep ? zero : zero + uu;
		const v4d mm      = (keep ? zero + l : a) * r;
		M[i]              = mm;
		SW[i]             = ~keep;
		const v4d na      = keep ? dd - mm * b : b - mm * dd;
		b                 = keep ? zero + uu : -(mm * uu);
		a                 = na;
	}
	RP[N - 1] = 1.0 / ((a == 0.0) ? zero + tiny : a);
	for (int i = 0; i < n; ++i)
		X[i] = v4d { start_value(uint64_t(jj[0]), uint64_t(i)), start_value(uint64_t(jj[1]), uint64_t(i)),
			     start_value(uint64_t(jj[2]), uint64_t(i)), start_value(uint64_t(jj[3]), uint64_t(i)) };
	for (int iter = 0; iter < 3; ++iter) {
		for (int i = 0; i + 1 < n; ++i) {
			const v4d xi = X[i], xi1 = X[i + 1];
			const v4l s  = SW[i];
			X[i]         = s ? xi1 : xi;
			X[i + 1]     = s ? xi - M[i] * xi1 : xi1 - M[i] * xi;
		}
		for (int i = n - 1; i >= 0; --i) {
			v4d s = X[i];
			if (i + 1 < n)
				s -= U1[i] * X[i + 1];
			if (i + 2 < n)
				s -= U2[i] * X[i + 2];
			X[i] = s * RP[i];
		}
		v4d nrm = zero;
		for (int i = 0; i < n; ++i)
			nrm += X[i] * X[i];
		v4d r = zero;
		for (int q = 0; q < 4; ++q) {
			const double t = std::sqrt(nrm[q]);
			if (!(t > 0.0) || !std::isfinite(t)) { // this lane starts again from a unit vector
				for (int i = 0; i < n; ++i)
					X[i][q] = i == jj[q] % n ? 1.0 : 0.0;
				r[q] = 1.0;
			} else {
				r[q] = 1.0 / t;
			}
		}
		for (int i = 0; i < n; ++i)
			X[i] *= r;
	}
	for (int q = 0; q < 4; ++q) {
		double big = 0.0;
		int    arg = 0;
		for (int i = 0; i < n; ++i)
			if (std::fabs(X[i][q]) > big) {
				big = std::fabs(X[i][q]);
				arg = i;
			}
		const double sgn = X[size_t(arg)][q] < 0.0 ? -1.0 : 1.0;
		double*      x   = xs[q];
		for (int i = 0; i < n; ++i)
			x[i] = sgn < 0.0 ? -X[i][q] : X[i][q];
	}
}

__attribute__((target("avx2"))) void batch4_avx2(int n, const double* d, const double* off, const double* wj,
                                                 const int* jj, double tiny, double* const* xs, v4d* X, v4d* RP,
                                                 v4d* U1, v4d* U2, v4d* M, v4l* SW)
{
	batch4_body(n, d, off, wj, jj, tiny, xs, X, RP, U1, U2, M, SW);
}

void batch4_base(int n, const double* d, const double* off, const double* wj, const int* jj, double tiny,
                 double* const* xs, v4d* X, v4d* RP, v4d* U1, v4d* U2, v4d* M, v4l* SW)
{
	batch4_body(n, d, off, wj, jj, tiny, xs, X, RP, U1, U2, M, SW);
}

// 0 turns the four-lane batches off (tests compare the two)
std::atomic<int> g_batch_vectors { 1 };

// Vectors j0 .. j1 - 1 of tridiag_eigenvectors (n >= 2, norm > 0); j0 starts
// a cluster, so the range needs no vector before it.  The vectors that start
// their cluster (no Gram-Schmidt) go four at a time, the others follow one
// by one in order, after the earlier vectors of their cluster.
void eigenvectors_range(int n, const double* d, const double* off, const double* w, int j0, int j1, double norm,
                        double* z)
{
	const size_t N     = size_t(n);
	const double ortol = 1e-3 * norm;
	const double tiny  = norm * 1e-15;
	auto         col   = [&](int j) { return z + size_t(j - j0) * N; };
	auto         starts = [&](int j) { return j == j0 || w[j] - w[j - 1] > ortol; };
	std::vector<int> lone, rest;
	for (int j = j0; j < j1; ++j)
		(starts(j) ? lone : rest).push_back(j);
	size_t done = 0;
	if (g_batch_vectors.load(std::memory_order_relaxed) && lone.size() >= 4) {
		std::vector<double>    buf(20 * N); // X, RP, U1, U2, M: four lanes per row
		std::vector<long long> swb(4 * N);
		v4d* const             X    = reinterpret_cast<v4d*>(buf.data());
		v4d* const             RP   = X + N;
		v4d* const             U1   = RP + N;
		v4d* const             U2   = U1 + N;
		v4d* const             M    = U2 + N;
		v4l* const             SW   = reinterpret_cast<v4l*>(swb.data());
		const bool             avx2 = g_pass_isa.load(std::memory_order_relaxed) && host_has_avx2();
		for (; done + 4 <= lone.size(); done += 4) {
			const int     jj[4] = { lone[done], lone[done + 1], lone[done + 2], lone[done + 3] };
			const double  wj[4] = { w[jj[0]], w[jj[1]], w[jj[2]], w[jj[3]] };
			double* const xs[4] = { col(jj[0]), col(jj[1]), col(jj[2]), col(jj[3]) };
			if (avx2)
				batch4_avx2(n, d, off, wj, jj, tiny, xs, X, RP, U1, U2, M, SW);
			else
				batch4_base(n, d, off, wj, jj, tiny, xs, X, RP, U1, U2, M, SW);
		}
	}
	std::vector<double>        rp(N), u1(N), u2(N), m(N);
	std::vector<char>          sw(N);
	std::vector<const double*> ys;
	auto one = [&](int j) {
		ys.clear();
		int c = j; // first vector of j's cluster
		while (!starts(c))
			--c;
		for (int q = c; q < j; ++q)
			ys.push_back(col(q));
		eigenvector_one(n, d, off, w[j], j, tiny, ys.data(), int(ys.size()), col(j), rp.data(), u1.data(),
		                u2.data(), m.data(), sw.data());
	};
	for (; done < lone.size(); ++done)
		one(lone[done]);
	for (int j : rest)
		one(j);
}

// the matrices where every vector is fixed without iterating: n = 1, and the
// zero matrix (any orthonormal set); true when z was filled here
bool trivial_eigenvectors(int n, int k, double norm, double* z)
{
	const size_t N = size_t(n);
	if (n == 1) {
		for (int j = 0; j < k; ++j)
			z[j] = 1.0;
		return true;
	}
	if (!(norm > 0.0)) {
		std::fill(z, z + N * size_t(k), 0.0);
		for (int j = 0; j < k; ++j)
			z[size_t(j) * N + size_t(j % n)] = 1.0;
		return true;
	}
	return false;
}

// The kept vectors whose eigenvalues are rounding noise (at most n eps |T|
// in magnitude: a density matrix of lower rank than its group) span a part
// of the numerical null space that inverse iteration cannot resolve; each
// Gram-Schmidt pass inside that cluster carries over the errors of the
// earlier vectors, which renormalisation amplifies.  Since a group's kept
// vectors are its largest, every eigenvector above such a vector is kept
// too: they are projected out of the null vectors (twice), and the null
// vectors are orthonormalised again among themselves (twice).  z: n x k for
// the ascending eigenvalues w[0..k).
void clean_null_vectors(int n, int k, const double* w, double norm, double* z)
{
	const size_t N    = size_t(n);
	const double null = double(n) * DBL_EPSILON * norm;
	int          jn   = 0; // vectors [0, jn) are null
	while (jn < k && std::fabs(w[jn]) <= null)
		++jn;
	if (jn == 0 || (jn == 1 && jn == k))
		return;
	auto project = [&](double* x, const double* y) {
		double p = 0.0;
		for (size_t i = 0; i < N; ++i)
			p += y[i] * x[i];
		for (size_t i = 0; i < N; ++i)
			x[i] -= p * y[i];
	};
	for (int j = 0; j < jn; ++j) {
		double* x = z + size_t(j) * N;
		for (int pass = 0; pass < 2; ++pass) {
			for (int q = jn; q < k; ++q)
				project(x, z + size_t(q) * N);
			for (int q = 0; q < j; ++q)
				project(x, z + size_t(q) * N);
		}
		double nrm = 0.0;
		for (size_t i = 0; i < N; ++i)
			nrm += x[i] * x[i];
		nrm = std::sqrt(nrm);
		if (nrm > 0.0 && std::isfinite(nrm)) {
			const double r = 1.0 / nrm;
			for (size_t i = 0; i < N; ++i)
				x[i] *= r;
		}
	}
}

} // namespace

void eigenvectors_set_batch(int on) { g_batch_vectors.store(on ? 1 : 0); }

void tridiag_eigenvectors(int n, const double* d, const double* off, const double* w, int k, double* z)
{
	if (n <= 0 || k <= 0)
		return;
	const double norm = n > 1 ? tridiag_norm(n, d, off) : 0.0;
	if (trivial_eigenvectors(n, k, norm, z))
		return;
	eigenvectors_range(n, d, off, w, 0, k, norm, z);
	clean_null_vectors(n, k, w, norm, z);
}

void group_eigenvectors(size_t ng, const size_t* n, const size_t* k, const GroupReduction* red,
                        const double* const* w, double* const* z, int threads)
{
	// work items: runs of at least 16 vectors of one group, cut only where a
	// cluster ends, so each item computes what the serial call would
	struct Item {
		size_t g;
		int    j0, j1;
		double cost;
	};
	std::vector<Item>   items;
	std::vector<double> norm(ng, 0.0);
	// a group reduced as 2^shift A: its own eigenvalues of that matrix (the
	// unscaled ones may have lost bits below the normal range)
	std::vector<const double*> ws(w, w + ng);
	for (size_t g = 0; g < ng; ++g)
		if (red[g].shift && k[g] > 0 && red[g].scaled_values.size() == n[g])
			ws[g] = red[g].scaled_values.data() + (n[g] - k[g]);
	w = ws.data();
	for (size_t g = 0; g < ng; ++g) {
		const int n_g = int(n[g]), k_g = int(k[g]);
		if (n_g <= 0 || k_g <= 0)
			continue;
		norm[g] = n_g > 1 ? tridiag_norm(n_g, red[g].d.data(), red[g].off.data()) : 0.0;
		if (trivial_eigenvectors(n_g, k_g, norm[g], z[g]))
			continue;
		const double ortol = 1e-3 * norm[g];
		int          j0    = 0;
		for (int j = 1; j <= k_g; ++j)
			if (j == k_g || (j - j0 >= 16 && w[g][j] - w[g][j - 1] > ortol)) {
				items.push_back({ g, j0, j, double(j - j0) * double(n_g) });
				j0 = j;
			}
	}
	std::stable_sort(items.begin(), items.end(), [](const Item& a, const Item& b) { return a.cost > b.cost; });
	std::atomic<size_t> next { 0 };
	auto                drain = [&] {
		for (size_t q; (q = next.fetch_add(1)) < items.size();) {
			const Item& it = items[q];
			const int   n_g = int(n[it.g]);
			eigenvectors_range(n_g, red[it.g].d.data(), red[it.g].off.data(), w[it.g], it.j0, it.j1, norm[it.g],
			                   z[it.g] + size_t(it.j0) * size_t(n_g));
		}
	};
	std::vector<std::thread> pool;
	const int                nt = int(std::min<size_t>(size_t(std::max(1, threads)), std::max<size_t>(items.size(), 1)));
	for (int t = 1; t < nt; ++t)
		pool.emplace_back(drain);
	drain();
	for (std::thread& th : pool)
		th.join();
	// the groups' null vectors, once all their vectors are there
	std::atomic<size_t> ng_next { 0 };
	auto                clean = [&] {
		for (size_t g; (g = ng_next.fetch_add(1)) < ng;)
			if (n[g] >= 2 && k[g] > 0 && norm[g] > 0.0)
				clean_null_vectors(int(n[g]), int(k[g]), w[g], norm[g], z[g]);
	};
	pool.clear();
	for (int t = 1; t < nt; ++t)
		pool.emplace_back(clean);
	clean();
	for (std::thread& th : pool)
		th.join();
}

} // namespace dmrgpp
