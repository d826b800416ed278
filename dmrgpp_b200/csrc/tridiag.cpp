// Symmetric tridiagonal eigensolver for the Lanczos and Davidson drivers.
//
// The reference obtains the Ritz values of its Lanczos tridiagonal with
// LAPACK dstedc (PsimagLite/src/PsimagLite/TridiagonalMatrix.cpp:21) and the
// Ritz vectors from a dense symmetric eigensolve of the same matrix
// (LanczosSolver.h:76-84).  Here both come from one implementation of the
// implicit QL algorithm with shifts taken from the leading 2x2 block
// (Bowdler, Martin, Reinsch and Wilkinson, Numer. Math. 11 (1968) 293-306;
// Golub and Van Loan, Matrix Computations, section 8.3), in FP64.
#include "tridiag.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <numeric>
#include <vector>

namespace dmrgpp {

bool tridiag_eigen(int n, double* d, const double* off, double* z)
{
	if (n <= 0)
		return true;
	std::vector<double> e(size_t(n), 0.0);
	for (int i = 0; i + 1 < n; ++i)
		e[size_t(i)] = off[i];
	if (z) {
		std::fill(z, z + size_t(n) * size_t(n), 0.0);
		for (int i = 0; i < n; ++i)
			z[size_t(i) + size_t(i) * size_t(n)] = 1.0;
	}
	for (int l = 0; l < n; ++l) {
		int iter = 0;
		for (;;) {
			// smallest m >= l whose off-diagonal element is negligible
			int m = l;
			for (; m + 1 < n; ++m) {
				const double dd = std::fabs(d[m]) + std::fabs(d[m + 1]);
				if (std::fabs(e[size_t(m)]) <= DBL_EPSILON * dd)
					break;
			}
			if (m == l)
				break;
			if (++iter > 60)
				return false;
			// shift: eigenvalue of the leading 2x2 block closer to d[l]
			double g = (d[l + 1] - d[l]) / (2.0 * e[size_t(l)]);
			double r = std::hypot(g, 1.0);
			g        = d[m] - d[l] + e[size_t(l)] / (g + std::copysign(r, g));
			double s = 1.0, c = 1.0, p = 0.0;
			bool   split = false;
			for (int i = m - 1; i >= l; --i) {
				const double f = s * e[size_t(i)];
				const double b = c * e[size_t(i)];
				r              = std::hypot(f, g);
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
				if (z) {
					double* zi  = z + size_t(i) * size_t(n);
					double* zi1 = zi + size_t(n);
					for (int k = 0; k < n; ++k) {
						const double t = zi1[k];
						zi1[k]         = s * zi[k] + c * t;
						zi[k]          = c * zi[k] - s * t;
					}
				}
			}
			if (split)
				continue;
			d[l] -= p;
			e[size_t(l)] = g;
			e[size_t(m)] = 0.0;
		}
	}
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

} // namespace dmrgpp

namespace dmrgpp {

bool sym_lowest(int n, const double* a, double* w, double* v)
{
	if (n <= 0)
		return false;
	if (n == 1) {
		*w   = a[0];
		v[0] = 1.0;
		return true;
	}
	// Householder reduction T = Q^T A Q, Q = P_0 P_1 ... P_{n-3}; P_k acts on
	// rows / columns k+1..n-1 with P_k = I - beta_k h_k h_k^T, h_k(0) = 1
	// (Golub and Van Loan, algorithms 5.1.1 and 8.3.1)
	const size_t        N = size_t(n);
	std::vector<double> m(a, a + N * N), d(N), off(N - 1), hv(N * N, 0.0), beta(N, 0.0), p(N), q(N);
	auto                M = [&](int i, int j) -> double& { return m[size_t(i) + size_t(j) * N]; };
	for (int k = 0; k + 2 < n; ++k) {
		const int len   = n - k - 1;
		double*   h     = hv.data() + size_t(k) * N; // h[0..len)
		double    sigma = 0.0;
		for (int i = 1; i < len; ++i)
			sigma += M(k + 1 + i, k) * M(k + 1 + i, k);
		const double x0 = M(k + 1, k);
		d[size_t(k)]    = M(k, k);
		if (sigma == 0.0) { // already tridiagonal in this column
			off[size_t(k)] = x0;
			continue;
		}
		const double mu = std::sqrt(x0 * x0 + sigma);
		const double h0 = x0 <= 0.0 ? x0 - mu : -sigma / (x0 + mu);
		beta[size_t(k)] = 2.0 * h0 * h0 / (sigma + h0 * h0);
		h[0]            = 1.0;
		for (int i = 1; i < len; ++i)
			h[i] = M(k + 1 + i, k) / h0;
		off[size_t(k)] = mu;
		// trailing block A22 <- P A22 P = A22 - h w^T - w h^T with
		// p = beta A22 h, w = p - (beta / 2)(p^T h) h
		const double b = beta[size_t(k)];
		for (int i = 0; i < len; ++i) {
			double s = 0.0;
			for (int j = 0; j < len; ++j)
				s += M(k + 1 + i, k + 1 + j) * h[j];
			p[size_t(i)] = b * s;
		}
		double ph = 0.0;
		for (int i = 0; i < len; ++i)
			ph += p[size_t(i)] * h[i];
		for (int i = 0; i < len; ++i)
			q[size_t(i)] = p[size_t(i)] - 0.5 * b * ph * h[i];
		for (int j = 0; j < len; ++j)
			for (int i = 0; i < len; ++i)
				M(k + 1 + i, k + 1 + j) -= h[i] * q[size_t(j)] + q[size_t(i)] * h[j];
	}
	d[N - 2]   = M(n - 2, n - 2);
	d[N - 1]   = M(n - 1, n - 1);
	off[N - 2] = M(n - 1, n - 2);
	// lowest eigenpair of T, then v = Q z
	*w = tridiag_kth_lowest(n, d.data(), off.data(), 1);
	tridiag_inverse_iteration(n, d.data(), off.data(), *w, v);
	for (int k = n - 3; k >= 0; --k) {
		if (beta[size_t(k)] == 0.0)
			continue;
		const double* h   = hv.data() + size_t(k) * N;
		const int     len = n - k - 1;
		double        s   = 0.0;
		for (int i = 0; i < len; ++i)
			s += h[i] * v[k + 1 + i];
		s *= beta[size_t(k)];
		for (int i = 0; i < len; ++i)
			v[k + 1 + i] -= s * h[i];
	}
	return true;
}

} // namespace dmrgpp
