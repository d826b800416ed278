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
