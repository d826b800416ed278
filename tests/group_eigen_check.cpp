// Host check of the eigenvalue phase of the density-matrix truncation
// (tridiag.cpp): the reduction's AVX2 and baseline passes give bitwise the
// same reflectors, serial and by thread teams; tridiag_values (square-root-
// free QL) agrees with tridiag_eigen (QL with rotations) on random, graded,
// low-rank and clustered matrices and falls back to it outside the range of
// the squares; group_eigenvalues on a mix of group sizes (0, 1, 2, odd, one
// large enough for a thread team) and thread counts gives each group the
// eigenvalues of its own serial reduction, symmetrising the input in place;
// the kept eigenvectors by inverse iteration four lanes at a time bitwise
// equal to one at a time, group_eigenvectors bitwise equal to the serial
// tridiag_eigenvectors of each group, with small residuals and orthonormal
// columns, on matrices with clusters and exactly repeated eigenvalues; and
// groups of subnormal or huge entries reduced scaled by a power of two.
// Prints "ok <worst eigenvalue difference / norm>" or "FAIL ...".
#include "tridiag.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <random>
#include <vector>

namespace {

std::mt19937_64                        rng(2027);
std::uniform_real_distribution<double> u(-1.0, 1.0);

// symmetric n x n (column-major): 0 random, 1 graded diagonal, 2 Gram matrix
// X^T X of a rank-n/3 X with decaying rows (a density matrix), 3 Gram
// matrix of a square X (full rank, eigenvalues down to ~1/n^2 of the norm)
std::vector<double> matrix(int n, int kind)
{
	const size_t        N = size_t(n);
	std::vector<double> a(N * N, 0.0);
	if (kind >= 2) {
		const int           r = kind == 2 ? std::max(1, n / 3) : n;
		std::vector<double> x(size_t(r) * N);
		for (size_t q = 0; q < x.size(); ++q)
			x[q] = u(rng) * (kind == 2 ? std::exp(-0.5 * double(q % size_t(r))) : 1.0);
		for (int j = 0; j < n; ++j)
			for (int i = 0; i <= j; ++i) {
				double s = 0.0;
				for (int k = 0; k < r; ++k)
					s += x[size_t(k) + size_t(i) * size_t(r)] * x[size_t(k) + size_t(j) * size_t(r)];
				a[size_t(i) + size_t(j) * N] = a[size_t(j) + size_t(i) * N] = s;
			}
		return a;
	}
	for (int j = 0; j < n; ++j)
		for (int i = 0; i <= j; ++i) {
			double x = u(rng);
			if (kind == 1)
				x = i == j ? std::pow(10.0, -0.1 * i) * x : 1e-3 * std::pow(10.0, -0.05 * (i + j)) * x;
			a[size_t(i) + size_t(j) * N] = a[size_t(j) + size_t(i) * N] = x;
		}
	return a;
}

double norm_of(const std::vector<double>& w)
{
	double s = 1e-300;
	for (double x : w)
		s = std::max(s, std::fabs(x));
	return s;
}

} // namespace

int main()
{
	double worst = 0.0;
	// 1. the two instruction-set builds of the reduction's passes
	for (int n : { 2, 3, 4, 5, 6, 7, 8, 9, 31, 64, 65, 130, 211 }) {
		const auto          a = matrix(n, n % 4);
		std::vector<double> d[2], e[2], h[2], b[2];
		for (int isa = 0; isa < 2; ++isa) {
			dmrgpp::householder_set_isa(isa);
			dmrgpp::householder_tridiag(n, a.data(), d[isa], e[isa], h[isa], b[isa]);
		}
		if (d[0] != d[1] || e[0] != e[1] || h[0] != h[1] || b[0] != b[1]) {
			std::printf("FAIL isa serial %d\n", n);
			return 1;
		}
		for (int t : { 2, 3, 5 }) {
			std::vector<double> dp[2], ep[2], hp[2], bp[2];
			for (int isa = 0; isa < 2; ++isa) {
				dmrgpp::householder_set_isa(isa);
				dmrgpp::householder_tridiag_parallel(n, a.data(), dp[isa], ep[isa], hp[isa], bp[isa], t);
			}
			if (dp[0] != dp[1] || ep[0] != ep[1] || hp[0] != hp[1] || bp[0] != bp[1]) {
				std::printf("FAIL isa team %d %d\n", n, t);
				return 1;
			}
		}
	}
	dmrgpp::householder_set_isa(1);
	// 2. tridiag_values against tridiag_eigen, on reductions of dense
	// matrices and on tridiagonals with zeros and exactly repeated blocks
	for (int trial = 0; trial < 200; ++trial) {
		const int           n = 1 + (trial * 13) % 160;
		std::vector<double> d, e, h, b;
		if (trial % 5 == 4) {
			d.resize(size_t(n));
			e.assign(size_t(n), 0.0);
			for (int i = 0; i < n; ++i) {
				d[size_t(i)] = i < n / 2 ? u(rng) : d[size_t(i - n / 2)];
				e[size_t(i)] = (i + 1 == n / 2 || i % 7 == 6) ? 0.0 : u(rng);
			}
			if (trial % 10 == 9)
				std::fill(d.begin(), d.end(), 0.0), std::fill(e.begin(), e.end(), 0.0);
		} else if (n == 1) {
			d.assign(1, u(rng));
			e.assign(1, 0.0);
		} else {
			const auto a = matrix(n, trial % 4);
			dmrgpp::householder_tridiag(n, a.data(), d, e, h, b);
		}
		std::vector<double> w1(d), w2(d);
		if (!dmrgpp::tridiag_eigen(n, w1.data(), e.data(), nullptr) || !dmrgpp::tridiag_values(n, w2.data(), e.data())) {
			std::printf("FAIL values converge %d\n", trial);
			return 1;
		}
		const double scale = norm_of(w1);
		for (int i = 0; i < n; ++i) {
			const double x = std::fabs(w1[size_t(i)] - w2[size_t(i)]) / scale;
			if (!(x <= 1e-13) || (i && w2[size_t(i)] < w2[size_t(i) - 1])) {
				std::printf("FAIL values %d n %d %g\n", trial, n, x);
				return 1;
			}
			worst = std::max(worst, x);
		}
	}
	// outside the squares' exponent range: the rotations' result exactly
	for (double scale : { 1e120, 1e-120 }) {
		const int           n = 40;
		std::vector<double> d(static_cast<size_t>(n)), e(static_cast<size_t>(n), 0.0);
		for (int i = 0; i < n; ++i)
			d[size_t(i)] = scale * u(rng), e[size_t(i)] = i + 1 < n ? scale * u(rng) : 0.0;
		std::vector<double> w1(d), w2(d);
		dmrgpp::tridiag_eigen(n, w1.data(), e.data(), nullptr);
		dmrgpp::tridiag_values(n, w2.data(), e.data());
		if (w1 != w2) {
			std::printf("FAIL range fallback %g\n", scale);
			return 1;
		}
	}
	// 3. group_eigenvalues: every group's eigenvalues those of its own
	// serial reduction (team groups to rounding), inputs symmetrised in place
	const std::vector<size_t> sizes = { 0, 1, 2, 3, 5, 300, 17, 64, 2, 1, 131, 0, 40, 7 };
	for (int threads : { 1, 2, 4, 7, 16 }) {
		const size_t                     ng = sizes.size();
		std::vector<std::vector<double>> a(ng), w(ng);
		std::vector<double*>             ap(ng), wp(ng);
		for (size_t g = 0; g < ng; ++g) {
			const int n = int(sizes[g]);
			a[g]        = matrix(std::max(n, 1), int(g % 4));
			a[g].resize(size_t(n) * size_t(n));
			for (size_t q = 0; q < a[g].size(); ++q) // unequal triangles: round-off of a Gram product
				a[g][q] *= 1.0 + 1e-15 * double(q % 3);
			w[g].assign(size_t(n), 0.0);
			ap[g] = a[g].data();
			wp[g] = w[g].data();
		}
		const auto                              orig = a;
		std::vector<dmrgpp::GroupReduction> red;
		if (!dmrgpp::group_eigenvalues(ng, sizes.data(), ap.data(), wp.data(), red, threads) || red.size() != ng) {
			std::printf("FAIL group_eigenvalues %d\n", threads);
			return 1;
		}
		for (size_t g = 0; g < ng; ++g) {
			const int n = int(sizes[g]);
			for (int j = 0; j < n; ++j)
				for (int i = 0; i < n; ++i) {
					const double x = a[g][size_t(i) + size_t(j) * size_t(n)], y = a[g][size_t(j) + size_t(i) * size_t(n)];
					const double z = 0.5 * (orig[g][size_t(i) + size_t(j) * size_t(n)] + orig[g][size_t(j) + size_t(i) * size_t(n)]);
					if (x != y || std::fabs(x - z) > 1e-15 * std::fabs(z)) {
						std::printf("FAIL symmetrised %zu\n", g);
						return 1;
					}
				}
			if (n == 0)
				continue;
			std::vector<double> d, e, h, b, ref;
			if (n == 1) {
				ref.assign(1, a[g][0]);
			} else {
				dmrgpp::householder_tridiag(n, a[g].data(), d, e, h, b);
				ref = d;
				dmrgpp::tridiag_values(n, ref.data(), e.data());
			}
			const bool   team  = threads >= 4 && n == 300;
			const double scale = norm_of(ref);
			for (int i = 0; i < n; ++i) {
				const double x = std::fabs(ref[size_t(i)] - w[g][size_t(i)]);
				if (team ? x > 1e-13 * scale : x != 0.0) {
					std::printf("FAIL group %zu n %d threads %d %g\n", g, n, threads, x / scale);
					return 1;
				}
			}
			if (!team && n > 1 && (red[g].d != d || red[g].off != e || red[g].hv != h || red[g].beta != b)) {
				std::printf("FAIL group reduction %zu threads %d\n", g, threads);
				return 1;
			}
		}
	}
	// 4. the kept eigenvectors
	{
		const std::vector<size_t> vs = { 1, 2, 3, 9, 40, 0, 120, 64, 33, 5, 200, 16 };
		const size_t              ng = vs.size();
		std::vector<dmrgpp::GroupReduction> red(ng);
		std::vector<std::vector<double>>    w(ng);
		std::vector<size_t>                 k(ng);
		for (size_t g = 0; g < ng; ++g) {
			const int n = int(vs[g]);
			if (n == 0)
				continue;
			auto& R = red[g];
			if (n == 1) {
				R.d.assign(1, 0.5);
				R.off.assign(1, 0.0);
			} else if (g % 4 == 3) { // two decoupled copies of one block: repeated eigenvalues
				R.d.resize(size_t(n));
				R.off.assign(size_t(n) - 1, 0.0);
				for (int i = 0; i < n; ++i)
					R.d[size_t(i)] = i < n / 2 ? u(rng) : R.d[size_t(i - n / 2)];
				for (int i = 0; i + 1 < n; ++i)
					R.off[size_t(i)] = i + 1 == n / 2 ? 0.0 : (i < n / 2 ? u(rng) : R.off[size_t(i - n / 2)]);
			} else if (g == 9) { // the zero matrix
				R.d.assign(size_t(n), 0.0);
				R.off.assign(size_t(n) - 1, 0.0);
			} else {
				const auto a = matrix(n, int(g % 4));
				dmrgpp::householder_tridiag(n, a.data(), R.d, R.off, R.hv, R.beta);
			}
			w[g] = R.d;
			dmrgpp::tridiag_values(n, w[g].data(), R.off.data());
			k[g] = size_t(std::max(1, (2 * n) / 3));
		}
		std::vector<std::vector<double>> z1(ng), z2(ng), z3(ng);
		std::vector<const double*>       wk(ng);
		std::vector<double*>             zp(ng);
		for (size_t g = 0; g < ng; ++g) {
			const int n = int(vs[g]), kg = int(k[g]);
			if (n == 0)
				continue;
			wk[g] = w[g].data() + (n - kg);
			z1[g].assign(size_t(n) * size_t(kg), 0.0);
			z2[g] = z1[g];
			dmrgpp::eigenvectors_set_batch(1);
			dmrgpp::tridiag_eigenvectors(n, red[g].d.data(), red[g].off.data(), wk[g], kg, z1[g].data());
			dmrgpp::eigenvectors_set_batch(0);
			dmrgpp::tridiag_eigenvectors(n, red[g].d.data(), red[g].off.data(), wk[g], kg, z2[g].data());
			dmrgpp::eigenvectors_set_batch(1);
			if (z1[g] != z2[g]) {
				std::printf("FAIL batched vectors %zu\n", g);
				return 1;
			}
			// residuals and orthonormality
			const double* d = red[g].d.data();
			const double* e = red[g].off.data();
			const double  scale = std::max(1.0, norm_of(w[g]));
			for (int c = 0; c < kg; ++c) {
				const double* x  = z1[g].data() + size_t(c) * size_t(n);
				const double  th = wk[g][c];
				for (int i = 0; i < n; ++i) {
					double t = (d[i] - th) * x[i];
					if (i > 0)
						t += e[i - 1] * x[i - 1];
					if (i + 1 < n)
						t += e[i] * x[i + 1];
					if (std::fabs(t) > 1e-12 * scale) {
						std::printf("FAIL vector residual %zu %d %g\n", g, c, t);
						return 1;
					}
				}
				for (int c2 = 0; c2 <= c; ++c2) {
					const double* y = z1[g].data() + size_t(c2) * size_t(n);
					double        s = 0.0;
					for (int i = 0; i < n; ++i)
						s += x[i] * y[i];
					if (std::fabs(s - (c == c2 ? 1.0 : 0.0)) > 1e-12) {
						std::printf("FAIL vector orthonormality %zu %d %d %g\n", g, c, c2, s);
						return 1;
					}
				}
			}
		}
		for (int threads : { 1, 3, 8 }) {
			for (size_t g = 0; g < ng; ++g) {
				z3[g].assign(z1[g].size(), -7.0);
				zp[g] = z3[g].data();
			}
			dmrgpp::group_eigenvectors(ng, vs.data(), k.data(), red.data(), wk.data(), zp.data(), threads);
			for (size_t g = 0; g < ng; ++g)
				if (z3[g] != z1[g]) {
					std::printf("FAIL group_eigenvectors %zu threads %d\n", g, threads);
					return 1;
				}
		}
	}
	// 5. groups near the underflow threshold and far above 1: reduced scaled
	// by a power of two; eigenvalues and kept vectors those of the exactly
	// rescaled matrix
	for (int e2 : { -1060, -1030, -150, 620 }) {
		const int           n = 70;
		std::vector<double> b = matrix(n, 2); // normal range: the reference
		std::vector<double> a(b.size());
		for (size_t q = 0; q < b.size(); ++q) {
			a[q] = std::ldexp(b[q], e2);        // the group as given (possibly subnormal)
			b[q] = std::ldexp(a[q], -e2);       // exactly what the scaled reduction sees
		}
		std::vector<double> wa(static_cast<size_t>(n)), wb(static_cast<size_t>(n));
		double*             ap[1] = { a.data() };
		double*             wp[1] = { wa.data() };
		const size_t        nn[1] = { size_t(n) };
		std::vector<dmrgpp::GroupReduction> red;
		if (!dmrgpp::group_eigenvalues(1, nn, ap, wp, red, 1)) {
			std::printf("FAIL scaled group %d converge\n", e2);
			return 1;
		}
		std::vector<double> d, e, h, b2;
		dmrgpp::householder_tridiag(n, b.data(), d, e, h, b2);
		wb = d;
		dmrgpp::tridiag_values(n, wb.data(), e.data());
		for (int i = 0; i < n; ++i)
			if (wa[size_t(i)] != std::ldexp(wb[size_t(i)], e2)) {
				std::printf("FAIL scaled group %d eigenvalue %d\n", e2, i);
				return 1;
			}
		const int           kk = n / 2;
		std::vector<double> z1(size_t(n) * size_t(kk)), z2(z1.size());
		const double*       wk[1] = { wa.data() + (n - kk) };
		double*             zp[1] = { z1.data() };
		const size_t        kv[1] = { size_t(kk) };
		dmrgpp::group_eigenvectors(1, nn, kv, red.data(), wk, zp, 2);
		dmrgpp::tridiag_eigenvectors(n, d.data(), e.data(), wb.data() + (n - kk), kk, z2.data());
		if (z1 != z2) {
			std::printf("FAIL scaled group %d vectors\n", e2);
			return 1;
		}
	}
	std::printf("ok %.3e\n", worst);
	return 0;
}
