// Host check of the tridiagonal helpers of the group Lanczos (tridiag.cpp):
// the k-th lowest eigenvalue by Sturm bisection against the QL solver, and
// the inverse-iteration eigenvector's residual, on seeded random and
// Lanczos-like (graded, nearly degenerate) tridiagonals; and the lowest pair
// of dense symmetric matrices by sym_lowest, and all pairs by sym_eigen_full,
// against the Jacobi solver.
// Prints "ok <worst eigenvalue error> <worst residual>" or "FAIL ...".
#include "tridiag.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <random>
#include <vector>

int main()
{
	std::mt19937_64                        rng(99);
	std::uniform_real_distribution<double> u(-1.0, 1.0);
	double                                 worst_e = 0.0, worst_r = 0.0;
	for (int trial = 0; trial < 400; ++trial) {
		const int           n = 1 + trial % 120;
		std::vector<double> d(static_cast<size_t>(n)), e(static_cast<size_t>(n), 0.0);
		const int           kind = trial % 3;
		for (int i = 0; i < n; ++i) {
			d[size_t(i)] = kind == 0 ? u(rng) * 10.0 : -50.0 + 0.01 * u(rng);
			e[size_t(i)] = kind == 2 ? 1e-9 * u(rng) : u(rng);
		}
		std::vector<double> w(d);
		if (!dmrgpp::tridiag_eigen(n, w.data(), e.data(), nullptr)) {
			std::printf("FAIL ql %d\n", trial);
			return 1;
		}
		double scale = 1.0;
		for (double x : w)
			scale = std::max(scale, std::fabs(x));
		for (int k = 1; k <= std::min(n, 3); ++k) {
			const double th = dmrgpp::tridiag_kth_lowest(n, d.data(), e.data(), k);
			worst_e         = std::max(worst_e, std::fabs(th - w[size_t(k - 1)]) / scale);
		}
		const double        th = dmrgpp::tridiag_kth_lowest(n, d.data(), e.data(), 1);
		std::vector<double> z(static_cast<size_t>(n));
		dmrgpp::tridiag_inverse_iteration(n, d.data(), e.data(), th, z.data());
		double res = 0.0, nz = 0.0;
		for (int i = 0; i < n; ++i) {
			double t = d[size_t(i)] * z[size_t(i)] - th * z[size_t(i)];
			if (i > 0)
				t += e[size_t(i - 1)] * z[size_t(i - 1)];
			if (i + 1 < n)
				t += e[size_t(i)] * z[size_t(i + 1)];
			res = std::max(res, std::fabs(t));
			nz += z[size_t(i)] * z[size_t(i)];
		}
		if (std::fabs(nz - 1.0) > 1e-12) {
			std::printf("FAIL norm %d %g\n", trial, nz);
			return 1;
		}
		worst_r = std::max(worst_r, res / scale);
	}
	// lowest pair of dense symmetric matrices (sym_lowest) against the Jacobi
	// solver (sym_eigen): eigenvalue and residual of the eigenvector; random
	// matrices and Davidson-like ones (graded diagonal, small couplings)
	for (int trial = 0; trial < 300; ++trial) {
		const int           n = 1 + trial % 48;
		const size_t        N = size_t(n);
		std::vector<double> A(N * N), ev(N), V(N * N), z(N);
		for (int j = 0; j < n; ++j)
			for (int i = 0; i <= j; ++i) {
				double x = u(rng);
				if (trial % 2)
					x = i == j ? -10.0 + 0.5 * i + 1e-3 * x : 1e-2 * x;
				A[size_t(i) + size_t(j) * N] = A[size_t(j) + size_t(i) * N] = x;
			}
		dmrgpp::sym_eigen(n, A.data(), ev.data(), V.data());
		double th = 0.0;
		dmrgpp::sym_lowest(n, A.data(), &th, z.data());
		double scale = 1.0, res = 0.0, nz = 0.0;
		for (double x : ev)
			scale = std::max(scale, std::fabs(x));
		for (int i = 0; i < n; ++i) {
			double t = -th * z[size_t(i)];
			for (int j = 0; j < n; ++j)
				t += A[size_t(i) + size_t(j) * N] * z[size_t(j)];
			res = std::max(res, std::fabs(t));
			nz += z[size_t(i)] * z[size_t(i)];
		}
		if (std::fabs(th - ev[0]) > 1e-13 * scale || res > 1e-12 * scale || std::fabs(nz - 1.0) > 1e-12) {
			std::printf("FAIL dense %d %g %g %g\n", trial, th - ev[0], res, nz);
			return 1;
		}
		worst_e = std::max(worst_e, std::fabs(th - ev[0]) / scale);
		worst_r = std::max(worst_r, res / scale);
	}
	// all pairs of dense symmetric matrices (sym_eigen_full): eigenvalues
	// against the Jacobi solver, residuals and orthonormality of the vectors;
	// random, graded, and density-matrix-like (Gram matrices, eigenvalues down
	// to round-off) cases
	for (int trial = 0; trial < 240; ++trial) {
		const int           n = 1 + (trial * 7) % 90;
		const size_t        N = size_t(n);
		std::vector<double> A(N * N, 0.0), ev(N), V(N * N), w(N), Z(N * N);
		if (trial % 3 == 2) { // X^T X with X n/2 x n: rank deficient
			const int           r = std::max(1, n / 2);
			std::vector<double> X(size_t(r) * N);
			for (size_t q = 0; q < X.size(); ++q) // rows of X decay like a DMRG spectrum in half the cases
				X[q] = trial % 2 ? u(rng) * std::exp(-0.7 * double(q % size_t(r)))
				                 : u(rng) * std::exp(-4.0 * std::fabs(u(rng)));
			for (int j = 0; j < n; ++j)
				for (int i = 0; i < n; ++i) {
					double s = 0.0;
					for (int k = 0; k < r; ++k)
						s += X[size_t(k) + size_t(i) * size_t(r)] * X[size_t(k) + size_t(j) * size_t(r)];
					A[size_t(i) + size_t(j) * N] = s;
				}
		} else {
			for (int j = 0; j < n; ++j)
				for (int i = 0; i <= j; ++i) {
					double x = u(rng);
					if (trial % 3 == 1)
						x = i == j ? -10.0 + 0.5 * i + 1e-3 * x : 1e-2 * x;
					A[size_t(i) + size_t(j) * N] = A[size_t(j) + size_t(i) * N] = x;
				}
		}
		dmrgpp::sym_eigen(n, A.data(), ev.data(), V.data());
		if (!dmrgpp::sym_eigen_full(n, A.data(), w.data(), Z.data())) {
			std::printf("FAIL full %d\n", trial);
			return 1;
		}
		double scale = 1.0, de = 0.0, res = 0.0, orth = 0.0;
		for (double x : ev)
			scale = std::max(scale, std::fabs(x));
		for (int c = 0; c < n; ++c) {
			de = std::max(de, std::fabs(w[size_t(c)] - ev[size_t(c)]));
			for (int i = 0; i < n; ++i) {
				double t = -w[size_t(c)] * Z[size_t(i) + size_t(c) * N];
				for (int j = 0; j < n; ++j)
					t += A[size_t(i) + size_t(j) * N] * Z[size_t(j) + size_t(c) * N];
				res = std::max(res, std::fabs(t));
			}
			for (int c2 = 0; c2 <= c; ++c2) {
				double s = 0.0;
				for (int i = 0; i < n; ++i)
					s += Z[size_t(i) + size_t(c) * N] * Z[size_t(i) + size_t(c2) * N];
				orth = std::max(orth, std::fabs(s - (c == c2 ? 1.0 : 0.0)));
			}
		}
		if (de > 1e-13 * scale || res > 1e-12 * scale || orth > 1e-12) {
			std::printf("FAIL full %d %g %g %g\n", trial, de, res, orth);
			return 1;
		}
		worst_e = std::max(worst_e, de / scale);
		worst_r = std::max(worst_r, res / scale);
	}
	// the top k eigenvectors by inverse iteration (tridiag_eigenvectors):
	// residuals and orthonormality, on random, graded and clustered
	// tridiagonals (exactly repeated diagonal blocks give repeated eigenvalues)
	for (int trial = 0; trial < 150; ++trial) {
		const int           n = 1 + (trial * 5) % 70;
		const size_t        N = size_t(n);
		std::vector<double> d(N), e(N, 0.0), w;
		for (int i = 0; i < n; ++i) {
			d[size_t(i)] = trial % 3 == 1 ? std::exp(-0.5 * i) * u(rng) : u(rng);
			e[size_t(i)] = trial % 3 == 1 ? 1e-3 * std::exp(-0.5 * i) * u(rng) : u(rng);
		}
		if (trial % 10 == 9) // the zero matrix (a density-matrix group without patches)
			std::fill(d.begin(), d.end(), 0.0), std::fill(e.begin(), e.end(), 0.0);
		else if (trial % 3 == 2 && n >= 4) // two decoupled copies of one block
			for (int i = 0; i < n / 2; ++i) {
				d[size_t(n / 2 + i)] = d[size_t(i)];
				e[size_t(n / 2 + i)] = i + 1 < n / 2 ? e[size_t(i)] : 0.0;
				if (i + 1 == n / 2)
					e[size_t(i)] = 0.0;
			}
		w = d;
		dmrgpp::tridiag_eigen(n, w.data(), e.data(), nullptr);
		const int           k = std::max(1, n / 3);
		std::vector<double> Z(N * size_t(k));
		dmrgpp::tridiag_eigenvectors(n, d.data(), e.data(), w.data() + (n - k), k, Z.data());
		double scale = 1.0, res = 0.0, orth = 0.0;
		for (double x : w)
			scale = std::max(scale, std::fabs(x));
		for (int c = 0; c < k; ++c) {
			const double th = w[size_t(n - k + c)];
			for (int i = 0; i < n; ++i) {
				double t = (d[size_t(i)] - th) * Z[size_t(i) + size_t(c) * N];
				if (i > 0)
					t += e[size_t(i - 1)] * Z[size_t(i - 1) + size_t(c) * N];
				if (i + 1 < n)
					t += e[size_t(i)] * Z[size_t(i + 1) + size_t(c) * N];
				res = std::max(res, std::fabs(t));
			}
			for (int c2 = 0; c2 <= c; ++c2) {
				double s = 0.0;
				for (int i = 0; i < n; ++i)
					s += Z[size_t(i) + size_t(c) * N] * Z[size_t(i) + size_t(c2) * N];
				orth = std::max(orth, std::fabs(s - (c == c2 ? 1.0 : 0.0)));
			}
		}
		if (res > 1e-12 * scale || orth > 1e-12) {
			std::printf("FAIL vectors %d %g %g\n", trial, res, orth);
			return 1;
		}
		worst_r = std::max(worst_r, res / scale);
	}
	// the thread-team Householder reduction: same eigenvalues, and Q from its
	// reflectors orthogonal, as the serial one
	for (int trial = 0; trial < 12; ++trial) {
		const int           n = 60 + 37 * trial;
		const size_t        N = size_t(n);
		std::vector<double> A(N * N);
		for (int j = 0; j < n; ++j)
			for (int i = 0; i <= j; ++i)
				A[size_t(i) + size_t(j) * N] = A[size_t(j) + size_t(i) * N] = u(rng);
		std::vector<double> d1, e1, h1, b1, d2, e2, h2, b2;
		dmrgpp::householder_tridiag(n, A.data(), d1, e1, h1, b1);
		dmrgpp::householder_tridiag_parallel(n, A.data(), d2, e2, h2, b2, 1 + trial % 7);
		dmrgpp::tridiag_eigen(n, d1.data(), e1.data(), nullptr);
		dmrgpp::tridiag_eigen(n, d2.data(), e2.data(), nullptr);
		double scale = 1.0, de = 0.0;
		for (int i = 0; i < n; ++i) {
			scale = std::max(scale, std::fabs(d1[size_t(i)]));
			de    = std::max(de, std::fabs(d1[size_t(i)] - d2[size_t(i)]));
		}
		if (de > 1e-12 * scale) {
			std::printf("FAIL parallel householder %d %g\n", n, de);
			return 1;
		}
		worst_e = std::max(worst_e, de / scale * 1e-1);
	}
	// the lowest eigenpair for the Lanczos Ritz vector (tridiag_lowest):
	// the energy bitwise tridiag_eigen's, the vector QL's first up to sign;
	// a pair degenerate to the last bit (two decoupled copies of one block,
	// as a Lanczos run without reorthogonalisation makes) takes QL's vector
	for (int trial = 0; trial < 60; ++trial) {
		const int           n    = 1 + (trial * 29) % 400;
		const bool          copy = trial % 6 == 5 && n >= 4;
		std::vector<double> d(static_cast<size_t>(n)), e(static_cast<size_t>(n), 0.0);
		for (int i = 0; i < n; ++i) {
			d[size_t(i)] = -2533.0 + 50.0 * u(rng);
			e[size_t(i)] = 20.0 + 5.0 * u(rng);
		}
		if (copy)
			for (int i = 0; i < n / 2; ++i) {
				d[size_t(n / 2 + i)] = d[size_t(i)];
				e[size_t(n / 2 + i)] = i + 1 < n / 2 ? e[size_t(i)] : 0.0;
				if (i + 1 == n / 2)
					e[size_t(i)] = 0.0;
			}
		std::vector<double> w(d), Z(size_t(n) * size_t(n)), z(static_cast<size_t>(n));
		dmrgpp::tridiag_eigen(n, w.data(), e.data(), Z.data());
		double theta = 0.0;
		if (!dmrgpp::tridiag_lowest(n, d.data(), e.data(), &theta, z.data()) || theta != w[0]) {
			std::printf("FAIL lowest value %d\n", trial);
			return 1;
		}
		double ov = 0.0, res = 0.0;
		for (int i = 0; i < n; ++i) {
			ov += z[size_t(i)] * Z[size_t(i)];
			double t = (d[size_t(i)] - theta) * z[size_t(i)];
			if (i > 0)
				t += e[size_t(i - 1)] * z[size_t(i - 1)];
			if (i + 1 < n)
				t += e[size_t(i)] * z[size_t(i + 1)];
			res = std::max(res, std::fabs(t));
		}
		const bool degenerate = n >= 2 && w[1] - w[0] <= 1e-8 * std::max(1.0, std::fabs(w[0]));
		if ((copy && !degenerate) || (degenerate && !std::equal(z.begin(), z.end(), Z.begin()))
		    || std::fabs(1.0 - std::fabs(ov)) > 1e-12 || res > 1e-11 * std::fabs(theta)) {
			std::printf("FAIL lowest vector %d n %d %g %g\n", trial, n, 1.0 - std::fabs(ov), res);
			return 1;
		}
		worst_r = std::max(worst_r, res / std::fabs(theta));
	}
	if (worst_e > 1e-13 || worst_r > 1e-12) {
		std::printf("FAIL %g %g\n", worst_e, worst_r);
		return 1;
	}
	std::printf("ok %.3e %.3e\n", worst_e, worst_r);
	return 0;
}
