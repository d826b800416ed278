// Density-matrix truncation after a sector solve (dmrgpp_density_truncate in
// dmrgpp_kron.h): the reference's per-patch SVD route
// (DensityMatrixSvd.h:285-410 ParallelPsiSplit / ParallelSvd, Truncation.h:
// 218-285 changeBasis, 373-519 updateKeptStates / computeKeptStates).
//
// The reference stacks, for every group g of the block being truncated, the
// sector-vector entries of all patches of g (one column block per patch and
// target, scaled by sqrt(weight)) into M_g and takes svd('A', M_g); the
// density-matrix eigenvalues are the squared singular values and the kept
// transformation is U.  Here rho_g = M_g M_g^T is formed directly as a sum of
// X_p^T X_p (system side) or X_p X_p^T (environment side) by one grouped DGEMM
// launch on the FP64 tensor pipe, the rho_g come to the host, are reduced to
// tridiagonal form and their eigenvalues found there, group by group on the
// host cores (Householder and implicit QL, tridiag.cpp), the eigenvectors are
// formed on the device from the recorded QL rotations and Householder
// reflectors, and the kept number follows computeKeptStates.
#include "devmem.h"
#include "trace.h"
#include "dmrgpp_kron.h"
#include "handle.h"
#include "kron_gemm.cuh"
#include "tridiag.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <climits>
#include <memory>
#include <cmath>
#include <numeric>
#include <string>
#include <vector>

namespace dmrgpp {
namespace {

// one 32 x 32 tile of a weighted transpose: XT (cols x rows, ld cols) =
// w * X (rows x cols, ld rows)
struct TransposeTile {
	long long src, dst;
	int       rows, cols, r0, c0;
	double    w;
};

__global__ void __launch_bounds__(256)
k_transpose_tiles(const double* __restrict__ x, double* __restrict__ xt, const TransposeTile* __restrict__ tiles,
                  int ntiles)
{
	__shared__ double s[32][33];
	const int         tx = threadIdx.x & 31, ty = threadIdx.x >> 5; // 32 x 8
	for (int q = blockIdx.x; q < ntiles; q += gridDim.x) {
		const TransposeTile t = tiles[q];
		__syncthreads();
		for (int j = ty; j < 32; j += 8) { // column c0 + j, row r0 + tx
			const int r = t.r0 + tx, c = t.c0 + j;
			s[j][tx]    = (r < t.rows && c < t.cols) ? x[t.src + r + (long long)c * t.rows] : 0.0;
		}
		__syncthreads();
		for (int j = ty; j < 32; j += 8) { // XT row c0 + tx, column r0 + j
			const int c = t.c0 + tx, r = t.r0 + j;
			if (r < t.rows && c < t.cols)
				xt[t.dst + c + (long long)r * t.cols] = t.w * s[tx][j];
		}
	}
}

// Eigenvectors on the device.  The host reduces each rho_g to tridiagonal
// form (Householder reflectors h_k, beta_k), finds all its eigenvalues (QL
// without vectors), ranks the states, and for the kept ones only computes
// the tridiagonal eigenvectors Z by inverse iteration; the device applies the
// reflectors to them (V = Q Z), the O(n^2) per vector part of the work.

// V[:, j] = Q Z[:, j] for every kept column j of every group: one warp per
// column, the reflectors h_k (k = n-3 .. 0) applied in turn to the column in
// global memory (it stays in L1)
struct ColumnJob {
	long long z_off, v_off, h_off, b_off; // Z and V (n x kept), reflectors (n x n), beta (n)
	int       n, src;                     // src: the Z column
	int       j;
	int       pad;
};

__global__ void __launch_bounds__(256)
k_back_transform(const double* __restrict__ z, double* __restrict__ v, const double* __restrict__ hv,
                 const double* __restrict__ beta, const ColumnJob* __restrict__ jobs, int njobs)
{
	const int lane = threadIdx.x & 31;
	for (int q = blockIdx.x * 8 + (threadIdx.x >> 5); q < njobs; q += gridDim.x * 8) {
		const ColumnJob jb = jobs[q];
		const int       n  = jb.n;
		double*         x  = v + jb.v_off + (long long)jb.j * n;
		const double*   zc = z + jb.z_off + (long long)jb.src * n;
		for (int i = lane; i < n; i += 32)
			x[i] = zc[i];
		__syncwarp();
		for (int k = n - 3; k >= 0; --k) {
			const double bk = beta[jb.b_off + k];
			if (bk == 0.0)
				continue;
			const double* h   = hv + jb.h_off + (long long)k * n; // h[0..len)
			const int     len = n - k - 1;
			double        s   = 0.0;
			for (int i = lane; i < len; i += 32)
				s += h[i] * x[k + 1 + i];
			for (int o = 16; o > 0; o >>= 1)
				s += __shfl_xor_sync(0xffffffffu, s, o);
			s *= bk;
			for (int i = lane; i < len; i += 32)
				x[k + 1 + i] -= s * h[i];
			__syncwarp();
		}
	}
}

// Truncation.h:476-512 (eigs ascending; tolerance < 0 keeps keptStates)
size_t compute_kept(size_t kept_states, double tolerance, size_t m_min, const std::vector<double>& eigs)
{
	if (tolerance < 0)
		return kept_states;
	const long long n     = (long long)eigs.size();
	long long       start = n - (long long)kept_states;
	if (start < 0)
		start = 0;
	long long max_to_remove = n - (long long)m_min;
	if (max_to_remove < 0)
		max_to_remove = 0;
	size_t total = m_min;
	double disc  = 0.0;
	for (long long i = 0; i < start; ++i)
		disc += std::fabs(eigs[size_t(i)]);
	for (long long i = start; i < max_to_remove; ++i) {
		disc += std::fabs(eigs[size_t(i)]);
		if (disc > tolerance) {
			total = size_t(n - i);
			break;
		}
	}
	if (total >= kept_states)
		return kept_states;
	if (total < m_min)
		return m_min;
	return total;
}

int fail(int status, const std::string& msg) { return handle_fail(nullptr, status, msg); }

using Clock = std::chrono::steady_clock;
thread_local double g_trunc_times[DMRGPP_TRUNC_NPHASES] = {};

// Page-locked host buffers of the calling thread, kept between calls (the
// density matrices, reflectors and vectors cross PCIe every call; pageable
// copies and first-touch page faults would cost more than the transfers).
struct PinnedSlot {
	void*  p   = nullptr;
	size_t cap = 0;
	~PinnedSlot()
	{
		if (p)
			cudaFreeHost(p);
	}
};
thread_local PinnedSlot g_pinned[4];

template <class T> T* pinned(int slot, size_t n)
{
	PinnedSlot& s     = g_pinned[slot];
	const size_t bytes = std::max<size_t>(n, 1) * sizeof(T);
	if (s.cap < bytes) {
		if (s.p)
			cudaFreeHost(s.p);
		s.p   = nullptr;
		s.cap = 0;
		if (cudaHostAlloc(&s.p, bytes, cudaHostAllocDefault) != cudaSuccess)
			return nullptr;
		s.cap = bytes;
	}
	return static_cast<T*>(s.p);
}

double seconds_since(Clock::time_point t0) { return std::chrono::duration<double>(Clock::now() - t0).count(); }

int cuda_fail(cudaError_t e, const char* where)
{
	return fail(e == cudaErrorMemoryAllocation ? DMRGPP_OOM : DMRGPP_CUDA_ERROR,
	            std::string(where) + ": " + cudaGetErrorString(e));
}

} // namespace
} // namespace dmrgpp

extern "C" int dmrgpp_density_truncate(const dmrgpp_density_desc* d, size_t m, double tolerance,
                                       size_t m_min, double* eigenvalues, double* vectors, size_t* kept,
                                       size_t* kept_total, double* discarded)
{
	DMRGPP_TRACE("dmrgpp_density_truncate");
	using namespace dmrgpp;
	if (!d || !eigenvalues || !kept || !kept_total || !discarded)
		return fail(DMRGPP_INVALID_ARG, "null argument");
	if (d->npatches == 0 || d->ngroups == 0 || d->ntargets == 0)
		return fail(DMRGPP_INVALID_ARG, "npatches, ngroups and ntargets must be >= 1");
	if (!d->left_patch_size || !d->right_patch_size || !d->patch_group || !d->group_size || !d->psi)
		return fail(DMRGPP_INVALID_ARG, "null table");
	if (d->side != 0 && d->side != 1)
		return fail(DMRGPP_INVALID_ARG, "side must be 0 (system) or 1 (environment)");
	const size_t np = d->npatches, ng = d->ngroups, nt = d->ntargets;
	const auto   t_start = Clock::now();
	for (double& x : g_trunc_times)
		x = 0.0;
	// sector layout, group membership and sizes
	std::vector<long long> xy(np + 1, 0);
	for (size_t p = 0; p < np; ++p) {
		const size_t l = d->left_patch_size[p], r = d->right_patch_size[p];
		if (l < 1 || r < 1 || l > size_t(INT_MAX) || r > size_t(INT_MAX))
			return fail(DMRGPP_INVALID_ARG, "patch " + std::to_string(p) + " has an empty or oversized group");
		if (d->patch_group[p] >= ng)
			return fail(DMRGPP_INVALID_ARG, "patch " + std::to_string(p) + ": group out of range");
		const size_t n = d->side == 0 ? l : r;
		if (d->group_size[d->patch_group[p]] != n)
			return fail(DMRGPP_INVALID_ARG,
			            "patch " + std::to_string(p) + ": its group's size differs from the patch's "
			                + (d->side == 0 ? "left" : "right") + " size");
		xy[p + 1] = xy[p] + (long long)(l * r);
	}
	const long long D = xy[np];
	std::vector<long long> goff(ng + 1, 0);
	size_t                 nmax = 0, N = 0;
	for (size_t g = 0; g < ng; ++g) {
		const size_t n = d->group_size[g];
		if (n > 46340) // n^2 within INT_MAX for the GEMM tiles' leading dimensions
			return fail(DMRGPP_INVALID_ARG, "group " + std::to_string(g) + " is too large");
		goff[g + 1] = goff[g] + (long long)(n * n);
		nmax        = std::max(nmax, n);
		N += n;
	}
	if (m_min > m)
		return fail(DMRGPP_INVALID_ARG, "m_min must not exceed m");
	std::vector<double> w(nt, 1.0);
	if (d->weights)
		for (size_t t = 0; t < nt; ++t)
			w[t] = d->weights[t];

	int prev = -1;
	cudaGetDevice(&prev);
	const int dev = d->device >= 0 ? d->device : prev;
	if (dev != prev && cudaSetDevice(dev) != cudaSuccess)
		return fail(DMRGPP_INVALID_ARG, "cannot select device " + std::to_string(dev));
	struct Restore {
		int dev, prev;
		~Restore()
		{
			if (dev != prev && prev >= 0)
				cudaSetDevice(prev);
		}
	} restore { dev, prev };
	cudaStream_t st = static_cast<cudaStream_t>(d->stream);

	// weighted transposed copies of every patch block, and the GEMM lists:
	// side 0: rho_g += (w X_p^T)(X_p), A = XT (l x r), B = X (r x l), K = r
	// side 1: rho_g += (X_p)(w X_p^T), A = X (r x l), B = XT (l x r), K = l
	std::vector<TransposeTile> tt;
	std::vector<std::vector<GemmSeg>> gseg(ng);
	for (size_t t = 0; t < nt; ++t)
		for (size_t p = 0; p < np; ++p) {
			const int       l = int(d->left_patch_size[p]), r = int(d->right_patch_size[p]);
			const long long off = (long long)t * D + xy[p];
			for (int c0 = 0; c0 < l; c0 += 32)
				for (int r0 = 0; r0 < r; r0 += 32)
					tt.push_back({ off, off, r, l, r0, c0, w[t] });
			GemmSeg s {};
			s.a_off = off;
			s.b_off = off;
			if (d->side == 0) {
				s.lda = l;
				s.ldb = r;
				s.K   = r;
			} else {
				s.lda = r;
				s.ldb = l;
				s.K   = l;
			}
			s.dep = int(p);
			gseg[d->patch_group[p]].push_back(s);
		}
	const int            bm = nmax > 192 ? 64 : 32;
	std::vector<GemmSeg>  segs;
	std::vector<GemmTile> tiles;
	for (size_t g = 0; g < ng; ++g) {
		if (gseg[g].empty())
			continue;
		const int sb = int(segs.size());
		segs.insert(segs.end(), gseg[g].begin(), gseg[g].end());
		const int n = int(d->group_size[g]);
		for (int n0 = 0; n0 < n; n0 += bm)
			for (int m0 = 0; m0 < n; m0 += bm) {
				GemmTile tl {};
				tl.c_off     = goff[g];
				tl.ldc       = n;
				tl.M         = n;
				tl.N         = n;
				tl.m0        = m0;
				tl.n0        = n0;
				tl.seg_begin = sb;
				tl.seg_end   = int(segs.size());
				tiles.push_back(tl);
			}
	}

	double*        xt    = nullptr;
	double*        rho   = nullptr;
	TransposeTile* d_tt  = nullptr;
	GemmSeg*       d_seg = nullptr;
	GemmTile*      d_til = nullptr;
	struct Free {
		double**        a;
		double**        b;
		TransposeTile** c;
		GemmSeg**       s;
		GemmTile**      t;
		~Free()
		{
			dev_free(*a);
			dev_free(*b);
			dev_free(*c);
			dev_free(*s);
			dev_free(*t);
		}
	} release { &xt, &rho, &d_tt, &d_seg, &d_til };
	cudaError_t e;
	const size_t rho_elems = size_t(std::max<long long>(goff[ng], 1));
	if ((e = init_grouped_dgemm()) || (e = dev_malloc(&xt, size_t(nt) * size_t(std::max<long long>(D, 1)) * sizeof(double)))
	    || (e = dev_malloc(&rho, rho_elems * sizeof(double)))
	    || (e = dev_malloc(&d_tt, std::max<size_t>(tt.size(), 1) * sizeof(TransposeTile)))
	    || (e = dev_malloc(&d_seg, std::max<size_t>(segs.size(), 1) * sizeof(GemmSeg)))
	    || (e = dev_malloc(&d_til, std::max<size_t>(tiles.size(), 1) * sizeof(GemmTile))))
		return cuda_fail(e, "density-matrix allocation");
	if ((e = cudaMemcpyAsync(d_tt, tt.data(), tt.size() * sizeof(TransposeTile), cudaMemcpyHostToDevice, st))
	    || (e = cudaMemcpyAsync(d_seg, segs.data(), segs.size() * sizeof(GemmSeg), cudaMemcpyHostToDevice, st))
	    || (e = cudaMemcpyAsync(d_til, tiles.data(), tiles.size() * sizeof(GemmTile), cudaMemcpyHostToDevice, st))
	    || (e = cudaMemsetAsync(rho, 0, rho_elems * sizeof(double), st)))
		return cuda_fail(e, "density-matrix set-up");
	const int tgrid = int(std::min<size_t>(std::max<size_t>(tt.size(), 1), 148 * 16));
	k_transpose_tiles<<<tgrid, 256, 0, st>>>(d->psi, xt, d_tt, int(tt.size()));
	if (!tiles.empty()) {
		GemmArgs ga {};
		ga.A      = d->side == 0 ? xt : d->psi;
		ga.B      = d->side == 0 ? d->psi : xt;
		ga.C      = rho;
		ga.segs   = d_seg;
		ga.tiles  = d_til;
		ga.ntiles = int(tiles.size());
		if ((e = launch_grouped_dgemm(ga, bm, bm, st)))
			return cuda_fail(e, "density-matrix GEMM launch");
	}
	double* h_rho = pinned<double>(0, rho_elems);
	if (!h_rho)
		return fail(DMRGPP_OOM, "page-locked host buffer for the density matrices");
	if ((e = cudaGetLastError()) || (e = cudaMemcpyAsync(h_rho, rho, rho_elems * sizeof(double), cudaMemcpyDeviceToHost, st))
	    || (e = cudaStreamSynchronize(st)))
		return cuda_fail(e, "density matrices");

	g_trunc_times[DMRGPP_TRUNC_RHO] = seconds_since(t_start);
	auto tp                         = Clock::now();
	// eigenvalues of every group on the host cores (Householder reduction,
	// QL without vectors)
	std::vector<long long> eoff(ng + 1, 0);
	for (size_t g = 0; g < ng; ++g)
		eoff[g + 1] = eoff[g] + (long long)d->group_size[g];
	// largest groups first (the order of the eigenvector work below)
	std::vector<size_t> by_size(ng);
	std::iota(by_size.begin(), by_size.end(), size_t(0));
	std::stable_sort(by_size.begin(), by_size.end(),
	                 [&](size_t x, size_t y) { return d->group_size[x] > d->group_size[y]; });
	std::vector<double*> ga(ng), gw(ng);
	for (size_t g = 0; g < ng; ++g) {
		ga[g] = h_rho + goff[g];
		gw[g] = eigenvalues + eoff[g];
	}
	std::vector<GroupReduction> ge;
	const int                   hw = host_threads();
	if (!group_eigenvalues(ng, d->group_size, ga.data(), gw.data(), ge, hw)) {
		size_t g = 0;
		while (g < ng && ge[g].ok)
			++g;
		return fail(DMRGPP_NOT_CONVERGED, "eigensolver of group " + std::to_string(g) + " did not converge");
	}

	g_trunc_times[DMRGPP_TRUNC_EIGENVALUES] = seconds_since(tp);
	tp                                      = Clock::now();
	// rank every state (ascending eigenvalue, then group, then index) and keep K
	std::vector<long long> order(N);
	std::iota(order.begin(), order.end(), 0LL);
	std::vector<size_t> group_of(N);
	for (size_t g = 0; g < ng; ++g)
		for (long long q = eoff[g]; q < eoff[g + 1]; ++q)
			group_of[size_t(q)] = g;
	std::stable_sort(order.begin(), order.end(),
	                 [&](long long a, long long b) { return eigenvalues[a] < eigenvalues[b]; });
	std::vector<double> sorted(N);
	for (size_t q = 0; q < N; ++q)
		sorted[q] = eigenvalues[order[q]];
	const size_t K      = std::min(compute_kept(m, tolerance, m_min, sorted), N);
	const size_t remove = N - K;
	double       disc   = 0.0;
	for (size_t g = 0; g < ng; ++g)
		kept[g] = d->group_size[g];
	for (size_t q = 0; q < remove; ++q) {
		disc += std::fabs(sorted[q]);
		--kept[group_of[size_t(order[q])]];
	}
	g_trunc_times[DMRGPP_TRUNC_SELECT] = seconds_since(tp);
	tp                                 = Clock::now();
	if (vectors) {
		// the kept eigenvectors: inverse iteration on each tridiagonal (host
		// cores), then V = Q Z on the device
		std::vector<long long> koff(ng + 1, 0);
		for (size_t g = 0; g < ng; ++g)
			koff[g + 1] = koff[g] + (long long)(d->group_size[g] * kept[g]);
		const size_t        kelems = size_t(std::max<long long>(koff[ng], 1));
		// the packed reflectors: every group with kept states copies its whole
		// n x n block; the rest is never read
		double* hv = pinned<double>(1, rho_elems);
		double* zk = pinned<double>(2, kelems);
		double* vo = pinned<double>(3, kelems);
		if (!hv || !zk || !vo)
			return fail(DMRGPP_OOM, "page-locked host buffers for the eigenvectors");
		std::vector<double> bt(size_t(std::max<long long>(eoff[ng], 1)), 0.0);
		std::vector<const double*> gwk(ng);
		std::vector<double*>       gz(ng);
		for (size_t g = 0; g < ng; ++g) {
			gwk[g] = eigenvalues + eoff[g] + (long long)(d->group_size[g] - kept[g]);
			gz[g]  = zk + koff[g];
		}
		group_eigenvectors(ng, d->group_size, kept, ge.data(), gwk.data(), gz.data(), hw);
		parallel_for(ng, [&](size_t t) {
			const size_t g = by_size[t];
			if (kept[g] == 0)
				return;
			std::copy(ge[g].hv.begin(), ge[g].hv.end(), hv + goff[g]);
			std::copy(ge[g].beta.begin(), ge[g].beta.end(), bt.begin() + eoff[g]);
		});
		g_trunc_times[DMRGPP_TRUNC_VECTORS_HOST] = seconds_since(tp);
		tp                                       = Clock::now();
		std::vector<ColumnJob> cj;
		for (size_t g = 0; g < ng; ++g)
			for (int j = 0; j < int(kept[g]); ++j)
				cj.push_back({ koff[g], koff[g], goff[g], eoff[g], int(d->group_size[g]), j, j, 0 });
		if (!cj.empty()) {
			double *   z = nullptr, *v = nullptr, *d_hv = nullptr, *d_bt = nullptr;
			ColumnJob* d_cj = nullptr;
			struct FreeV {
				double**    a[4];
				ColumnJob** j;
				~FreeV()
				{
					for (double** p : a)
						dev_free(*p);
					dev_free(*j);
				}
			} freev { { &z, &v, &d_hv, &d_bt }, &d_cj };
			if ((e = dev_malloc(&z, kelems * sizeof(double))) || (e = dev_malloc(&v, kelems * sizeof(double)))
			    || (e = dev_malloc(&d_hv, rho_elems * sizeof(double))) || (e = dev_malloc(&d_bt, bt.size() * sizeof(double)))
			    || (e = dev_malloc(&d_cj, cj.size() * sizeof(ColumnJob))))
				return cuda_fail(e, "eigenvector allocation");
			if ((e = cudaMemcpyAsync(z, zk, kelems * sizeof(double), cudaMemcpyHostToDevice, st))
			    || (e = cudaMemcpyAsync(d_hv, hv, rho_elems * sizeof(double), cudaMemcpyHostToDevice, st))
			    || (e = cudaMemcpyAsync(d_bt, bt.data(), bt.size() * sizeof(double), cudaMemcpyHostToDevice, st))
			    || (e = cudaMemcpyAsync(d_cj, cj.data(), cj.size() * sizeof(ColumnJob), cudaMemcpyHostToDevice, st)))
				return cuda_fail(e, "eigenvector set-up");
			const int cgrid = int(std::min<size_t>((cj.size() + 7) / 8, 148 * 8));
			k_back_transform<<<std::max(cgrid, 1), 256, 0, st>>>(z, v, d_hv, d_bt, d_cj, int(cj.size()));
			if ((e = cudaGetLastError())
			    || (e = cudaMemcpyAsync(vo, v, size_t(koff[ng]) * sizeof(double), cudaMemcpyDeviceToHost, st))
			    || (e = cudaStreamSynchronize(st)))
				return cuda_fail(e, "eigenvectors");
			parallel_for(ng, [&](size_t g) { // to the caller's (pageable) buffer, group by group
				std::copy(vo + koff[g], vo + koff[g + 1], vectors + koff[g]);
			});
		}
	}
	if (vectors)
		g_trunc_times[DMRGPP_TRUNC_VECTORS_DEVICE] = seconds_since(tp);
	g_trunc_times[DMRGPP_TRUNC_TOTAL] = seconds_since(t_start);
	*kept_total                       = K;
	*discarded                        = disc;
	return DMRGPP_OK;
}

extern "C" int dmrgpp_density_profile(double* t, int n)
{
	if (!t || n < 0 || n > DMRGPP_TRUNC_NPHASES)
		return dmrgpp::fail(DMRGPP_INVALID_ARG, "need 0 <= n <= DMRGPP_TRUNC_NPHASES and a buffer");
	for (int i = 0; i < n; ++i)
		t[i] = dmrgpp::g_trunc_times[i];
	return DMRGPP_OK;
}
