// Device-resident Lanczos for the lowest eigenpair of one sector, plus the
// bandwidth-bound vector kernels it is made of and the sector gather/scatter.
//
// The recurrence follows PsimagLite's LanczosCore::decomposition
// (PsimagLite/src/PsimagLite/LanczosCore.h:147-272) and
// LanczosVectors::oneStepDecomposition / reorthoIfNecessary
// (LanczosVectors.h:203-271) step by step: normalise the initial vector,
// V1 = H V0 - a0 V0, then for j >= 1: V2 = H V1, a_j = <V2,V1>,
// V2 -= a_j V1 + b_j V0, b_{j+1} = |V2|, V2 /= b_{j+1}, optional full
// reorthogonalisation against the stored vectors and renormalisation, then
// the stopping test on the lowest Ritz values (LanczosCore.h:222-240).
// Differences: the reorthogonalisation computes all projections from the
// same vector (classical Gram-Schmidt, two GEMV passes over the stored basis)
// where the reference subtracts them one at a time; and the host reads a_j,
// b_j back every `check_every` steps, applying the stopping test to each step
// in order (steps run past the stopping point are discarded).
//
// Reductions are deterministic: per-block partials in fixed-size grids, the
// last block to finish (arrival counter) sums them in block order.
#include "dmrgpp_kron.h"
#include "trace.h"
#include "devmem.h"
#include "handle.h"
#include "tridiag.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <string>
#include <limits>
#include <vector>

namespace dmrgpp {

namespace {

constexpr int kThreads   = 256;
constexpr int kMaxBlocks = 1184; // 8 per SM of a B200
constexpr int kDotGrid   = 592;  // blocks of the basis projections (4 per SM)
constexpr int kDotChunk  = 2048; // rows per block iteration of the basis projections
constexpr int kMaxCols   = 1024; // stored Lanczos vectors per solve

// blocks of the row-parallel basis kernels: at least 256 rows each
int basis_blocks_for(size_t n)
{
	const size_t b = (n + 255) / 256;
	return int(std::max<size_t>(1, std::min<size_t>(b, kMaxBlocks)));
}

int blocks_for(size_t n)
{
	const size_t b = (n + size_t(kThreads) * 4 - 1) / (size_t(kThreads) * 4);
	return int(std::max<size_t>(1, std::min<size_t>(b, kMaxBlocks)));
}

__device__ __forceinline__ double block_sum(double v, double* red)
{
	for (int o = 16; o > 0; o >>= 1)
		v += __shfl_down_sync(0xffffffffu, v, o);
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	if (lane == 0)
		red[warp] = v;
	__syncthreads();
	double s = 0.0;
	if (threadIdx.x == 0)
		for (int w = 0; w < kThreads / 32; ++w)
			s += red[w];
	__syncthreads();
	return s; // valid in thread 0
}

// Called by thread 0 after writing this block's partial: true in the last
// block to arrive; the counter is reset for the next launch.
__device__ __forceinline__ bool last_block(unsigned* ctr)
{
	__threadfence();
	const unsigned old = atomicAdd(ctr, 1u);
	if (old == gridDim.x - 1) {
		__threadfence();
		*ctr = 0u;
		return true;
	}
	return false;
}

// Grid-wide sum of one value per block, deterministic: every block stores its
// value, the last block to arrive sums them with all its threads (fixed
// strided order, then a fixed tree) and thread 0 writes *out (its square root
// when root is set).  All threads of every block must call it.
__device__ __forceinline__ void grid_sum(double block_value, double* partial, unsigned* ctr,
                                         double* out, bool root, double* red)
{
	__shared__ bool last;
	if (threadIdx.x == 0) {
		partial[blockIdx.x] = block_value;
		last                = last_block(ctr);
	}
	__syncthreads();
	if (!last)
		return;
	double t = 0.0;
	for (int b = threadIdx.x; b < int(gridDim.x); b += blockDim.x)
		t += __ldcg(partial + b);
	t = block_sum(t, red);
	if (threadIdx.x == 0)
		*out = root ? sqrt(t) : t;
}

// *out = <x, y>
__device__ __forceinline__ void dot_body(const double* __restrict__ x, const double* __restrict__ y,
                                         size_t n, double* out, double* partial, unsigned* ctr)
{
	__shared__ double red[kThreads / 32];
	double            s = 0.0;
	for (size_t i = blockIdx.x * size_t(kThreads) + threadIdx.x; i < n;
	     i += size_t(gridDim.x) * kThreads)
		s += x[i] * y[i];
	s = block_sum(s, red);
	grid_sum(s, partial, ctr, out, false, red);
}

__global__ void __launch_bounds__(kThreads)
k_dot(const double* __restrict__ x, const double* __restrict__ y, size_t n, double* out,
      double* partial, unsigned* ctr)
{
	dot_body(x, y, n, out, partial, ctr);
}

// dst = src / sqrt(*nrm2) (nrm2 = <src,src> from k_dot)
__global__ void __launch_bounds__(kThreads)
k_scale_rsqrt(const double* src, double* dst, size_t n, const double* nrm2)
{
	const double a = 1.0 / sqrt(*nrm2);
	for (size_t i = blockIdx.x * size_t(kThreads) + threadIdx.x; i < n;
	     i += size_t(gridDim.x) * kThreads)
		dst[i] = src[i] * a;
}

// v2 = v2 - alpha*v1 - beta*v0 (v0 may be null); *beta_out = |v2|
__device__ __forceinline__ void update_body(double* __restrict__ v2, const double* __restrict__ v1,
                                            const double* __restrict__ v0, size_t n,
                                            const double* alpha, const double* beta,
                                            double* beta_out, double* partial, unsigned* ctr)
{
	__shared__ double red[kThreads / 32];
	const double      a = *alpha;
	const double      b = v0 ? *beta : 0.0;
	double            s = 0.0;
	for (size_t i = blockIdx.x * size_t(kThreads) + threadIdx.x; i < n;
	     i += size_t(gridDim.x) * kThreads) {
		double w = v2[i] - a * v1[i];
		if (v0)
			w -= b * v0[i];
		v2[i] = w;
		s += w * w;
	}
	s = block_sum(s, red);
	grid_sum(s, partial, ctr, beta_out, true, red);
}

__global__ void __launch_bounds__(kThreads)
k_lanczos_update(double* __restrict__ v2, const double* __restrict__ v1,
                 const double* __restrict__ v0, size_t n, const double* alpha,
                 const double* beta, double* beta_out, double* partial, unsigned* ctr)
{
	update_body(v2, v1, v0, n, alpha, beta, beta_out, partial, ctr);
}

// v *= 1 / *s when *s > 0 (LanczosVectors.h:233-237)
__device__ __forceinline__ void scale_inv_body(double* v, size_t n, const double* s)
{
	const double d = *s;
	if (!(d > 0.0))
		return;
	const double a = 1.0 / d;
	for (size_t i = blockIdx.x * size_t(kThreads) + threadIdx.x; i < n;
	     i += size_t(gridDim.x) * kThreads)
		v[i] *= a;
}

__global__ void __launch_bounds__(kThreads) k_scale_inv(double* v, size_t n, const double* s)
{
	scale_inv_body(v, n, s);
}

// Per-block partial projections partial[b][c] = <V[rows of b, c], v[rows of b]>
// for c < ncols.  Block b takes the kDotChunk-row chunks b, b + grid, ...;
// each chunk of v is staged in shared memory and every warp streams whole
// columns of it (warp w: columns w, w + 8, ...).  VEC: 16-byte loads (V, v
// 16-byte aligned and ld even), 8 loads in flight per lane.  The order of
// every sum is fixed, so results are bitwise reproducible.
template <bool VEC>
__device__ __forceinline__ void basis_dots_body(const double* __restrict__ V, size_t ld, int ncols,
                                                const double* __restrict__ v, size_t n,
                                                double* __restrict__ partial)
{
	__shared__ __align__(16) double vs[kDotChunk];
	__shared__ double acc[kMaxCols];
	const int         lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	for (int c = threadIdx.x; c < ncols; c += kThreads)
		acc[c] = 0.0;
	for (size_t base = size_t(blockIdx.x) * kDotChunk; base < n; base += size_t(gridDim.x) * kDotChunk) {
		const int len = int(std::min<size_t>(kDotChunk, n - base));
		__syncthreads();
		for (int i = threadIdx.x; i < len; i += kThreads)
			vs[i] = v[base + i];
		__syncthreads();
		for (int c = warp; c < ncols; c += kThreads / 32) {
			const double* col = V + size_t(c) * ld + base;
			double        s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
			if (VEC && len == kDotChunk) {
				const double2* c2 = reinterpret_cast<const double2*>(col);
				const double2* v2 = reinterpret_cast<const double2*>(vs);
#pragma unroll 2
				for (int q = lane; q < kDotChunk / 2; q += 128) {
					const double2 a0 = __ldg(c2 + q), a1 = __ldg(c2 + q + 32);
					const double2 a2 = __ldg(c2 + q + 64), a3 = __ldg(c2 + q + 96);
					const double2 b0 = v2[q], b1 = v2[q + 32], b2 = v2[q + 64], b3 = v2[q + 96];
					s0 += a0.x * b0.x + a0.y * b0.y;
					s1 += a1.x * b1.x + a1.y * b1.y;
					s2 += a2.x * b2.x + a2.y * b2.y;
					s3 += a3.x * b3.x + a3.y * b3.y;
				}
			} else {
				int i = lane;
				for (; i + 96 < len; i += 128) {
					s0 += col[i] * vs[i];
					s1 += col[i + 32] * vs[i + 32];
					s2 += col[i + 64] * vs[i + 64];
					s3 += col[i + 96] * vs[i + 96];
				}
				for (; i < len; i += 32)
					s0 += col[i] * vs[i];
			}
			double s = (s0 + s1) + (s2 + s3);
			for (int o = 16; o > 0; o >>= 1)
				s += __shfl_down_sync(0xffffffffu, s, o);
			if (lane == 0)
				acc[c] += s;
		}
	}
	__syncthreads();
	for (int c = threadIdx.x; c < ncols; c += kThreads)
		partial[size_t(blockIdx.x) * kMaxCols + c] = acc[c];
}

template <bool VEC>
__global__ void __launch_bounds__(kThreads, 4)
k_basis_dots(const double* __restrict__ V, size_t ld, int ncols, const double* __restrict__ v,
             size_t n, double* __restrict__ partial)
{
	basis_dots_body<VEC>(V, ld, ncols, v, n, partial);
}

// r[c] = sum over blocks b < nblocks of partial[b][c], one block per column,
// fixed order
__device__ __forceinline__ void reduce_cols_body(const double* __restrict__ partial, int nblocks,
                                                 double* __restrict__ r)
{
	__shared__ double red[kThreads / 32];
	const int         c = blockIdx.x;
	double            s = 0.0;
	for (int b = threadIdx.x; b < nblocks; b += kThreads)
		s += partial[size_t(b) * kMaxCols + c];
	s = block_sum(s, red);
	if (threadIdx.x == 0)
		r[c] = s;
}

__global__ void __launch_bounds__(kThreads)
k_reduce_cols(const double* __restrict__ partial, int nblocks, double* __restrict__ r)
{
	reduce_cols_body(partial, nblocks, r);
}

// v -= V[:, 0..ncols) r ; *nrm_out = |v|.  VEC: each thread owns row pairs
// (16-byte loads), 8 columns of loads issued before their updates; the
// subtractions run in column order, as in the scalar form.
template <bool VEC>
__device__ __forceinline__ void basis_subtract_body(double* __restrict__ v, const double* __restrict__ V,
                                                    size_t ld, int ncols, const double* __restrict__ r,
                                                    size_t n, double* nrm_out, double* partial,
                                                    unsigned* ctr)
{
	__shared__ double rs[kMaxCols];
	__shared__ double red[kThreads / 32];
	for (int c = threadIdx.x; c < ncols; c += kThreads)
		rs[c] = r[c];
	__syncthreads();
	double       s      = 0.0;
	const size_t stride = size_t(gridDim.x) * kThreads;
	const size_t first  = blockIdx.x * size_t(kThreads) + threadIdx.x;
	if (VEC) {
		double2*     v2  = reinterpret_cast<double2*>(v);
		const size_t np2 = n / 2;
		for (size_t p = first; p < np2; p += stride) {
			double2 w = v2[p];
			int     c = 0;
			for (; c + 8 <= ncols; c += 8) {
				double2 a[8];
#pragma unroll
				for (int u = 0; u < 8; ++u)
					a[u] = __ldg(reinterpret_cast<const double2*>(V + size_t(c + u) * ld) + p);
#pragma unroll
				for (int u = 0; u < 8; ++u) {
					w.x -= a[u].x * rs[c + u];
					w.y -= a[u].y * rs[c + u];
				}
			}
			for (; c < ncols; ++c) {
				const double2 a = __ldg(reinterpret_cast<const double2*>(V + size_t(c) * ld) + p);
				w.x -= a.x * rs[c];
				w.y -= a.y * rs[c];
			}
			v2[p] = w;
			s += w.x * w.x + w.y * w.y;
		}
		if ((n & 1) && first == 0) { // odd length: the last element
			const size_t i = n - 1;
			double       w = v[i];
			for (int c = 0; c < ncols; ++c)
				w -= V[size_t(c) * ld + i] * rs[c];
			v[i] = w;
			s += w * w;
		}
	} else {
		for (size_t i = first; i < n; i += stride) {
			double w = v[i];
			for (int c = 0; c < ncols; ++c)
				w -= V[size_t(c) * ld + i] * rs[c];
			v[i] = w;
			s += w * w;
		}
	}
	s = block_sum(s, red);
	grid_sum(s, partial, ctr, nrm_out, true, red);
}

template <bool VEC>
__global__ void __launch_bounds__(kThreads)
k_basis_subtract(double* __restrict__ v, const double* __restrict__ V, size_t ld, int ncols,
                 const double* __restrict__ r, size_t n, double* nrm_out, double* partial,
                 unsigned* ctr)
{
	basis_subtract_body<VEC>(v, V, ld, ncols, r, n, nrm_out, partial, ctr);
}

// ---- one Lanczos step with its columns chosen on the device, so that a
// captured CUDA graph of check_every steps is replayed unchanged for the
// whole solve.  k_step_advance moves the step record to the next j before
// every step (LanczosVectors::oneStepDecomposition, LanczosVectors.h:203-241).
struct LanczosStep {
	StepIO  io;      // the step's H*x: x = V_j, y = V_{j+1}
	double* v0;      // V_{j-1}
	double* v1;      // V_j
	double* v2;      // V_{j+1}
	double* alpha_j;
	double* beta_j;
	double* beta_j1;
	int     ncols;   // j + 1 stored vectors (reorthogonalisation)
	int     j;
};

__global__ void k_step_set(LanczosStep* sp, int j) { sp->j = j; }

__global__ void k_step_advance(LanczosStep* sp, double* V, size_t D, double* alpha, double* beta)
{
	const int j = sp->j + 1;
	sp->j       = j;
	sp->v0      = V + size_t(j - 1) * D;
	sp->v1      = V + size_t(j) * D;
	sp->v2      = V + size_t(j + 1) * D;
	sp->io.x    = sp->v1;
	sp->io.y    = sp->v2;
	sp->alpha_j = alpha + j;
	sp->beta_j  = beta + j;
	sp->beta_j1 = beta + j + 1;
	sp->ncols   = j + 1;
}

__global__ void __launch_bounds__(kThreads)
k_dot_step(const LanczosStep* sp, size_t n, double* partial, unsigned* ctr)
{
	dot_body(sp->v2, sp->v1, n, sp->alpha_j, partial, ctr);
}

__global__ void __launch_bounds__(kThreads)
k_update_step(const LanczosStep* sp, size_t n, double* partial, unsigned* ctr)
{
	update_body(sp->v2, sp->v1, sp->v0, n, sp->alpha_j, sp->beta_j, sp->beta_j1, partial, ctr);
}

// v2 *= 1 / *s (s = beta_{j+1} when null)
__global__ void __launch_bounds__(kThreads)
k_scale_inv_step(const LanczosStep* sp, size_t n, const double* s)
{
	scale_inv_body(sp->v2, n, s ? s : sp->beta_j1);
}

template <bool VEC>
__global__ void __launch_bounds__(kThreads, 4)
k_basis_dots_step(const LanczosStep* sp, const double* __restrict__ V, size_t ld, size_t n,
                  double* __restrict__ partial)
{
	basis_dots_body<VEC>(V, ld, sp->ncols, sp->v2, n, partial);
}

// launched with the largest column count; blocks past the step's ncols exit
__global__ void __launch_bounds__(kThreads)
k_reduce_cols_step(const LanczosStep* sp, const double* __restrict__ partial, int nblocks,
                   double* __restrict__ r)
{
	if (int(blockIdx.x) >= sp->ncols)
		return;
	reduce_cols_body(partial, nblocks, r);
}

template <bool VEC>
__global__ void __launch_bounds__(kThreads)
k_basis_subtract_step(const LanczosStep* sp, const double* __restrict__ V, size_t ld,
                      const double* __restrict__ r, size_t n, double* nrm_out, double* partial,
                      unsigned* ctr)
{
	basis_subtract_body<VEC>(sp->v2, V, ld, sp->ncols, r, n, nrm_out, partial, ctr);
}

// z = sum_c coef[c] V[:, c] (LanczosVectors::excitedVector, LanczosVectors.h:192-201)
template <bool VEC>
__global__ void __launch_bounds__(kThreads)
k_basis_combine(double* __restrict__ z, const double* __restrict__ V, size_t ld, int ncols,
                const double* __restrict__ coef, size_t n)
{
	__shared__ double cs[kMaxCols];
	for (int c = threadIdx.x; c < ncols; c += kThreads)
		cs[c] = coef[c];
	__syncthreads();
	const size_t stride = size_t(gridDim.x) * kThreads;
	const size_t first  = blockIdx.x * size_t(kThreads) + threadIdx.x;
	if (VEC) {
		const size_t np2 = n / 2;
		for (size_t p = first; p < np2; p += stride) {
			double2 w = make_double2(0.0, 0.0);
			int     c = 0;
			for (; c + 8 <= ncols; c += 8) {
				double2 a[8];
#pragma unroll
				for (int u = 0; u < 8; ++u)
					a[u] = __ldg(reinterpret_cast<const double2*>(V + size_t(c + u) * ld) + p);
#pragma unroll
				for (int u = 0; u < 8; ++u) {
					w.x += cs[c + u] * a[u].x;
					w.y += cs[c + u] * a[u].y;
				}
			}
			for (; c < ncols; ++c) {
				const double2 a = __ldg(reinterpret_cast<const double2*>(V + size_t(c) * ld) + p);
				w.x += cs[c] * a.x;
				w.y += cs[c] * a.y;
			}
			reinterpret_cast<double2*>(z)[p] = w;
		}
		if ((n & 1) && first == 0) {
			const size_t i = n - 1;
			double       w = 0.0;
			for (int c = 0; c < ncols; ++c)
				w += cs[c] * V[size_t(c) * ld + i];
			z[i] = w;
		}
	} else {
		for (size_t i = first; i < n; i += stride) {
			double w = 0.0;
			for (int c = 0; c < ncols; ++c)
				w += cs[c] * V[size_t(c) * ld + i];
			z[i] = w;
		}
	}
}

bool vec2_ok(const void* a, const void* b, size_t ld)
{
	return ld % 2 == 0 && (reinterpret_cast<uintptr_t>(a) & 15) == 0
	    && (reinterpret_cast<uintptr_t>(b) & 15) == 0;
}

// r[c] = <V[:,c], v>, c < ncols (two launches: partials, per-column sums)
void basis_dots(const double* V, size_t ld, int ncols, const double* v, size_t n, double* r,
                double* partial, cudaStream_t st)
{
	if (ncols <= 0)
		return;
	const int grid = int(std::max<size_t>(1, std::min<size_t>((n + kDotChunk - 1) / kDotChunk, kDotGrid)));
	if (vec2_ok(V, v, ld))
		k_basis_dots<true><<<grid, kThreads, 0, st>>>(V, ld, ncols, v, n, partial);
	else
		k_basis_dots<false><<<grid, kThreads, 0, st>>>(V, ld, ncols, v, n, partial);
	k_reduce_cols<<<ncols, kThreads, 0, st>>>(partial, grid, r);
}

// v -= V r, *nrm_out = |v|
void basis_subtract(double* v, const double* V, size_t ld, int ncols, const double* r, size_t n,
                    double* nrm_out, double* partial, unsigned* ctr, cudaStream_t st)
{
	const int grid = basis_blocks_for(n);
	if (vec2_ok(V, v, ld))
		k_basis_subtract<true><<<grid, kThreads, 0, st>>>(v, V, ld, ncols, r, n, nrm_out, partial, ctr);
	else
		k_basis_subtract<false><<<grid, kThreads, 0, st>>>(v, V, ld, ncols, r, n, nrm_out, partial, ctr);
}

// z = V coef
void basis_combine(double* z, const double* V, size_t ld, int ncols, const double* coef, size_t n,
                   cudaStream_t st)
{
	const int grid = basis_blocks_for(n);
	if (vec2_ok(V, z, ld))
		k_basis_combine<true><<<grid, kThreads, 0, st>>>(z, V, ld, ncols, coef, n);
	else
		k_basis_combine<false><<<grid, kThreads, 0, st>>>(z, V, ld, ncols, coef, n);
}

__global__ void __launch_bounds__(kThreads)
k_gather(const double* __restrict__ src, const long long* __restrict__ idx,
         double* __restrict__ dst, size_t n)
{
	for (size_t q = blockIdx.x * size_t(kThreads) + threadIdx.x; q < n;
	     q += size_t(gridDim.x) * kThreads)
		dst[q] = src[idx[q]];
}

__global__ void __launch_bounds__(kThreads)
k_scatter(const double* __restrict__ src, const long long* __restrict__ idx,
          double* __restrict__ dst, size_t n)
{
	for (size_t q = blockIdx.x * size_t(kThreads) + threadIdx.x; q < n;
	     q += size_t(gridDim.x) * kThreads)
		dst[idx[q]] = src[q];
}

} // namespace

// Device buffers of the eigensolver of one handle.
struct LanczosWork {
	size_t    dim     = 0;
	int       cols    = 0;       // columns of V
	double*   V       = nullptr; // dim x cols, column-major
	double*   scal    = nullptr; // alpha[cols], beta[cols+1], work[8]
	double*   partial = nullptr; // kMaxBlocks * kMaxCols
	double*   r       = nullptr; // projection coefficients / Ritz coefficients
	unsigned* ctr     = nullptr; // arrival counters (one per reduction kernel)
	double*   host    = nullptr; // pinned mirror of alpha/beta
	void*     step    = nullptr; // LanczosStep record of graph-replayed steps
};

void release_lanczos(dmrgpp_kron_handle h)
{
	LanczosWork* w = h->lanczos;
	if (!w)
		return;
	dmrgpp::dev_free(w->V);
	dmrgpp::dev_free(w->scal);
	dmrgpp::dev_free(w->partial);
	dmrgpp::dev_free(w->r);
	dmrgpp::dev_free(w->ctr);
	dmrgpp::dev_free(w->step);
	if (w->host)
		cudaFreeHost(w->host);
	delete w;
	h->lanczos = nullptr;
}

namespace {

int cuda_status(dmrgpp_kron_handle h, cudaError_t e, const char* where)
{
	return handle_fail(h, e == cudaErrorMemoryAllocation ? DMRGPP_OOM : DMRGPP_CUDA_ERROR,
	                   std::string(where) + ": " + cudaGetErrorString(e));
}

int ensure_work(dmrgpp_kron_handle h, size_t dim, int cols)
{
	LanczosWork* w = h->lanczos;
	if (w && w->dim == dim && w->cols >= cols)
		return DMRGPP_OK;
	release_lanczos(h);
	w           = new LanczosWork();
	h->lanczos  = w;
	w->dim      = dim;
	w->cols     = cols;
	cudaError_t e;
	if ((e = dmrgpp::dev_malloc(&w->V, dim * size_t(cols) * sizeof(double))))
		return cuda_status(h, e, "device allocation (Lanczos basis)");
	if ((e = dmrgpp::dev_malloc(&w->scal, (2 * size_t(cols) + 16) * sizeof(double))))
		return cuda_status(h, e, "device allocation (Lanczos scalars)");
	if ((e = dmrgpp::dev_malloc(&w->partial, size_t(kMaxBlocks) * kMaxCols * sizeof(double))))
		return cuda_status(h, e, "device allocation (partials)");
	if ((e = dmrgpp::dev_malloc(&w->r, size_t(kMaxCols) * sizeof(double))))
		return cuda_status(h, e, "device allocation (coefficients)");
	if ((e = dmrgpp::dev_malloc(&w->ctr, 16 * sizeof(unsigned))))
		return cuda_status(h, e, "device allocation (counters)");
	if ((e = dmrgpp::clear_async(w->ctr, 16 * sizeof(unsigned), h->stream)))
		return cuda_status(h, e, "clear counters");
	if ((e = dmrgpp::clear_async(w->scal, (2 * size_t(cols) + 16) * sizeof(double), h->stream)))
		return cuda_status(h, e, "clear scalars");
	if ((e = cudaHostAlloc(&w->host, 2 * (2 * size_t(cols) + 16) * sizeof(double), 0)))
		return cuda_status(h, e, "cudaHostAlloc(scalars)");
	if ((e = dmrgpp::dev_malloc(&w->step, sizeof(LanczosStep))))
		return cuda_status(h, e, "device allocation (step record)");
	return DMRGPP_OK;
}

} // namespace
} // namespace dmrgpp

using dmrgpp::LanczosWork;

extern "C" {

void dmrgpp_lanczos_params_init(dmrgpp_lanczos_params* p)
{
	if (!p)
		return;
	p->steps         = 200;   // ParametersForSolver.h:97 (LanczosSteps)
	p->min_steps     = 4;     // ParametersForSolver.h:102
	p->eigs_for_stop = 1;     // ParametersForSolver.h:105
	p->tolerance     = 1e-12; // ParametersForSolver.h:103
	p->reortho       = 1;     // Options=reortho
	p->check_every   = 8;
	p->use_graph     = 1;
	p->residual_gap_ratio = 0.0;
}

int dmrgpp_tridiag_eigen(size_t n, const double* diag, const double* offdiag, double* eigs,
                         double* vectors)
{
	if (n == 0)
		return DMRGPP_OK;
	if (!diag || !eigs || (n > 1 && !offdiag) || n > (1u << 20))
		return DMRGPP_INVALID_ARG;
	std::copy(diag, diag + n, eigs);
	return dmrgpp::tridiag_eigen(int(n), eigs, offdiag, vectors) ? DMRGPP_OK
	                                                            : DMRGPP_NOT_CONVERGED;
}

int dmrgpp_gather(const double* src, const int64_t* idx, double* dst, size_t n, void* stream)
{
	DMRGPP_TRACE("dmrgpp_gather");
	if (n == 0)
		return DMRGPP_OK;
	if (!src || !idx || !dst)
		return DMRGPP_INVALID_ARG;
	const int nb = dmrgpp::blocks_for(n);
	dmrgpp::k_gather<<<nb, dmrgpp::kThreads, 0, static_cast<cudaStream_t>(stream)>>>(
	    src, reinterpret_cast<const long long*>(idx), dst, n);
	return cudaGetLastError() == cudaSuccess ? DMRGPP_OK : DMRGPP_CUDA_ERROR;
}

int dmrgpp_scatter(const double* src, const int64_t* idx, double* dst, size_t n, void* stream)
{
	DMRGPP_TRACE("dmrgpp_scatter");
	if (n == 0)
		return DMRGPP_OK;
	if (!src || !idx || !dst)
		return DMRGPP_INVALID_ARG;
	const int nb = dmrgpp::blocks_for(n);
	dmrgpp::k_scatter<<<nb, dmrgpp::kThreads, 0, static_cast<cudaStream_t>(stream)>>>(
	    src, reinterpret_cast<const long long*>(idx), dst, n);
	return cudaGetLastError() == cudaSuccess ? DMRGPP_OK : DMRGPP_CUDA_ERROR;
}

int dmrgpp_lanczos_lowest(dmrgpp_kron_handle          h,
                          const dmrgpp_lanczos_params* p,
                          const double*               init,
                          int                         on_device,
                          double*                     energy,
                          double*                     z,
                          size_t*                     steps_taken)
{
	DMRGPP_TRACE("dmrgpp_lanczos_lowest");
	if (h && h->complex_sector)
		return dmrgpp::handle_fail(h, DMRGPP_NOT_SUPPORTED, "the device eigensolvers take real sectors");
	using namespace dmrgpp;
	if (!h)
		return DMRGPP_INVALID_ARG;
	if (!p || !init || !energy || !z)
		return handle_fail(h, DMRGPP_INVALID_ARG, "null argument");
	if (p->steps < 1 || p->check_every < 1 || p->eigs_for_stop < 1)
		return handle_fail(h, DMRGPP_INVALID_ARG, "steps, check_every and eigs_for_stop must be >= 1");
	const size_t D = size_t(h->plan.dim());
	size_t       maxn = std::min(p->steps, D); // LanczosCore.h:177-178
	if (maxn + 1 > size_t(kMaxCols))
		return handle_fail(h, DMRGPP_INVALID_ARG, "at most 1023 Lanczos steps");

	int prev = -1;
	cudaGetDevice(&prev);
	if (prev != h->device)
		cudaSetDevice(h->device);
	struct Restore {
		int dev, prev;
		~Restore()
		{
			if (dev != prev && prev >= 0)
				cudaSetDevice(prev);
		}
	} restore { h->device, prev };

	if (int rc = ensure_work(h, D, int(maxn) + 1))
		return rc;
	LanczosWork* w  = h->lanczos;
	cudaStream_t st = h->stream;
	const int    nb = blocks_for(D);
	double*      V  = w->V;
	double*      alpha = w->scal;
	double*      beta  = w->scal + w->cols;
	double*      work  = w->scal + 2 * size_t(w->cols); // [0] norm^2 of init, [1] reortho norm
	auto         col   = [&](size_t c) { return V + c * D; };
	cudaError_t  e;

	// V0 = init / |init|  (LanczosCore.h:166-175)
	if (!on_device) {
		if ((e = cudaMemcpyAsync(col(1), init, D * sizeof(double), cudaMemcpyHostToDevice, st)))
			return cuda_status(h, e, "copy initial vector");
	} else if ((e = cudaMemcpyAsync(col(1), init, D * sizeof(double), cudaMemcpyDeviceToDevice, st))) {
		return cuda_status(h, e, "copy initial vector");
	}
	k_dot<<<nb, kThreads, 0, st>>>(col(1), col(1), D, work, w->partial, w->ctr);
	k_scale_rsqrt<<<nb, kThreads, 0, st>>>(col(1), col(0), D, work);
	cudaMemsetAsync(beta, 0, sizeof(double), st); // beta_0 = 0

	// first step (LanczosCore.h:186-208)
	if (int rc = kron_apply_device(h, col(0), col(1)))
		return rc;
	k_dot<<<nb, kThreads, 0, st>>>(col(1), col(0), D, alpha, w->partial, w->ctr + 1);
	k_lanczos_update<<<nb, kThreads, 0, st>>>(col(1), col(0), nullptr, D, alpha, beta, beta + 1,
	                                          w->partial, w->ctr + 2);
	k_scale_inv<<<nb, kThreads, 0, st>>>(col(1), D, beta + 1);

	// graph-replayed steps: every kernel of a step reads its columns from the
	// step record, so one captured graph of check_every steps serves the
	// whole solve (same kernels and grids as the launches below: bitwise
	// identical results)
	LanczosStep* sp       = static_cast<LanczosStep*>(w->step);
	const bool   vec      = vec2_ok(V, V + D, D);
	const int    dgrid    = int(std::max<size_t>(1, std::min<size_t>((D + kDotChunk - 1) / kDotChunk, kDotGrid)));
	const int    sgrid    = basis_blocks_for(D);
	const bool   use_graph = p->use_graph != 0;
	auto         enqueue_step = [&](cudaStream_t s) -> int {
		k_step_advance<<<1, 1, 0, s>>>(sp, V, D, alpha, beta);
		if (int rc = kron_apply_device(h, nullptr, nullptr, &sp->io))
			return rc;
		k_dot_step<<<nb, kThreads, 0, s>>>(sp, D, w->partial, w->ctr + 1);
		k_update_step<<<nb, kThreads, 0, s>>>(sp, D, w->partial, w->ctr + 2);
		k_scale_inv_step<<<nb, kThreads, 0, s>>>(sp, D, nullptr);
		if (p->reortho) {
			if (vec) {
				k_basis_dots_step<true><<<dgrid, kThreads, 0, s>>>(sp, V, D, D, w->partial);
			} else {
				k_basis_dots_step<false><<<dgrid, kThreads, 0, s>>>(sp, V, D, D, w->partial);
			}
			k_reduce_cols_step<<<w->cols, kThreads, 0, s>>>(sp, w->partial, dgrid, w->r);
			if (vec) {
				k_basis_subtract_step<true><<<sgrid, kThreads, 0, s>>>(sp, V, D, w->r, D, work + 1,
				                                                      w->partial, w->ctr + 4);
			} else {
				k_basis_subtract_step<false><<<sgrid, kThreads, 0, s>>>(sp, V, D, w->r, D, work + 1,
				                                                       w->partial, w->ctr + 4);
			}
			k_scale_inv_step<<<nb, kThreads, 0, s>>>(sp, D, work + 1);
		}
		return DMRGPP_OK;
	};
	struct Graph {
		cudaGraph_t     g = nullptr;
		cudaGraphExec_t x = nullptr;
		~Graph()
		{
			if (x)
				cudaGraphExecDestroy(x);
			if (g)
				cudaGraphDestroy(g);
		}
	} graph;
	// capture check_every steps on a private stream (the handle's stream may
	// be the legacy default stream, which cannot be captured)
	auto capture = [&]() -> int {
		cudaStream_t cs = nullptr;
		if ((e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking)))
			return cuda_status(h, e, "capture stream");
		const cudaStream_t saved = h->stream;
		h->stream                = cs;
		int rc                   = DMRGPP_OK;
		e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
		if (e == cudaSuccess) {
			for (int q = 0; q < p->check_every && rc == DMRGPP_OK; ++q)
				rc = enqueue_step(cs);
			const cudaError_t e2 = cudaStreamEndCapture(cs, &graph.g);
			if (rc == DMRGPP_OK && e2 != cudaSuccess)
				rc = cuda_status(h, e2, "end of graph capture");
		} else {
			rc = cuda_status(h, e, "graph capture");
		}
		h->stream = saved;
		cudaStreamDestroy(cs);
		if (rc == DMRGPP_OK && (e = cudaGraphInstantiate(&graph.x, graph.g, 0)))
			rc = cuda_status(h, e, "graph instantiation");
		return rc;
	};
	if (use_graph)
		k_step_set<<<1, 1, 0, st>>>(sp, 0); // the first step is j = 1

	// Groups of check_every steps are enqueued one group ahead of the host's
	// stopping test (two pinned copies of alpha/beta alternate), so the GPU
	// runs the next group while the host tests the last one; steps past the
	// stopping point are discarded, as in the one-group-at-a-time form.
	auto enqueue_group = [&](size_t j0, size_t j1) -> int {
		if (use_graph) {
			if (j1 - j0 == size_t(p->check_every)) {
				if (!graph.x)
					if (int rc = capture())
						return rc;
				if ((e = cudaGraphLaunch(graph.x, st)))
					return cuda_status(h, e, "graph launch");
			} else {
				for (size_t jj = j0; jj < j1; ++jj)
					if (int rc = enqueue_step(st))
						return rc;
			}
			return DMRGPP_OK;
		}
		for (size_t jj = j0; jj < j1; ++jj) {
			// oneStepDecomposition (LanczosVectors.h:203-241), V2 lives in column jj+1
			double* v0 = col(jj - 1);
			double* v1 = col(jj);
			double* v2 = col(jj + 1);
			if (int rc = kron_apply_device(h, v1, v2))
				return rc;
			k_dot<<<nb, kThreads, 0, st>>>(v2, v1, D, alpha + jj, w->partial, w->ctr + 1);
			k_lanczos_update<<<nb, kThreads, 0, st>>>(v2, v1, v0, D, alpha + jj, beta + jj,
			                                          beta + jj + 1, w->partial, w->ctr + 2);
			k_scale_inv<<<nb, kThreads, 0, st>>>(v2, D, beta + jj + 1);
			if (p->reortho) { // reorthoIfNecessary (LanczosVectors.h:243-271)
				const int nc = int(jj) + 1;
				basis_dots(V, D, nc, v2, D, w->r, w->partial, st);
				basis_subtract(v2, V, D, nc, w->r, D, work + 1, w->partial, w->ctr + 4, st);
				k_scale_inv<<<nb, kThreads, 0, st>>>(v2, D, work + 1);
			}
		}
		return DMRGPP_OK;
	};
	struct Events {
		cudaEvent_t ev[2] = { nullptr, nullptr };
		~Events()
		{
			for (cudaEvent_t x : ev)
				if (x)
					cudaEventDestroy(x);
		}
	} events;
	for (int b = 0; b < 2; ++b)
		if ((e = cudaEventCreateWithFlags(&events.ev[b], cudaEventDisableTiming)))
			return cuda_status(h, e, "events");
	const size_t host_stride = 2 * size_t(w->cols) + 16;
	struct Group {
		size_t j0, j1;
		int    buf;
	};
	std::vector<Group> inflight;
	std::vector<double> eold(p->eigs_for_stop, 0.0), dd, ee, rz;
	size_t              j_stop = 0;
	bool                done   = false;
	size_t              next   = 1;
	int                 buf    = 0;
	const double*       hb     = w->host; // alpha/beta of the last tested group
	while (!done) {
		while (inflight.size() < 2 && next < maxn) {
			const size_t jend = std::min(maxn, next + size_t(p->check_every));
			if (int rc = enqueue_group(next, jend))
				return rc;
			if ((e = cudaGetLastError()))
				return cuda_status(h, e, "Lanczos step launch");
			// alpha[0..jend) and beta[0..jend] back to the host
			double* hbuf = w->host + size_t(buf) * host_stride;
			if ((e = cudaMemcpyAsync(hbuf, w->scal, 2 * size_t(w->cols) * sizeof(double),
			                         cudaMemcpyDeviceToHost, st))
			    || (e = cudaEventRecord(events.ev[buf], st)))
				return cuda_status(h, e, "read alpha/beta");
			inflight.push_back({ next, jend, buf });
			next = jend;
			buf ^= 1;
		}
		if (inflight.empty())
			break;
		const Group g = inflight.front();
		inflight.erase(inflight.begin());
		if ((e = cudaEventSynchronize(events.ev[g.buf])))
			return cuda_status(h, e, "Lanczos steps");
		if (h->err_host && *reinterpret_cast<volatile int*>(h->err_host))
			return handle_fail(h, DMRGPP_TIMEOUT, "H*x kernel wait gave up during Lanczos");
		hb               = w->host + size_t(g.buf) * host_stride;
		const double* ah = hb;
		const double* bh = hb + w->cols;
		// stopping test per step, in order (LanczosCore.h:215-240); the
		// lowest Ritz values by Sturm bisection of the step's tridiagonal
		for (size_t jj = g.j0; jj < g.j1; ++jj) {
			const size_t n = jj + 1;
			dd.assign(ah, ah + n);
			ee.assign(bh + 1, bh + n);
			const size_t ne   = std::min(p->eigs_for_stop, n);
			double       dmax = 0.0;
			for (size_t k = 0; k < ne; ++k) {
				const double th = tridiag_kth_lowest(int(n), dd.data(), ee.data(), int(k) + 1);
				dmax            = std::max(dmax, std::fabs(th - eold[k]));
				eold[k]         = th;
			}
			bool exit_flag = dmax < p->tolerance || jj == maxn - 1;
			if (!exit_flag && p->residual_gap_ratio > 0.0 && n >= 2) {
				// residual of the lowest Ritz pair: beta_{j+1} |last component|
				const double th2 = tridiag_kth_lowest(int(n), dd.data(), ee.data(), 2);
				rz.resize(n);
				tridiag_inverse_iteration(int(n), dd.data(), ee.data(), eold[0], rz.data());
				const double res = std::fabs(bh[n]) * std::fabs(rz[n - 1]);
				exit_flag        = res <= p->residual_gap_ratio * (th2 - eold[0]);
			}
			if ((exit_flag && D <= 4) || (exit_flag && jj >= p->min_steps)) {
				j_stop = jj;
				done   = true;
				break;
			}
		}
	}
	if (!done)
		j_stop = maxn - 1;
	if (maxn == 1)
		j_stop = 0;

	// Ritz vector of the (j_stop+1)-dimensional tridiagonal (LanczosSolver.h:76-84):
	// the lowest of the QL eigenvalues and its eigenvector (by inverse
	// iteration, O(n), unless the next eigenvalue coincides with it)
	const size_t        n = j_stop + 1;
	std::vector<double> d(hb, hb + n), off(hb + w->cols + 1, hb + w->cols + n), zt(n);
	if (maxn == 1) { // no loop ran: alpha[0] has not been read back yet
		if ((e = dmrgpp::download_sync(w->host, w->scal, sizeof(double), h->stream)))
			return cuda_status(h, e, "read alpha");
		d[0] = w->host[0];
	}
	if (!tridiag_lowest(int(n), d.data(), off.data(), energy, zt.data()))
		return handle_fail(h, DMRGPP_NOT_CONVERGED, "tridiagonal eigensolve failed");
	if ((e = cudaMemcpyAsync(w->r, zt.data(), n * sizeof(double), cudaMemcpyHostToDevice, st)))
		return cuda_status(h, e, "upload Ritz coefficients");
	double* zdst = on_device ? z : col(j_stop + 1); // that column is free after the solve
	basis_combine(zdst, V, D, int(n), w->r, D, st);
	if (!on_device
	    && (e = cudaMemcpyAsync(z, zdst, D * sizeof(double), cudaMemcpyDeviceToHost, st)))
		return cuda_status(h, e, "copy Ritz vector");
	if ((e = cudaStreamSynchronize(st)))
		return cuda_status(h, e, "Ritz vector");
	if (steps_taken)
		*steps_taken = j_stop;
	return DMRGPP_OK;
}

} // extern "C"

// ---------------------------------------------------------------------------
// Davidson for the lowest eigenpair (no counterpart in the reference, which
// only has Lanczos): the correction of each step comes from a preconditioner
// applied to the residual -- none, the diagonal (Jacobi) one, or the learned
// MLP of mlp.cu -- and the search space is orthonormalised on the device.
// With a mixed-precision handle the first phase runs every matvec in the
// handle's mixed mode and the second restarts from its Ritz vector in FP64,
// so the energy and residual that are reported are FP64 quantities.
// ---------------------------------------------------------------------------
#include "mlp.h"

namespace dmrgpp {

namespace {

// r = hu - theta*u, *nrm = |r|
__global__ void __launch_bounds__(kThreads)
k_residual(const double* __restrict__ hu, const double* __restrict__ u, double theta,
           double* __restrict__ r, size_t n, double* nrm, double* partial, unsigned* ctr)
{
	__shared__ double red[kThreads / 32];
	double            s = 0.0;
	for (size_t i = blockIdx.x * size_t(kThreads) + threadIdx.x; i < n;
	     i += size_t(gridDim.x) * kThreads) {
		const double w = hu[i] - theta * u[i];
		r[i]           = w;
		s += w * w;
	}
	s = block_sum(s, red);
	grid_sum(s, partial, ctr, nrm, true, red);
}

// diagonal (Jacobi) correction: t = r / (theta - d), denominators kept away
// from zero
__global__ void __launch_bounds__(kThreads)
k_jacobi(const double* __restrict__ r, const double* __restrict__ d, double theta, double floor_,
         double* __restrict__ t, size_t n)
{
	for (size_t i = blockIdx.x * size_t(kThreads) + threadIdx.x; i < n;
	     i += size_t(gridDim.x) * kThreads) {
		double den = theta - d[i];
		if (fabs(den) < floor_)
			den = den < 0 ? -floor_ : floor_;
		t[i] = r[i] / den;
	}
}

__global__ void __launch_bounds__(kThreads)
k_copy(const double* __restrict__ src, double* __restrict__ dst, size_t n)
{
	for (size_t i = blockIdx.x * size_t(kThreads) + threadIdx.x; i < n;
	     i += size_t(gridDim.x) * kThreads)
		dst[i] = src[i];
}

} // namespace

struct DavidsonWork {
	size_t    dim     = 0;
	int       mmax    = 0;
	double*   V       = nullptr; // dim x mmax, orthonormal basis
	double*   W       = nullptr; // dim x mmax, H V
	double*   u       = nullptr; // Ritz vector, H u, residual, correction
	double*   hu      = nullptr;
	double*   r       = nullptr;
	double*   t       = nullptr;
	double*   coef    = nullptr; // kMaxCols
	double*   scal    = nullptr; // scalars written by reductions
	double*   partial = nullptr;
	unsigned* ctr     = nullptr;
	double*   host    = nullptr; // pinned, kMaxCols + 8
};

void release_davidson(dmrgpp_kron_handle h)
{
	DavidsonWork* w = h->davidson;
	if (!w)
		return;
	dmrgpp::dev_free(w->V);
	dmrgpp::dev_free(w->W);
	dmrgpp::dev_free(w->u);
	dmrgpp::dev_free(w->coef);
	dmrgpp::dev_free(w->scal);
	dmrgpp::dev_free(w->partial);
	dmrgpp::dev_free(w->ctr);
	if (w->host)
		cudaFreeHost(w->host);
	delete w;
	h->davidson = nullptr;
}

namespace {

int ensure_davidson(dmrgpp_kron_handle h, size_t dim, int mmax)
{
	DavidsonWork* w = h->davidson;
	if (w && w->dim == dim && w->mmax >= mmax)
		return DMRGPP_OK;
	release_davidson(h);
	w           = new DavidsonWork();
	h->davidson = w;
	w->dim      = dim;
	w->mmax     = mmax;
	cudaError_t e;
	if ((e = dmrgpp::dev_malloc(&w->V, dim * size_t(mmax) * sizeof(double)))
	    || (e = dmrgpp::dev_malloc(&w->W, dim * size_t(mmax) * sizeof(double)))
	    || (e = dmrgpp::dev_malloc(&w->u, 4 * dim * sizeof(double)))
	    || (e = dmrgpp::dev_malloc(&w->coef, size_t(kMaxCols) * sizeof(double)))
	    || (e = dmrgpp::dev_malloc(&w->scal, 16 * sizeof(double)))
	    || (e = dmrgpp::dev_malloc(&w->partial, size_t(kMaxBlocks) * kMaxCols * sizeof(double)))
	    || (e = dmrgpp::dev_malloc(&w->ctr, 16 * sizeof(unsigned)))
	    || (e = dmrgpp::clear_async(w->ctr, 16 * sizeof(unsigned), h->stream))
	    || (e = cudaHostAlloc(&w->host, (size_t(kMaxCols) + 8) * sizeof(double), 0)))
		return cuda_status(h, e, "Davidson buffers");
	w->hu = w->u + dim;
	w->r  = w->u + 2 * dim;
	w->t  = w->u + 3 * dim;
	return DMRGPP_OK;
}

} // namespace
} // namespace dmrgpp

extern "C" {

void dmrgpp_davidson_params_init(dmrgpp_davidson_params* p)
{
	if (!p)
		return;
	p->max_iterations  = 500;
	p->max_subspace    = 32;
	p->tolerance       = 1e-8;
	p->preconditioner  = DMRGPP_PRECOND_JACOBI;
	p->mlp             = nullptr;
	p->mixed_tolerance = 1e-4;
	p->denominator_floor = 1e-3;
}

int dmrgpp_davidson_lowest(dmrgpp_kron_handle            h,
                           const dmrgpp_davidson_params* p,
                           const double*                 init,
                           int                           on_device,
                           double*                       energy,
                           double*                       z,
                           dmrgpp_davidson_stats*        stats)
{
	DMRGPP_TRACE("dmrgpp_davidson_lowest");
	if (h && h->complex_sector)
		return dmrgpp::handle_fail(h, DMRGPP_NOT_SUPPORTED, "the device eigensolvers take real sectors");
	using namespace dmrgpp;
	if (!h)
		return DMRGPP_INVALID_ARG;
	if (!p || !init || !energy || !z)
		return handle_fail(h, DMRGPP_INVALID_ARG, "null argument");
	if (p->max_subspace < 2 || p->max_subspace > 512 || p->max_iterations < 1)
		return handle_fail(h, DMRGPP_INVALID_ARG, "max_subspace must be in [2, 512]");
	if (p->preconditioner == DMRGPP_PRECOND_MLP && !p->mlp)
		return handle_fail(h, DMRGPP_INVALID_ARG, "learned preconditioner selected without a network");
	const size_t D = size_t(h->plan.dim());
	int          prev = -1;
	cudaGetDevice(&prev);
	if (prev != h->device)
		cudaSetDevice(h->device);
	struct Restore {
		int dev, prev;
		~Restore()
		{
			if (dev != prev && prev >= 0)
				cudaSetDevice(prev);
		}
	} restore { h->device, prev };

	const int mmax = int(p->max_subspace);
	if (int rc = ensure_davidson(h, D, mmax))
		return rc;
	DavidsonWork* w   = h->davidson;
	cudaStream_t  st  = h->stream;
	const int     nb  = blocks_for(D);
	cudaError_t   e;
	auto          Vc  = [&](int c) { return w->V + size_t(c) * D; };
	auto          Wc  = [&](int c) { return w->W + size_t(c) * D; };

	// two phases when the handle computes in a mixed mode
	const int user_precision = h->precision;
	int       phase          = user_precision == DMRGPP_FP64 ? 1 : 0;
	dmrgpp_davidson_stats s {};

	if ((e = cudaMemcpyAsync(w->t, init, D * sizeof(double),
	                         on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st)))
		return cuda_status(h, e, "copy initial vector");

	const size_t        mm = static_cast<size_t>(mmax);
	std::vector<double> G(mm * mm, 0.0), ev(mm, 0.0), evec(mm * mm, 0.0);
	int    k       = 0;
	double theta   = 0.0, rnorm = 0.0;
	double best_mixed = 1e300;
	int    stall   = 0;
	bool   converged = false;
	auto   set_phase = [&](int ph) {
                phase        = ph;
                h->precision = (ph == 0) ? user_precision : DMRGPP_FP64;
	};
	set_phase(phase);
	int rc = DMRGPP_OK;

	for (size_t it = 0; it < p->max_iterations; ++it) {
		// orthonormalise the correction against the basis (two classical
		// Gram-Schmidt passes) and append it
		for (int pass = 0; pass < (k > 0 ? 2 : 0); ++pass) {
			basis_dots(w->V, D, k, w->t, D, w->coef, w->partial, st);
			basis_subtract(w->t, w->V, D, k, w->coef, D, w->scal + 0, w->partial, w->ctr + 1, st);
		}
		k_dot<<<nb, kThreads, 0, st>>>(w->t, w->t, D, w->scal + 1, w->partial, w->ctr + 2);
		k_scale_rsqrt<<<nb, kThreads, 0, st>>>(w->t, Vc(k), D, w->scal + 1);
		if ((rc = kron_apply_device(h, Vc(k), Wc(k))))
			break;
		if (phase == 0)
			++s.mixed_matvecs;
		else
			++s.fp64_matvecs;
		// new column of the projected matrix G = V^T H V
		basis_dots(w->V, D, k + 1, Wc(k), D, w->coef, w->partial, st);
		if ((e = cudaMemcpyAsync(w->host, w->coef, size_t(k + 1) * sizeof(double),
		                         cudaMemcpyDeviceToHost, st))
		    || (e = cudaStreamSynchronize(st))) {
			rc = cuda_status(h, e, "Davidson projection");
			break;
		}
		if (h->err_host && *reinterpret_cast<volatile int*>(h->err_host)) {
			rc = handle_fail(h, DMRGPP_TIMEOUT, "H*x kernel wait gave up during Davidson");
			break;
		}
		for (int i = 0; i <= k; ++i) {
			G[size_t(i) + size_t(k) * mmax] = w->host[i];
			G[size_t(k) + size_t(i) * mmax] = w->host[i];
		}
		++k;
		// Rayleigh-Ritz on the k-dimensional space
		std::vector<double> Gk(size_t(k) * size_t(k));
		for (int j = 0; j < k; ++j)
			for (int i = 0; i < k; ++i)
				Gk[size_t(i) + size_t(j) * k] = G[size_t(i) + size_t(j) * mmax];
		sym_eigen(k, Gk.data(), ev.data(), evec.data());
		theta = ev[0];
		if ((e = cudaMemcpyAsync(w->coef, evec.data(), size_t(k) * sizeof(double),
		                         cudaMemcpyHostToDevice, st))) {
			rc = cuda_status(h, e, "Ritz coefficients");
			break;
		}
		basis_combine(w->u, w->V, D, k, w->coef, D, st);
		basis_combine(w->hu, w->W, D, k, w->coef, D, st);
		k_residual<<<nb, kThreads, 0, st>>>(w->hu, w->u, theta, w->r, D, w->scal + 2, w->partial,
		                                    w->ctr + 4);
		if ((e = cudaMemcpyAsync(w->host, w->scal + 2, sizeof(double), cudaMemcpyDeviceToHost, st))
		    || (e = cudaStreamSynchronize(st))) {
			rc = cuda_status(h, e, "Davidson residual");
			break;
		}
		rnorm = w->host[0];
		++s.iterations;
		const double scale = std::max(1.0, std::fabs(theta));
		if (phase == 1 && rnorm <= p->tolerance * scale) {
			converged = true;
			break;
		}
		bool restart = (k == mmax);
		if (phase == 0) {
			// leave the mixed phase once its residual is small or stalls
			if (rnorm < 0.9 * best_mixed) {
				best_mixed = rnorm;
				stall      = 0;
			} else {
				++stall;
			}
			if (rnorm <= p->mixed_tolerance * scale || stall >= 8) {
				set_phase(1);
				restart = true; // the FP64 phase starts from the Ritz vector alone
			}
		}
		if (restart) {
			// V = [u], W = [H u] (recomputed in FP64 on the phase change)
			k_copy<<<nb, kThreads, 0, st>>>(w->u, w->t, D);
			k = 0;
			if (phase == 1 && s.fp64_matvecs == 0) {
				++s.restarts;
				continue; // t = u is orthonormalised and multiplied in the next pass
			}
			k_dot<<<nb, kThreads, 0, st>>>(w->u, w->u, D, w->scal + 1, w->partial, w->ctr + 2);
			k_scale_rsqrt<<<nb, kThreads, 0, st>>>(w->u, Vc(0), D, w->scal + 1);
			k_scale_rsqrt<<<nb, kThreads, 0, st>>>(w->hu, Wc(0), D, w->scal + 1);
			G[0] = theta;
			k    = 1;
			++s.restarts;
		}
		// correction from the preconditioner
		if (p->preconditioner == DMRGPP_PRECOND_JACOBI) {
			k_jacobi<<<nb, kThreads, 0, st>>>(w->r, h->d_diag, theta,
			                                  p->denominator_floor * std::max(1.0, std::fabs(theta)),
			                                  w->t, D);
		} else if (p->preconditioner == DMRGPP_PRECOND_MLP) {
			if ((rc = mlp_precondition(static_cast<dmrgpp_mlp_handle>(p->mlp), h->d_diag, w->r,
			                           theta, rnorm, w->t, D, st))) {
				handle_fail(h, rc, "learned preconditioner failed");
				break;
			}
		} else {
			k_copy<<<nb, kThreads, 0, st>>>(w->r, w->t, D);
		}
		if ((e = cudaGetLastError())) {
			rc = cuda_status(h, e, "Davidson launch");
			break;
		}
	}
	h->precision = user_precision;
	if (rc)
		return rc;
	s.residual_norm = rnorm;
	s.converged     = converged ? 1 : 0;
	// the Ritz vector u is normalised by construction (V orthonormal, |s| = 1)
	if ((e = cudaMemcpyAsync(z, w->u, D * sizeof(double),
	                         on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st))
	    || (e = cudaStreamSynchronize(st)))
		return cuda_status(h, e, "copy Ritz vector");
	*energy = theta;
	if (stats)
		*stats = s;
	return converged ? DMRGPP_OK : handle_fail(h, DMRGPP_NOT_CONVERGED, "Davidson did not converge");
}

} // extern "C"

namespace dmrgpp {
namespace {

// y += a x
__global__ void __launch_bounds__(kThreads)
k_axpy(double a, const double* __restrict__ x, double* __restrict__ y, size_t n)
{
	for (size_t i = blockIdx.x * size_t(kThreads) + threadIdx.x; i < n;
	     i += size_t(gridDim.x) * kThreads)
		y[i] += a * x[i];
}

// y -= (*a) x  (scalar from a reduction kernel)
__global__ void __launch_bounds__(kThreads)
k_axpy_neg_dev(const double* a, const double* __restrict__ x, double* __restrict__ y, size_t n)
{
	const double c = *a;
	for (size_t i = blockIdx.x * size_t(kThreads) + threadIdx.x; i < n;
	     i += size_t(gridDim.x) * kThreads)
		y[i] -= c * x[i];
}

// conjugate-gradient update with device scalars: alpha = rr / pAp;
// t += alpha p; res -= alpha Aq; *rr_next = |res|^2.  A non-positive pAp (or
// an earlier one, *broken) freezes the iteration: alpha = 0 and *broken = 1.
__global__ void __launch_bounds__(kThreads)
k_cg_update(double* __restrict__ t, double* __restrict__ res, const double* __restrict__ p,
            const double* __restrict__ Aq, const double* rr, const double* pAp, double* rr_next,
            double* broken, size_t n, double* partial, unsigned* ctr)
{
	__shared__ double red[kThreads / 32];
	const bool        stop  = *broken != 0.0 || !(*pAp > 0.0);
	const double      alpha = stop ? 0.0 : *rr / *pAp;
	if (stop && blockIdx.x == 0 && threadIdx.x == 0)
		*broken = 1.0;
	double s = 0.0;
	for (size_t i = blockIdx.x * size_t(kThreads) + threadIdx.x; i < n;
	     i += size_t(gridDim.x) * kThreads) {
		t[i] += alpha * p[i];
		const double w = res[i] - alpha * Aq[i];
		res[i]         = w;
		s += w * w;
	}
	s = block_sum(s, red);
	grid_sum(s, partial, ctr, rr_next, false, red);
}

// p = res + (rr_next / rr) p, skipped once the iteration is frozen
__global__ void __launch_bounds__(kThreads)
k_cg_direction(double* __restrict__ p, const double* __restrict__ res, const double* rr_next,
               const double* rr, const double* broken, size_t n)
{
	if (*broken != 0.0)
		return;
	const double beta = *rr > 0.0 ? *rr_next / *rr : 0.0;
	for (size_t i = blockIdx.x * size_t(kThreads) + threadIdx.x; i < n;
	     i += size_t(gridDim.x) * kThreads)
		p[i] = res[i] + beta * p[i];
}

// --- diagonal (Jacobi) preconditioner of the projected correction equation
// P (H - theta) P t = -P r on the complement of u:  K = diag(H) - theta, kept
// at least `floor`; the preconditioned direction z = K^-1 res - a K^-1 u with
// a = <u, K^-1 res> / <u, K^-1 u> stays orthogonal to u (the projected
// preconditioner P K P of Jacobi-Davidson).  wv = K^-1 u.
__device__ __forceinline__ double pcg_k(double d, double theta, double floor_)
{
	const double k = d - theta;
	return k > floor_ ? k : floor_;
}

// wv = K^-1 u, *uw = <u, wv>
__global__ void __launch_bounds__(kThreads)
k_pcg_setup(const double* __restrict__ u, const double* __restrict__ diag, double theta, double floor_,
            double* __restrict__ wv, size_t n, double* uw, double* partial, unsigned* ctr)
{
	__shared__ double red[kThreads / 32];
	double            s = 0.0;
	for (size_t i = blockIdx.x * size_t(kThreads) + threadIdx.x; i < n;
	     i += size_t(gridDim.x) * kThreads) {
		const double v = u[i] / pcg_k(diag[i], theta, floor_);
		wv[i]          = v;
		s += u[i] * v;
	}
	s = block_sum(s, red);
	grid_sum(s, partial, ctr, uw, false, red);
}

// four sums at once (deterministic: per-block partials in 4 strided slots,
// the last block adds them in block order): sums[0..3]
__device__ __forceinline__ void grid_sum4(double (&v)[4], double* partial, unsigned* ctr, double* sums,
                                          double* red)
{
	__shared__ bool last;
	double          b[4];
#pragma unroll
	for (int q = 0; q < 4; ++q)
		b[q] = block_sum(v[q], red);
	if (threadIdx.x == 0) {
#pragma unroll
		for (int q = 0; q < 4; ++q)
			partial[size_t(q) * gridDim.x + blockIdx.x] = b[q];
		last = last_block(ctr);
	}
	__syncthreads();
	if (!last)
		return;
#pragma unroll
	for (int q = 0; q < 4; ++q) {
		double t = 0.0;
		for (int k = threadIdx.x; k < int(gridDim.x); k += blockDim.x)
			t += __ldcg(partial + size_t(q) * gridDim.x + k);
		t = block_sum(t, red);
		if (threadIdx.x == 0)
			sums[q] = t;
	}
}

// sums = <u, K^-1 res>, <res, K^-1 res>, <res, wv>, <res, res>
__device__ __forceinline__ void pcg_sums_body(const double* __restrict__ res, const double* __restrict__ diag,
                                              double theta, double floor_, const double* __restrict__ u,
                                              const double* __restrict__ wv, size_t n, double* sums,
                                              double* partial, unsigned* ctr, double* red)
{
	double v[4] = { 0.0, 0.0, 0.0, 0.0 };
	for (size_t i = blockIdx.x * size_t(kThreads) + threadIdx.x; i < n;
	     i += size_t(gridDim.x) * kThreads) {
		const double r = res[i];
		const double z = r / pcg_k(diag[i], theta, floor_);
		v[0] += u[i] * z;
		v[1] += r * z;
		v[2] += r * wv[i];
		v[3] += r * r;
	}
	grid_sum4(v, partial, ctr, sums, red);
}

__global__ void __launch_bounds__(kThreads)
k_pcg_sums(const double* __restrict__ res, const double* __restrict__ diag, double theta, double floor_,
           const double* __restrict__ u, const double* __restrict__ wv, size_t n, double* sums,
           double* partial, unsigned* ctr)
{
	__shared__ double red[kThreads / 32];
	pcg_sums_body(res, diag, theta, floor_, u, wv, n, sums, partial, ctr, red);
}

// alpha = rho / pAp; t += alpha p; res -= alpha Aq; then the four sums of the
// new res.  A non-positive pAp (or an earlier one, *broken) freezes the
// iteration: alpha = 0 and *broken = 1.
__global__ void __launch_bounds__(kThreads)
k_pcg_update(double* __restrict__ t, double* __restrict__ res, const double* __restrict__ p,
             const double* __restrict__ Aq, const double* rho, const double* pAp, double* broken,
             const double* __restrict__ diag, double theta, double floor_, const double* __restrict__ u,
             const double* __restrict__ wv, size_t n, double* sums, double* partial, unsigned* ctr)
{
	__shared__ double red[kThreads / 32];
	const bool        stop  = *broken != 0.0 || !(*pAp > 0.0);
	const double      alpha = stop ? 0.0 : *rho / *pAp;
	if (stop && blockIdx.x == 0 && threadIdx.x == 0)
		*broken = 1.0;
	for (size_t i = blockIdx.x * size_t(kThreads) + threadIdx.x; i < n;
	     i += size_t(gridDim.x) * kThreads) {
		t[i] += alpha * p[i];
		res[i] -= alpha * Aq[i];
	}
	// each thread re-reads only the elements it wrote: no grid barrier needed
	pcg_sums_body(res, diag, theta, floor_, u, wv, n, sums, partial, ctr, red);
}

// z = K^-1 res - a wv with a = sums[0] / *uw; rho_new = sums[1] - a sums[2];
// p = z + (rho_new / *rho) p (p = z when first); *rho_next = rho_new.
// Skipped once the iteration is frozen.
__global__ void __launch_bounds__(kThreads)
k_pcg_direction(double* __restrict__ p, const double* __restrict__ res, const double* __restrict__ diag,
                double theta, double floor_, const double* __restrict__ wv, const double* uw,
                const double* sums, const double* rho, double* rho_next, const double* broken, int first,
                size_t n)
{
	if (*broken != 0.0)
		return;
	const double a       = *uw > 0.0 ? sums[0] / *uw : 0.0;
	const double rho_new = sums[1] - a * sums[2];
	const double beta    = first ? 0.0 : (*rho > 0.0 ? rho_new / *rho : 0.0);
	if (blockIdx.x == 0 && threadIdx.x == 0)
		*rho_next = rho_new;
	for (size_t i = blockIdx.x * size_t(kThreads) + threadIdx.x; i < n;
	     i += size_t(gridDim.x) * kThreads) {
		const double z = res[i] / pcg_k(diag[i], theta, floor_) - a * wv[i];
		p[i]           = z + beta * p[i];
	}
}

} // namespace
} // namespace dmrgpp

namespace dmrgpp {
namespace {

// The correction equation by conjugate gradients with the projected
// diagonal preconditioner (see k_pcg_setup); res (= -P r on entry, as the
// caller set it) and the Davidson buffers as in dmrgpp_correction_solve;
// the preconditioner's K^-1 u lives in the Davidson work's free column t.
int pcg_correction(dmrgpp_kron_handle h, const double* u, double theta, const double* r, double* t,
                   int max_iterations, double rel_tolerance, int* iterations, double* rel_residual)
{
	(void)r;
	const size_t  D  = size_t(h->plan.dim());
	DavidsonWork* w  = h->davidson;
	cudaStream_t  st = h->stream;
	const int     nb = blocks_for(D);
	double*       res = w->hu;
	double*       p   = w->r;
	double*       Aq  = w->V + D;
	double*       wv  = w->t;
	double*       sc  = w->scal; // [0] u.v [1] pAp [4] frozen [5] uw [6..9] sums [10,11] rho
	const double  floor_ = 1e-3 * std::max(1.0, std::fabs(theta));
	auto read = [&](double* dev, int count, double* host) {
		return cudaMemcpyAsync(host, dev, size_t(count) * sizeof(double), cudaMemcpyDeviceToHost, st)
		        == cudaSuccess
		    && cudaStreamSynchronize(st) == cudaSuccess;
	};
	k_pcg_setup<<<nb, kThreads, 0, st>>>(u, h->d_diag, theta, floor_, wv, D, sc + 5, w->partial, w->ctr + 8);
	k_pcg_sums<<<nb, kThreads, 0, st>>>(res, h->d_diag, theta, floor_, u, wv, D, sc + 6, w->partial, w->ctr + 9);
	k_pcg_direction<<<nb, kThreads, 0, st>>>(p, res, h->d_diag, theta, floor_, wv, sc + 5, sc + 6, sc + 10,
	                                         sc + 10, sc + 4, 1, D);
	double host[4] = { 0, 0, 0, 0 };
	if (!read(sc + 9, 1, host))
		return handle_fail(h, DMRGPP_CUDA_ERROR, "correction solve");
	const double b0  = std::sqrt(host[0]);
	double       rrh = host[0];
	int          it  = 0;
	int          cur = 0; // rho of the current direction lives in sc[10 + cur]
	cudaError_t  e;
	while (it < max_iterations && b0 > 0 && std::sqrt(rrh) > rel_tolerance * b0) {
		const int burst = std::min(8, max_iterations - it);
		for (int q = 0; q < burst; ++q, ++it) {
			// Aq = P (H - theta) p  (p orthogonal to u up to round-off)
			if (int rc = kron_apply_device(h, p, Aq))
				return rc;
			k_axpy<<<nb, kThreads, 0, st>>>(-theta, p, Aq, D);
			k_dot<<<nb, kThreads, 0, st>>>(u, Aq, D, sc + 0, w->partial, w->ctr + 5);
			k_axpy_neg_dev<<<nb, kThreads, 0, st>>>(sc + 0, u, Aq, D);
			k_dot<<<nb, kThreads, 0, st>>>(p, Aq, D, sc + 1, w->partial, w->ctr + 7);
			k_pcg_update<<<nb, kThreads, 0, st>>>(t, res, p, Aq, sc + 10 + cur, sc + 1, sc + 4, h->d_diag,
			                                      theta, floor_, u, wv, D, sc + 6, w->partial, w->ctr + 9);
			k_pcg_direction<<<nb, kThreads, 0, st>>>(p, res, h->d_diag, theta, floor_, wv, sc + 5, sc + 6,
			                                         sc + 10 + cur, sc + 11 - cur, sc + 4, 0, D);
			cur ^= 1;
		}
		if ((e = cudaGetLastError()))
			return cuda_status(h, e, "correction solve launch");
		double four[6];
		if (!read(sc + 4, 6, four))
			return handle_fail(h, DMRGPP_CUDA_ERROR, "correction solve");
		rrh = four[5]; // sums[3] = |res|^2
		if (four[0] != 0.0)
			break; // the projected operator was not positive definite
	}
	if (iterations)
		*iterations = it;
	if (rel_residual)
		*rel_residual = b0 > 0 ? std::sqrt(rrh) / b0 : 0.0;
	return cudaStreamSynchronize(st) == cudaSuccess ? DMRGPP_OK
	                                                : handle_fail(h, DMRGPP_CUDA_ERROR, "correction solve");
}

} // namespace
} // namespace dmrgpp

extern "C" {


int dmrgpp_kron_diagonal(dmrgpp_kron_handle h, double* diag)
{
	if (h && h->complex_sector)
		return dmrgpp::handle_fail(h, DMRGPP_NOT_SUPPORTED, "the device eigensolvers take real sectors");
	if (!h || !diag)
		return DMRGPP_INVALID_ARG;
	const size_t D = size_t(h->plan.dim());
	return cudaMemcpyAsync(diag, h->d_diag, D * sizeof(double), cudaMemcpyDeviceToDevice, h->stream)
	        == cudaSuccess
	    ? DMRGPP_OK
	    : DMRGPP_CUDA_ERROR;
}

int dmrgpp_set_correction_preconditioner(dmrgpp_kron_handle h, int preconditioner)
{
	if (!h)
		return DMRGPP_INVALID_ARG;
	if (preconditioner != DMRGPP_PRECOND_NONE && preconditioner != DMRGPP_PRECOND_JACOBI)
		return dmrgpp::handle_fail(h, DMRGPP_INVALID_ARG, "correction preconditioner: none or Jacobi");
	h->correction_precond = preconditioner;
	return DMRGPP_OK;
}

int dmrgpp_correction_solve(dmrgpp_kron_handle h, const double* u, double theta, const double* r,
                            double* t, int max_iterations, double rel_tolerance, int* iterations,
                            double* rel_residual)
{
	DMRGPP_TRACE("dmrgpp_correction_solve");
	if (h && h->complex_sector)
		return dmrgpp::handle_fail(h, DMRGPP_NOT_SUPPORTED, "the device eigensolvers take real sectors");
	using namespace dmrgpp;
	if (!h || !u || !r || !t || max_iterations < 1)
		return DMRGPP_INVALID_ARG;
	const size_t D = size_t(h->plan.dim());
	if (int rc = ensure_davidson(h, D, 2))
		return rc;
	DavidsonWork* w  = h->davidson;
	cudaStream_t  st = h->stream;
	const int     nb = blocks_for(D);
	// vectors: res = w->hu, p = w->r, Aq = second basis column; scalars
	// sc[0] = u.v, sc[1] = pAp, sc[2], sc[3] = |res|^2 (alternating),
	// sc[4] = frozen flag
	double*     res = w->hu;
	double*     p   = w->r;
	double*     Aq  = w->V + D;
	double*     sc  = w->scal;
	cudaError_t e;
	auto read = [&](double* dev, int count, double* host) {
		return cudaMemcpyAsync(host, dev, size_t(count) * sizeof(double), cudaMemcpyDeviceToHost, st)
		        == cudaSuccess
		    && cudaStreamSynchronize(st) == cudaSuccess;
	};
	// t = 0, res = -(I - uu^T) r, p = res
	cudaMemsetAsync(t, 0, D * sizeof(double), st);
	cudaMemsetAsync(res, 0, D * sizeof(double), st);
	cudaMemsetAsync(sc + 4, 0, sizeof(double), st);
	k_axpy<<<nb, kThreads, 0, st>>>(-1.0, r, res, D);
	k_dot<<<nb, kThreads, 0, st>>>(u, res, D, sc + 0, w->partial, w->ctr + 5);
	k_axpy_neg_dev<<<nb, kThreads, 0, st>>>(sc + 0, u, res, D);
	if (h->correction_precond == DMRGPP_PRECOND_JACOBI && h->d_diag)
		return pcg_correction(h, u, theta, r, t, max_iterations, rel_tolerance, iterations, rel_residual);
	cudaMemcpyAsync(p, res, D * sizeof(double), cudaMemcpyDeviceToDevice, st);
	k_dot<<<nb, kThreads, 0, st>>>(res, res, D, sc + 2, w->partial, w->ctr + 6);
	double host[4] = { 0, 0, 0, 0 };
	if (!read(sc + 2, 1, host))
		return handle_fail(h, DMRGPP_CUDA_ERROR, "correction solve");
	const double b0  = std::sqrt(host[0]);
	double       rrh = host[0];
	int          it  = 0;
	int          cur = 0; // |res|^2 of the current iterate lives in sc[2 + cur]
	while (it < max_iterations && b0 > 0 && std::sqrt(rrh) > rel_tolerance * b0) {
		const int burst = std::min(8, max_iterations - it);
		for (int q = 0; q < burst; ++q, ++it) {
			// Aq = P (H - theta) p  (p orthogonal to u up to round-off)
			if (int rc = kron_apply_device(h, p, Aq))
				return rc;
			k_axpy<<<nb, kThreads, 0, st>>>(-theta, p, Aq, D);
			k_dot<<<nb, kThreads, 0, st>>>(u, Aq, D, sc + 0, w->partial, w->ctr + 5);
			k_axpy_neg_dev<<<nb, kThreads, 0, st>>>(sc + 0, u, Aq, D);
			k_dot<<<nb, kThreads, 0, st>>>(p, Aq, D, sc + 1, w->partial, w->ctr + 7);
			k_cg_update<<<nb, kThreads, 0, st>>>(t, res, p, Aq, sc + 2 + cur, sc + 1, sc + 3 - cur,
			                                     sc + 4, D, w->partial, w->ctr + 6);
			k_cg_direction<<<nb, kThreads, 0, st>>>(p, res, sc + 3 - cur, sc + 2 + cur, sc + 4, D);
			cur ^= 1;
		}
		if ((e = cudaGetLastError()))
			return cuda_status(h, e, "correction solve launch");
		if (!read(sc + 2, 3, host))
			return handle_fail(h, DMRGPP_CUDA_ERROR, "correction solve");
		rrh = host[cur];
		if (host[2] != 0.0)
			break; // the projected operator was not positive definite
	}
	if (iterations)
		*iterations = it;
	if (rel_residual)
		*rel_residual = b0 > 0 ? std::sqrt(rrh) / b0 : 0.0;
	return cudaStreamSynchronize(st) == cudaSuccess ? DMRGPP_OK
	                                                : handle_fail(h, DMRGPP_CUDA_ERROR, "correction solve");
}

} // extern "C"

// ---------------------------------------------------------------------------
// FP64 residual refinement of an approximate lowest eigenvector computed with
// mixed-precision matvecs: each outer step forms the FP64 Rayleigh quotient
// theta = <psi|H|psi> and residual r = H psi - theta psi, solves the
// projected correction equation (I - psi psi^T)(H - theta)(I - psi psi^T) t
// = -r by conjugate gradients with the handle's (mixed) matvecs, and sets
// psi <- (psi + t)/|psi + t|.  No counterpart in the reference.
// ---------------------------------------------------------------------------
extern "C" {

int dmrgpp_refine_lowest(dmrgpp_kron_handle h, double* psi, int max_outer, double tolerance,
                         int inner_iterations, double inner_tolerance, double* energy,
                         dmrgpp_refine_stats* stats)
{
	DMRGPP_TRACE("dmrgpp_refine_lowest");
	if (h && h->complex_sector)
		return dmrgpp::handle_fail(h, DMRGPP_NOT_SUPPORTED, "the device eigensolvers take real sectors");
	using namespace dmrgpp;
	if (!h || !psi || !energy || max_outer < 0 || inner_iterations < 1)
		return DMRGPP_INVALID_ARG;
	const size_t D = size_t(h->plan.dim());
	int          prev = -1;
	cudaGetDevice(&prev);
	if (prev != h->device)
		cudaSetDevice(h->device);
	struct Restore {
		int dev, prev;
		~Restore()
		{
			if (dev != prev && prev >= 0)
				cudaSetDevice(prev);
		}
	} restore { h->device, prev };
	if (int rc = ensure_davidson(h, D, 2))
		return rc;
	DavidsonWork* w    = h->davidson;
	cudaStream_t  st   = h->stream;
	const int     nb   = blocks_for(D);
	double*       hpsi = w->W;     // W column 0
	double*       r    = w->W + D; // W column 1
	double*       t    = w->V;     // V column 0 (the correction solve uses column 1)
	const int     user = h->precision;
	dmrgpp_refine_stats s {};
	double        theta = 0.0, rnorm = 0.0;
	double        best  = std::numeric_limits<double>::infinity();
	int           stall = 0;
	int           rc    = DMRGPP_OK;
	cudaError_t   e;
	for (int outer = 0; outer <= max_outer; ++outer) {
		// normalise psi, then FP64 Rayleigh quotient and residual
		k_dot<<<nb, kThreads, 0, st>>>(psi, psi, D, w->scal + 8, w->partial, w->ctr + 8);
		k_scale_rsqrt<<<nb, kThreads, 0, st>>>(psi, psi, D, w->scal + 8);
		h->precision = DMRGPP_FP64;
		rc           = kron_apply_device(h, psi, hpsi);
		h->precision = user;
		if (rc)
			break;
		++s.fp64_matvecs;
		k_dot<<<nb, kThreads, 0, st>>>(psi, hpsi, D, w->scal + 9, w->partial, w->ctr + 9);
		if ((e = cudaMemcpyAsync(w->host, w->scal + 9, sizeof(double), cudaMemcpyDeviceToHost, st))
		    || (e = cudaStreamSynchronize(st))) {
			rc = cuda_status(h, e, "refinement Rayleigh quotient");
			break;
		}
		theta = w->host[0];
		k_residual<<<nb, kThreads, 0, st>>>(hpsi, psi, theta, r, D, w->scal + 10, w->partial,
		                                    w->ctr + 10);
		if ((e = cudaMemcpyAsync(w->host, w->scal + 10, sizeof(double), cudaMemcpyDeviceToHost, st))
		    || (e = cudaStreamSynchronize(st))) {
			rc = cuda_status(h, e, "refinement residual");
			break;
		}
		rnorm = w->host[0];
		s.outer_iterations = size_t(outer);
		if (rnorm <= tolerance * std::max(1.0, std::fabs(theta))) {
			s.converged = 1;
			break;
		}
		if (outer == max_outer)
			break;
		// a residual that has not halved over two outer steps means a failing
		// refinement (start above the first excitation): stop, unconverged
		if (rnorm < 0.5 * best) {
			best  = rnorm;
			stall = 0;
		} else if (++stall >= 2) {
			break;
		}
		int    its = 0;
		double rel = 0.0;
		if ((rc = dmrgpp_correction_solve(h, psi, theta, r, t, inner_iterations, inner_tolerance, &its,
		                                  &rel)))
			break;
		s.inner_matvecs += size_t(its);
		k_axpy<<<nb, kThreads, 0, st>>>(1.0, t, psi, D);
	}
	if (rc)
		return rc;
	if (h->err_host && *reinterpret_cast<volatile int*>(h->err_host))
		return handle_fail(h, DMRGPP_TIMEOUT, "H*x kernel wait gave up during refinement");
	*energy         = theta;
	s.residual_norm = rnorm;
	if (stats)
		*stats = s;
	return s.converged ? DMRGPP_OK : handle_fail(h, DMRGPP_NOT_CONVERGED, "refinement did not converge");
}

} // extern "C"
