// Lanczos for every sector of a group handle at once (dmrgpp_kron_create_group):
// all sectors advance in lockstep, one persistent launch applies H to all of
// them per step, and every vector operation is segmented by sector.
//
// Per sector the recurrence is that of the single-sector solver (lanczos.cu,
// following LanczosCore::decomposition, LanczosCore.h:147-272, and
// LanczosVectors::oneStepDecomposition / reorthoIfNecessary,
// LanczosVectors.h:203-271): normalise, V1 = H V0 - a0 V0, then
// V2 = H V1 - a_j V1 - b_j V0, b_{j+1} = |V2|, V2 /= b_{j+1}, full
// reorthogonalisation against the stored vectors (classical Gram-Schmidt)
// and renormalisation.  The stopping test runs on the host every
// check_every steps: a sector stops at the first test point where its lowest
// eigs_for_stop Ritz values changed by less than the tolerance over the last
// step (after min_steps steps), or when its Krylov space is exhausted.  A
// stopped sector is masked out of every later vector operation and out of
// the group H*x (the persistent kernel drops its items).  No counterpart in
// the reference.
//
// The sector vectors are cut into chunks of at most kChunk rows that never
// cross a sector boundary; every kernel walks chunks, so each block knows its
// sector, and every sum runs in a fixed order (bitwise reproducible).
#include "dmrgpp_kron.h"
#include "trace.h"
#include "devmem.h"
#include "handle.h"
#include "mlp.h"
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

constexpr int kThreads = 256;
constexpr int kChunk   = 2048; // rows per chunk
constexpr int kGrid    = 1184; // at most 8 blocks per SM

struct Chunk {
	long long begin;
	int       len;
	int       seg;
};

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

// partial[ch] = <x, y> over chunk ch (0 for stopped sectors)
__global__ void __launch_bounds__(kThreads)
k_g_dot(const double* __restrict__ x, const double* __restrict__ y, const Chunk* __restrict__ chunks,
        int nch, const int* __restrict__ active, double* __restrict__ partial)
{
	__shared__ double red[kThreads / 32];
	for (int ch = blockIdx.x; ch < nch; ch += gridDim.x) {
		const Chunk c = chunks[ch];
		double      s = 0.0;
		if (active[c.seg])
			for (int i = threadIdx.x; i < c.len; i += kThreads)
				s += x[c.begin + i] * y[c.begin + i];
		s = block_sum(s, red);
		if (threadIdx.x == 0)
			partial[ch] = s;
	}
}

// out[s] = sum of the sector's chunk partials (sqrt of it when root), for
// active sectors; one block per sector
__global__ void __launch_bounds__(kThreads)
k_g_finish(const double* __restrict__ partial, const int* __restrict__ seg_chunk,
           const int* __restrict__ active, double* __restrict__ out, int root)
{
	__shared__ double red[kThreads / 32];
	const int         s = blockIdx.x;
	if (!active[s])
		return;
	double t = 0.0;
	for (int ch = seg_chunk[s] + threadIdx.x; ch < seg_chunk[s + 1]; ch += kThreads)
		t += partial[ch];
	t = block_sum(t, red);
	if (threadIdx.x == 0)
		out[s] = root ? sqrt(t) : t;
}

// y = x * f(scal[sector]): mode 0 f = 1/sqrt(v) (v a squared norm), mode 1
// f = 1/v when v > 0 (else y = x); active sectors only.  y may be x (each
// element is read and then written by one thread), so they are not restrict.
__global__ void __launch_bounds__(kThreads)
k_g_scale(const double* x, double* y, const double* __restrict__ scal,
          int mode, const Chunk* __restrict__ chunks, int nch, const int* __restrict__ active)
{
	for (int ch = blockIdx.x; ch < nch; ch += gridDim.x) {
		const Chunk c = chunks[ch];
		if (!active[c.seg])
			continue;
		const double v = scal[c.seg];
		double       f = 1.0;
		if (mode == 0)
			f = 1.0 / sqrt(v);
		else if (v > 0.0)
			f = 1.0 / v;
		for (int i = threadIdx.x; i < c.len; i += kThreads)
			y[c.begin + i] = x[c.begin + i] * f;
	}
}

// v2 -= alpha[s] v1 + beta[s] v0 (v0 may be null); partial[ch] = |v2|^2 over ch
__global__ void __launch_bounds__(kThreads)
k_g_update(double* __restrict__ v2, const double* __restrict__ v1, const double* __restrict__ v0,
           const double* __restrict__ alpha, const double* __restrict__ beta,
           const Chunk* __restrict__ chunks, int nch, const int* __restrict__ active,
           double* __restrict__ partial)
{
	__shared__ double red[kThreads / 32];
	for (int ch = blockIdx.x; ch < nch; ch += gridDim.x) {
		const Chunk c = chunks[ch];
		double      s = 0.0;
		if (active[c.seg]) {
			const double a = alpha[c.seg], b = v0 ? beta[c.seg] : 0.0;
			for (int i = threadIdx.x; i < c.len; i += kThreads) {
				const long long q = c.begin + i;
				double          w = v2[q] - a * v1[q];
				if (v0)
					w -= b * v0[q];
				v2[q] = w;
				s += w * w;
			}
		}
		s = block_sum(s, red);
		if (threadIdx.x == 0)
			partial[ch] = s;
	}
}

// partial[ch * ldp + c] = <V[:, c], v> over chunk ch, c < ncols (active
// sectors).  Chunks that start on an even row use 16-byte loads (ld even).
__global__ void __launch_bounds__(kThreads)
k_g_basis_dots(const double* __restrict__ V, size_t ld, int ncols, const double* __restrict__ v,
               const Chunk* __restrict__ chunks, int nch, const int* __restrict__ active,
               double* __restrict__ partial, int ldp)
{
	__shared__ __align__(16) double vs[kChunk];
	const int                       lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	for (int ch = blockIdx.x; ch < nch; ch += gridDim.x) {
		const Chunk c = chunks[ch];
		if (!active[c.seg])
			continue;
		__syncthreads();
		for (int i = threadIdx.x; i < c.len; i += kThreads)
			vs[i] = v[c.begin + i];
		__syncthreads();
		const bool vec = ((c.begin | static_cast<long long>(ld)) & 1) == 0;
		for (int col = warp; col < ncols; col += kThreads / 32) {
			const double* cp = V + size_t(col) * ld + c.begin;
			double        s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
			if (vec) {
				const double2* c2 = reinterpret_cast<const double2*>(cp);
				const double2* v2 = reinterpret_cast<const double2*>(vs);
				const int      np = c.len >> 1;
				int            q  = lane;
				for (; q + 96 < np; q += 128) {
					const double2 a0 = __ldg(c2 + q), a1 = __ldg(c2 + q + 32);
					const double2 a2 = __ldg(c2 + q + 64), a3 = __ldg(c2 + q + 96);
					const double2 b0 = v2[q], b1 = v2[q + 32], b2 = v2[q + 64], b3 = v2[q + 96];
					s0 += a0.x * b0.x + a0.y * b0.y;
					s1 += a1.x * b1.x + a1.y * b1.y;
					s2 += a2.x * b2.x + a2.y * b2.y;
					s3 += a3.x * b3.x + a3.y * b3.y;
				}
				for (; q < np; q += 32) {
					const double2 a0 = __ldg(c2 + q), b0 = v2[q];
					s0 += a0.x * b0.x + a0.y * b0.y;
				}
				if ((c.len & 1) && lane == 0)
					s1 += __ldg(cp + c.len - 1) * vs[c.len - 1];
			} else {
				int i = lane;
				for (; i + 96 < c.len; i += 128) {
					s0 += __ldg(cp + i) * vs[i];
					s1 += __ldg(cp + i + 32) * vs[i + 32];
					s2 += __ldg(cp + i + 64) * vs[i + 64];
					s3 += __ldg(cp + i + 96) * vs[i + 96];
				}
				for (; i < c.len; i += 32)
					s0 += __ldg(cp + i) * vs[i];
			}
			double s = (s0 + s1) + (s2 + s3);
			for (int o = 16; o > 0; o >>= 1)
				s += __shfl_down_sync(0xffffffffu, s, o);
			if (lane == 0)
				partial[size_t(ch) * ldp + col] = s;
		}
	}
}

// r[s * ldp + c] = sum over the sector's chunks of partial[ch * ldp + c]
__global__ void __launch_bounds__(kThreads)
k_g_basis_reduce(const double* __restrict__ partial, int ldp, int ncols,
                 const int* __restrict__ seg_chunk, const int* __restrict__ active,
                 double* __restrict__ r)
{
	const int s = blockIdx.x;
	if (!active[s])
		return;
	for (int col = threadIdx.x; col < ncols; col += kThreads) {
		double t = 0.0;
		for (int ch = seg_chunk[s]; ch < seg_chunk[s + 1]; ++ch)
			t += partial[size_t(ch) * ldp + col];
		r[size_t(s) * ldp + col] = t;
	}
}

// v -= V[:, 0..ncols) r[sector]; partial[ch] = |v|^2 over ch.  Chunks that
// start on an even row: row pairs, 16-byte loads, 8 columns in flight.
__global__ void __launch_bounds__(kThreads)
k_g_basis_subtract(double* __restrict__ v, const double* __restrict__ V, size_t ld, int ncols,
                   const double* __restrict__ r, int ldp, const Chunk* __restrict__ chunks, int nch,
                   const int* __restrict__ active, double* __restrict__ partial)
{
	__shared__ double rs[1024];
	__shared__ double red[kThreads / 32];
	for (int ch = blockIdx.x; ch < nch; ch += gridDim.x) {
		const Chunk c = chunks[ch];
		double      s = 0.0;
		if (active[c.seg]) {
			__syncthreads();
			for (int col = threadIdx.x; col < ncols; col += kThreads)
				rs[col] = r[size_t(c.seg) * ldp + col];
			__syncthreads();
			const bool vec = ((c.begin | static_cast<long long>(ld)) & 1) == 0;
			if (vec) {
				const int np = c.len >> 1;
				double2*  v2 = reinterpret_cast<double2*>(v + c.begin);
				for (int p = threadIdx.x; p < np; p += kThreads) {
					double2 w   = v2[p];
					int     col = 0;
					for (; col + 8 <= ncols; col += 8) {
						double2 a[8];
#pragma unroll
						for (int u = 0; u < 8; ++u)
							a[u] = __ldg(reinterpret_cast<const double2*>(V + size_t(col + u) * ld + c.begin) + p);
#pragma unroll
						for (int u = 0; u < 8; ++u) {
							w.x -= a[u].x * rs[col + u];
							w.y -= a[u].y * rs[col + u];
						}
					}
					for (; col < ncols; ++col) {
						const double2 a = __ldg(reinterpret_cast<const double2*>(V + size_t(col) * ld + c.begin) + p);
						w.x -= a.x * rs[col];
						w.y -= a.y * rs[col];
					}
					v2[p] = w;
					s += w.x * w.x + w.y * w.y;
				}
				if ((c.len & 1) && threadIdx.x == 0) {
					const long long q = c.begin + c.len - 1;
					double          w = v[q];
					for (int col = 0; col < ncols; ++col)
						w -= __ldg(V + size_t(col) * ld + q) * rs[col];
					v[q] = w;
					s += w * w;
				}
			} else {
				for (int i = threadIdx.x; i < c.len; i += kThreads) {
					const long long q   = c.begin + i;
					double          w   = v[q];
					for (int col = 0; col < ncols; ++col)
						w -= __ldg(V + size_t(col) * ld + q) * rs[col];
					v[q] = w;
					s += w * w;
				}
			}
		}
		s = block_sum(s, red);
		if (threadIdx.x == 0)
			partial[ch] = s;
	}
}

// z = V[:, 0..ncols[s]) coef[s] for every sector (active ones when active
// is not NULL)
__global__ void __launch_bounds__(kThreads)
k_g_basis_combine(double* __restrict__ z, const double* __restrict__ V, size_t ld,
                  const int* __restrict__ ncols, const double* __restrict__ coef, int ldp,
                  const Chunk* __restrict__ chunks, int nch, const int* __restrict__ active)
{
	__shared__ double cs[1024];
	for (int ch = blockIdx.x; ch < nch; ch += gridDim.x) {
		const Chunk c  = chunks[ch];
		if (active && !active[c.seg])
			continue;
		const int   nc = ncols[c.seg];
		__syncthreads();
		for (int col = threadIdx.x; col < nc; col += kThreads)
			cs[col] = coef[size_t(c.seg) * ldp + col];
		__syncthreads();
		for (int i = threadIdx.x; i < c.len; i += kThreads) {
			const long long q = c.begin + i;
			double          w = 0.0;
			for (int col = 0; col < nc; ++col)
				w += cs[col] * __ldg(V + size_t(col) * ld + q);
			z[q] = w;
		}
	}
}

// ---- segmented kernels of the group refinement (dmrgpp_refine_lowest_group)

// y += sgn * c[sector] * x (c null: coefficient 1), active sectors
__global__ void __launch_bounds__(kThreads)
k_g_axpy(double* __restrict__ y, const double* __restrict__ x, const double* __restrict__ c, double sgn,
         const Chunk* __restrict__ chunks, int nch, const int* __restrict__ active)
{
	for (int ch = blockIdx.x; ch < nch; ch += gridDim.x) {
		const Chunk k = chunks[ch];
		if (!active[k.seg])
			continue;
		const double f = sgn * (c ? c[k.seg] : 1.0);
		for (int i = threadIdx.x; i < k.len; i += kThreads)
			y[k.begin + i] += f * x[k.begin + i];
	}
}

// r = hu - theta[sector] u; partial[ch] = |r|^2 over ch
__global__ void __launch_bounds__(kThreads)
k_g_residual(const double* __restrict__ hu, const double* __restrict__ u, const double* __restrict__ theta,
             double* __restrict__ r, const Chunk* __restrict__ chunks, int nch,
             const int* __restrict__ active, double* __restrict__ partial)
{
	__shared__ double red[kThreads / 32];
	for (int ch = blockIdx.x; ch < nch; ch += gridDim.x) {
		const Chunk k = chunks[ch];
		double      s = 0.0;
		if (active[k.seg]) {
			const double th = theta[k.seg];
			for (int i = threadIdx.x; i < k.len; i += kThreads) {
				const long long q = k.begin + i;
				const double    w = hu[q] - th * u[q];
				r[q]              = w;
				s += w * w;
			}
		}
		s = block_sum(s, red);
		if (threadIdx.x == 0)
			partial[ch] = s;
	}
}

// CG step of every active sector: alpha = rr / pAp (0 when pAp <= 0: the
// check below then stops the sector), t += alpha p, res -= alpha Aq;
// partial[ch] = |res|^2 over ch
__global__ void __launch_bounds__(kThreads)
k_g_cg_update(double* __restrict__ t, double* __restrict__ res, const double* __restrict__ p,
              const double* __restrict__ Aq, const double* __restrict__ rr, const double* __restrict__ pAp,
              const Chunk* __restrict__ chunks, int nch, const int* __restrict__ active,
              double* __restrict__ partial)
{
	__shared__ double red[kThreads / 32];
	for (int ch = blockIdx.x; ch < nch; ch += gridDim.x) {
		const Chunk k = chunks[ch];
		double      s = 0.0;
		if (active[k.seg]) {
			const double d     = pAp[k.seg];
			const double alpha = d > 0.0 ? rr[k.seg] / d : 0.0;
			for (int i = threadIdx.x; i < k.len; i += kThreads) {
				const long long q = k.begin + i;
				t[q] += alpha * p[q];
				const double w = res[q] - alpha * Aq[q];
				res[q]         = w;
				s += w * w;
			}
		}
		s = block_sum(s, red);
		if (threadIdx.x == 0)
			partial[ch] = s;
	}
}

// ---- diagonal (Jacobi) preconditioner of the group correction solves, per
// sector as in lanczos.cu (pcg_correction): K = diag(H) - theta[sector], kept
// at least 1e-3 max(1, |theta|); z = K^-1 res - a K^-1 u with a = <u, K^-1 res>
// / <u, K^-1 u>, orthogonal to the sector's u.
__device__ __forceinline__ double g_pcg_k(double d, double th)
{
	const double f = 1e-3 * fmax(1.0, fabs(th));
	const double k = d - th;
	return k > f ? k : f;
}

// wv = K^-1 u; partial[ch] = <u, wv> over ch
__global__ void __launch_bounds__(kThreads)
k_g_pcg_setup(const double* __restrict__ u, const double* __restrict__ diag, const double* __restrict__ theta,
              double* __restrict__ wv, const Chunk* __restrict__ chunks, int nch, const int* __restrict__ active,
              double* __restrict__ partial)
{
	__shared__ double red[kThreads / 32];
	for (int ch = blockIdx.x; ch < nch; ch += gridDim.x) {
		const Chunk k = chunks[ch];
		double      s = 0.0;
		if (active[k.seg]) {
			const double th = theta[k.seg];
			for (int i = threadIdx.x; i < k.len; i += kThreads) {
				const long long q = k.begin + i;
				const double    v = u[q] / g_pcg_k(diag[q], th);
				wv[q]             = v;
				s += u[q] * v;
			}
		}
		s = block_sum(s, red);
		if (threadIdx.x == 0)
			partial[ch] = s;
	}
}

// partial[ch], [nch + ch], [2 nch + ch] = <u, K^-1 res>, <res, K^-1 res>, <res, wv> over ch
__global__ void __launch_bounds__(kThreads)
k_g_pcg_sums(const double* __restrict__ res, const double* __restrict__ diag, const double* __restrict__ theta,
             const double* __restrict__ u, const double* __restrict__ wv, const Chunk* __restrict__ chunks,
             int nch, const int* __restrict__ active, double* __restrict__ partial)
{
	__shared__ double red[kThreads / 32];
	for (int ch = blockIdx.x; ch < nch; ch += gridDim.x) {
		const Chunk k = chunks[ch];
		double      v0 = 0.0, v1 = 0.0, v2 = 0.0;
		if (active[k.seg]) {
			const double th = theta[k.seg];
			for (int i = threadIdx.x; i < k.len; i += kThreads) {
				const long long q = k.begin + i;
				const double    r = res[q];
				const double    z = r / g_pcg_k(diag[q], th);
				v0 += u[q] * z;
				v1 += r * z;
				v2 += r * wv[q];
			}
		}
		v0 = block_sum(v0, red);
		v1 = block_sum(v1, red);
		v2 = block_sum(v2, red);
		if (threadIdx.x == 0) {
			partial[ch]           = v0;
			partial[nch + ch]     = v1;
			partial[2 * nch + ch] = v2;
		}
	}
}

// p = z + (rho_new / rho) p (p = z when first), rho_new = sums1 - a sums2,
// a = sums0 / uw; every chunk of a sector computes the same rho_new, and its
// sector's first chunk stores it in rho_next
__global__ void __launch_bounds__(kThreads)
k_g_pcg_direction(double* __restrict__ p, const double* __restrict__ res, const double* __restrict__ diag,
                  const double* __restrict__ theta, const double* __restrict__ wv, const double* __restrict__ uw,
                  const double* __restrict__ sums, int nseg, const double* __restrict__ rho,
                  double* __restrict__ rho_next, int first, const Chunk* __restrict__ chunks, int nch,
                  const int* __restrict__ seg_chunk, const int* __restrict__ active)
{
	for (int ch = blockIdx.x; ch < nch; ch += gridDim.x) {
		const Chunk k = chunks[ch];
		if (!active[k.seg])
			continue;
		const int    sg      = k.seg;
		const double a       = uw[sg] > 0.0 ? sums[sg] / uw[sg] : 0.0;
		const double rho_new = sums[nseg + sg] - a * sums[2 * nseg + sg];
		const double beta    = first ? 0.0 : (rho[sg] > 0.0 ? rho_new / rho[sg] : 0.0);
		if (threadIdx.x == 0 && ch == seg_chunk[sg])
			rho_next[sg] = rho_new;
		const double th = theta[sg];
		for (int i = threadIdx.x; i < k.len; i += kThreads) {
			const long long q = k.begin + i;
			const double    z = res[q] / g_pcg_k(diag[q], th) - a * wv[q];
			p[q]              = z + beta * p[q];
		}
	}
}

// one thread per sector: stop the sector's CG on a non-positive pAp or once
// |res| <= tol * b0
__global__ void k_g_cg_check(const double* __restrict__ pAp, const double* __restrict__ rr_next,
                             const double* __restrict__ b0, double tol, int* __restrict__ active, int nseg)
{
	const int s = blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= nseg || !active[s])
		return;
	if (!(pAp[s] > 0.0) || sqrt(rr_next[s]) <= tol * b0[s])
		active[s] = 0;
}

// one thread per sector: the CG runs for outer-active sectors with b0 > 0
__global__ void k_g_cg_start(const double* __restrict__ b0, const int* __restrict__ outer,
                             int* __restrict__ active, int nseg)
{
	const int s = blockIdx.x * blockDim.x + threadIdx.x;
	if (s < nseg)
		active[s] = outer[s] && b0[s] > 0.0 ? 1 : 0;
}

// p = res + (rr_next / rr) p, active sectors
__global__ void __launch_bounds__(kThreads)
k_g_cg_direction(double* __restrict__ p, const double* __restrict__ res, const double* __restrict__ rr_next,
                 const double* __restrict__ rr, const Chunk* __restrict__ chunks, int nch,
                 const int* __restrict__ active)
{
	for (int ch = blockIdx.x; ch < nch; ch += gridDim.x) {
		const Chunk k = chunks[ch];
		if (!active[k.seg])
			continue;
		const double beta = rr[k.seg] > 0.0 ? rr_next[k.seg] / rr[k.seg] : 0.0;
		for (int i = threadIdx.x; i < k.len; i += kThreads)
			p[k.begin + i] = res[k.begin + i] + beta * p[k.begin + i];
	}
}

// Jacobi correction of every active sector: t = r / (theta[s] - d), the
// denominator kept at least floor_rel * max(1, |theta[s]|) in magnitude
__global__ void __launch_bounds__(kThreads)
k_g_jacobi(const double* __restrict__ r, const double* __restrict__ d, const double* __restrict__ theta,
           double floor_rel, double* __restrict__ t, const Chunk* __restrict__ chunks, int nch,
           const int* __restrict__ active)
{
	for (int ch = blockIdx.x; ch < nch; ch += gridDim.x) {
		const Chunk k = chunks[ch];
		if (!active[k.seg])
			continue;
		const double th = theta[k.seg];
		const double fl = floor_rel * fmax(1.0, fabs(th));
		for (int i = threadIdx.x; i < k.len; i += kThreads) {
			const long long q   = k.begin + i;
			double          den = th - d[q];
			if (fabs(den) < fl)
				den = den < 0 ? -fl : fl;
			t[q] = r[q] / den;
		}
	}
}

int status(dmrgpp_kron_handle h, cudaError_t e, const char* where)
{
	return handle_fail(h, DMRGPP_CUDA_ERROR, std::string(where) + ": " + cudaGetErrorString(e));
}

} // namespace

// Device buffers of the group solver of one handle.
struct GroupWork {
	size_t  dim = 0;
	int     cols = 0, nseg = 0, nch = 0;
	double* V       = nullptr; // dim x cols
	double* z       = nullptr; // dim, Ritz vectors
	double* alpha   = nullptr; // cols x nseg (step-major)
	double* beta    = nullptr; // (cols + 1) x nseg
	double* scal    = nullptr; // nseg x 4 scratch (norms)
	double* partial = nullptr; // nch x cols
	double* r       = nullptr; // nseg x cols (projections, Ritz coefficients)
	Chunk*  chunks  = nullptr;
	int*    seg_chunk = nullptr; // nseg + 1
	int*    active  = nullptr;   // nseg
	int*    ncols   = nullptr;   // nseg (Ritz vector lengths)
	double* host    = nullptr;   // pinned: alpha, beta
	// refinement (dmrgpp_refine_lowest_group), allocated on first use
	double* rv    = nullptr; // 7 x dim: H psi, r, t, res, p, Aq, K^-1 psi (Jacobi corrections)
	double* rsc   = nullptr; // 8 x nseg scalars
	double* rpsc  = nullptr; // 6 x nseg: Jacobi corrections' <u,K^-1 u>, three sums, rho[2]
	double* rpart = nullptr; // 3 x nch chunk partials of those sums
	int*    rint  = nullptr; // 2 x nseg: outer active, CG active
	double* rhost = nullptr; // pinned: theta, |r| (2 x nseg), then 2 x nseg ints
	long long* sec_start = nullptr; // nseg + 1 sector offsets
	// Davidson (dmrgpp_davidson_lowest_group), allocated on first use
	int     dmax   = 0;       // basis columns of dV / dW
	double* dV     = nullptr; // dim x dmax, per-sector orthonormal bases
	double* dW     = nullptr; // dim x dmax, H V
	double* dvec   = nullptr; // 4 x dim: Ritz vectors, H u, residuals, corrections
	double* dsc    = nullptr; // 3 x nseg: theta, |r|, norms
	double* dcoef  = nullptr; // nseg x cols: Ritz coefficients
};

void release_group(dmrgpp_kron_handle h)
{
	GroupWork* w = h->group;
	if (!w)
		return;
	dmrgpp::dev_free(w->V);
	dmrgpp::dev_free(w->z);
	dmrgpp::dev_free(w->alpha);
	dmrgpp::dev_free(w->beta);
	dmrgpp::dev_free(w->scal);
	dmrgpp::dev_free(w->partial);
	dmrgpp::dev_free(w->r);
	dmrgpp::dev_free(w->chunks);
	dmrgpp::dev_free(w->seg_chunk);
	dmrgpp::dev_free(w->active);
	dmrgpp::dev_free(w->ncols);
	if (w->host)
		cudaFreeHost(w->host);
	dmrgpp::dev_free(w->rv);
	dmrgpp::dev_free(w->rsc);
	dmrgpp::dev_free(w->rpsc);
	dmrgpp::dev_free(w->rpart);
	dmrgpp::dev_free(w->rint);
	if (w->rhost)
		cudaFreeHost(w->rhost);
	dmrgpp::dev_free(w->sec_start);
	dmrgpp::dev_free(w->dV);
	dmrgpp::dev_free(w->dW);
	dmrgpp::dev_free(w->dvec);
	dmrgpp::dev_free(w->dsc);
	dmrgpp::dev_free(w->dcoef);
	delete w;
	h->group = nullptr;
}

namespace {

int ensure_group_work(dmrgpp_kron_handle h, int cols)
{
	const size_t dim  = size_t(h->plan.dim());
	const int    nseg = int(h->sector_start.size()) - 1;
	GroupWork*   w    = h->group;
	if (w && w->dim == dim && w->cols >= cols && w->nseg == nseg)
		return DMRGPP_OK;
	release_group(h);
	w        = new GroupWork();
	h->group = w;
	w->dim   = dim;
	w->cols  = cols;
	w->nseg  = nseg;
	std::vector<Chunk> ch;
	std::vector<int>   sc(1, 0);
	for (int s = 0; s < nseg; ++s) {
		// chunk boundaries on even offsets (16-byte aligned rows) after the first
		const long long end = h->sector_start[size_t(s) + 1];
		long long       b   = h->sector_start[size_t(s)];
		while (b < end) {
			const long long e = std::min(end, ((b + kChunk) / 2) * 2);
			ch.push_back({ b, int(e - b), s });
			b = e;
		}
		sc.push_back(int(ch.size()));
	}
	w->nch = int(ch.size());
	cudaError_t e;
	const size_t nsc = size_t(nseg) * size_t(cols);
	if ((e = dmrgpp::dev_malloc(&w->V, dim * size_t(cols) * sizeof(double))) || (e = dmrgpp::dev_malloc(&w->z, dim * sizeof(double)))
	    || (e = dmrgpp::dev_malloc(&w->alpha, nsc * sizeof(double)))
	    || (e = dmrgpp::dev_malloc(&w->beta, (nsc + size_t(nseg)) * sizeof(double)))
	    || (e = dmrgpp::dev_malloc(&w->scal, size_t(nseg) * 4 * sizeof(double)))
	    || (e = dmrgpp::dev_malloc(&w->partial, std::max<size_t>(1, ch.size()) * size_t(cols) * sizeof(double)))
	    || (e = dmrgpp::dev_malloc(&w->r, nsc * sizeof(double)))
	    || (e = dmrgpp::dev_malloc(&w->chunks, std::max<size_t>(1, ch.size()) * sizeof(Chunk)))
	    || (e = dmrgpp::dev_malloc(&w->seg_chunk, sc.size() * sizeof(int)))
	    || (e = dmrgpp::dev_malloc(&w->active, size_t(nseg) * sizeof(int)))
	    || (e = dmrgpp::dev_malloc(&w->ncols, size_t(nseg) * sizeof(int)))
	    || (e = dmrgpp::dev_malloc(&w->sec_start, (size_t(nseg) + 1) * sizeof(long long)))
	    || (e = cudaHostAlloc(&w->host, 2 * (2 * nsc + size_t(nseg)) * sizeof(double), 0)))
		return status(h, e, "group solver allocation");
	if ((e = dmrgpp::upload_sync(w->chunks, ch.data(), ch.size() * sizeof(Chunk), h->stream))
	    || (e = dmrgpp::upload_sync(w->seg_chunk, sc.data(), sc.size() * sizeof(int), h->stream))
	    || (e = dmrgpp::upload_sync(w->sec_start, h->sector_start.data(), (size_t(nseg) + 1) * sizeof(long long),
	                                h->stream))
	    || (e = dmrgpp::clear_async(w->beta, (nsc + size_t(nseg)) * sizeof(double), h->stream))
	    || (e = dmrgpp::clear_async(w->alpha, nsc * sizeof(double), h->stream)))
		return status(h, e, "group solver set-up");
	return DMRGPP_OK;
}

} // namespace

} // namespace dmrgpp

extern "C" int dmrgpp_lanczos_lowest_group_masked(dmrgpp_kron_handle h, const dmrgpp_lanczos_params* p,
                                                  const double* init, int on_device, const int* mask,
                                                  double* energies, double* z, size_t* steps_taken);

extern "C" int dmrgpp_lanczos_lowest_group(dmrgpp_kron_handle h, const dmrgpp_lanczos_params* p,
                                           const double* init, int on_device, double* energies,
                                           double* z, size_t* steps_taken)
{
	return dmrgpp_lanczos_lowest_group_masked(h, p, init, on_device, nullptr, energies, z, steps_taken);
}

// mask (host, one int per sector; NULL = every sector): sectors with mask 0
// take no part (no H*x items, no vector work); their energies are NaN, their
// part of z is zero and their steps_taken 0.
extern "C" int dmrgpp_lanczos_lowest_group_masked(dmrgpp_kron_handle h, const dmrgpp_lanczos_params* p,
                                                  const double* init, int on_device, const int* mask,
                                                  double* energies, double* z, size_t* steps_taken)
{
	DMRGPP_TRACE("dmrgpp_lanczos_lowest_group_masked");
	if (h && h->complex_sector)
		return dmrgpp::handle_fail(h, DMRGPP_NOT_SUPPORTED, "the device eigensolvers take real sectors");
	using namespace dmrgpp;
	if (!h)
		return DMRGPP_INVALID_ARG;
	if (!p || !init || !energies || !z)
		return handle_fail(h, DMRGPP_INVALID_ARG, "null argument");
	if (p->steps < 1 || p->check_every < 1 || p->eigs_for_stop < 1)
		return handle_fail(h, DMRGPP_INVALID_ARG, "steps, check_every and eigs_for_stop must be >= 1");
	const int    S = int(h->sector_start.size()) - 1;
	const size_t D = size_t(h->plan.dim());
	std::vector<size_t> maxn_s(static_cast<size_t>(S));
	size_t              maxn = 1;
	for (int s = 0; s < S; ++s) {
		const size_t Ds = size_t(h->sector_start[size_t(s) + 1] - h->sector_start[size_t(s)]);
		maxn_s[size_t(s)] = std::max<size_t>(1, std::min(p->steps, Ds)); // LanczosCore.h:177-178
		maxn              = std::max(maxn, maxn_s[size_t(s)]);
	}
	if (maxn + 1 > 1024)
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

	const int cols = int(maxn) + 1;
	if (int rc = ensure_group_work(h, cols))
		return rc;
	GroupWork*         w   = h->group;
	const cudaStream_t st  = h->stream;
	const int          nch = w->nch;
	const int          grid = std::max(1, std::min(nch, kGrid));
	const int          ldp = w->cols;
	auto               col = [&](size_t c) { return w->V + c * D; };
	auto               al  = [&](size_t j) { return w->alpha + j * size_t(S); };
	auto               be  = [&](size_t j) { return w->beta + j * size_t(S); };
	double*            nrm = w->scal;
	cudaError_t        e;

	// the group H*x skips stopped sectors while this solve runs
	h->sector_active = w->active;
	struct MaskOff {
		dmrgpp_kron_handle h;
		~MaskOff() { h->sector_active = nullptr; }
	} mask_off { h };

	std::vector<int> act(size_t(S), 1), skip(size_t(S), 0);
	for (int s = 0; mask && s < S; ++s)
		if (!mask[s]) {
			act[size_t(s)]  = 0;
			skip[size_t(s)] = 1;
		}
	if ((e = cudaMemcpyAsync(w->active, act.data(), size_t(S) * sizeof(int), cudaMemcpyHostToDevice, st))
	    || (e = cudaMemsetAsync(w->beta, 0, size_t(S) * sizeof(double), st))) // beta_0 = 0
		return status(h, e, "group solver start");
	if ((e = cudaMemcpyAsync(col(1), init, D * sizeof(double),
	                         on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st)))
		return status(h, e, "copy initial vectors");

	// per-sector reductions: partial per chunk, then one sum per sector
	auto dot = [&](const double* x, const double* y, double* out, int root) {
		k_g_dot<<<grid, kThreads, 0, st>>>(x, y, w->chunks, nch, w->active, w->partial);
		k_g_finish<<<S, kThreads, 0, st>>>(w->partial, w->seg_chunk, w->active, out, root);
	};
	// V0 = init / |init| per sector (LanczosCore.h:166-175)
	dot(col(1), col(1), nrm, 0);
	k_g_scale<<<grid, kThreads, 0, st>>>(col(1), col(0), nrm, 0, w->chunks, nch, w->active);
	// first step (LanczosCore.h:186-208)
	if (int rc = kron_apply_device(h, col(0), col(1)))
		return rc;
	dot(col(1), col(0), al(0), 0);
	k_g_update<<<grid, kThreads, 0, st>>>(col(1), col(0), nullptr, al(0), be(0), w->chunks, nch,
	                                      w->active, w->partial);
	k_g_finish<<<S, kThreads, 0, st>>>(w->partial, w->seg_chunk, w->active, be(1), 1);
	k_g_scale<<<grid, kThreads, 0, st>>>(col(1), col(1), be(1), 1, w->chunks, nch, w->active);

	std::vector<size_t> j_stop(size_t(S), 0);
	int                 n_active = S;
	for (int s = 0; s < S; ++s)
		if (skip[size_t(s)]) {
			--n_active;
		} else if (maxn_s[size_t(s)] == 1) { // nothing to iterate: the 1 x 1 tridiagonal
			act[size_t(s)] = 0;
			--n_active;
		}
	if (n_active < S
	    && (e = cudaMemcpyAsync(w->active, act.data(), size_t(S) * sizeof(int), cudaMemcpyHostToDevice, st)))
		return status(h, e, "update active sectors");
	const size_t nsc = size_t(S) * size_t(cols);
	std::vector<double> eold(size_t(S) * p->eigs_for_stop, 0.0);
	auto enqueue_group = [&](size_t j0, size_t j1) -> int {
		for (size_t jj = j0; jj < j1; ++jj) {
			double* v0 = col(jj - 1);
			double* v1 = col(jj);
			double* v2 = col(jj + 1);
			if (int rc = kron_apply_device(h, v1, v2))
				return rc;
			dot(v2, v1, al(jj), 0);
			k_g_update<<<grid, kThreads, 0, st>>>(v2, v1, v0, al(jj), be(jj), w->chunks, nch,
			                                      w->active, w->partial);
			k_g_finish<<<S, kThreads, 0, st>>>(w->partial, w->seg_chunk, w->active, be(jj + 1), 1);
			k_g_scale<<<grid, kThreads, 0, st>>>(v2, v2, be(jj + 1), 1, w->chunks, nch, w->active);
			if (p->reortho) { // reorthoIfNecessary (LanczosVectors.h:243-271)
				const int nc = int(jj) + 1;
				k_g_basis_dots<<<grid, kThreads, 0, st>>>(w->V, D, nc, v2, w->chunks, nch,
				                                          w->active, w->partial, ldp);
				k_g_basis_reduce<<<S, kThreads, 0, st>>>(w->partial, ldp, nc, w->seg_chunk,
				                                         w->active, w->r);
				k_g_basis_subtract<<<grid, kThreads, 0, st>>>(v2, w->V, D, nc, w->r, ldp, w->chunks,
				                                              nch, w->active, w->partial);
				k_g_finish<<<S, kThreads, 0, st>>>(w->partial, w->seg_chunk, w->active, nrm, 1);
				k_g_scale<<<grid, kThreads, 0, st>>>(v2, v2, nrm, 1, w->chunks, nch, w->active);
			}
		}
		return DMRGPP_OK;
	};
	// Groups of steps are enqueued one group ahead of the host's stopping test
	// (two pinned copies of alpha/beta alternate), so the GPU runs the next
	// group while the host tests the last one.  A group never passes the last
	// step of a sector that is still active when it is enqueued.
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
			return status(h, e, "events");
	const size_t hstride = 2 * nsc + size_t(S);
	struct Group {
		size_t j0, j1;
		int    buf;
	};
	std::vector<Group>  inflight;
	std::vector<double> d, off;
	size_t              next = 1;
	int                 buf  = 0;
	for (;;) {
		while (inflight.size() < 2 && n_active > 0 && next < maxn) {
			size_t cap = maxn;
			for (int s = 0; s < S; ++s)
				if (act[size_t(s)])
					cap = std::min(cap, maxn_s[size_t(s)]);
			if (cap <= next)
				break; // a sector ends here: test before going on
			const size_t jend = std::min(cap, next + size_t(p->check_every));
			if (int rc = enqueue_group(next, jend))
				return rc;
			if ((e = cudaGetLastError()))
				return status(h, e, "group Lanczos launch");
			double* hb = w->host + size_t(buf) * hstride;
			if ((e = cudaMemcpyAsync(hb, w->alpha, nsc * sizeof(double), cudaMemcpyDeviceToHost, st))
			    || (e = cudaMemcpyAsync(hb + nsc, w->beta, (nsc + size_t(S)) * sizeof(double),
			                            cudaMemcpyDeviceToHost, st))
			    || (e = cudaEventRecord(events.ev[buf], st)))
				return status(h, e, "read alpha/beta");
			inflight.push_back({ next, jend, buf });
			next = jend;
			buf ^= 1;
		}
		if (inflight.empty())
			break;
		const Group g = inflight.front();
		inflight.erase(inflight.begin());
		if ((e = cudaEventSynchronize(events.ev[g.buf])))
			return status(h, e, "group Lanczos steps");
		if (h->err_host && *reinterpret_cast<volatile int*>(h->err_host))
			return handle_fail(h, DMRGPP_TIMEOUT, "H*x kernel wait gave up during the group Lanczos");
		const double* ah = w->host + size_t(g.buf) * hstride;
		const double* bh = ah + nsc;
		bool          changed = false;
		for (int s = 0; s < S; ++s) {
			if (!act[size_t(s)])
				continue;
			// steps up to g.j1 - 1 are done; test at the last one
			const size_t jj   = g.j1 - 1;
			const size_t n    = jj + 1;
			const size_t ne   = std::min(p->eigs_for_stop, n);
			double       dmax = 0.0;
			for (size_t rep = 0; rep < 2; ++rep) { // Ritz values at steps jj - 1 and jj
				const size_t nn = rep == 0 ? n - 1 : n;
				if (nn == 0)
					continue;
				d.resize(nn);
				off.resize(nn);
				for (size_t q = 0; q < nn; ++q) {
					d[q]   = ah[q * size_t(S) + size_t(s)];
					off[q] = bh[(q + 1) * size_t(S) + size_t(s)];
				}
				for (size_t k = 0; k < std::min(ne, nn); ++k) {
					const double th = tridiag_kth_lowest(int(nn), d.data(), off.data(), int(k) + 1);
					if (rep == 1)
						dmax = std::max(dmax, std::fabs(th - eold[size_t(s) * p->eigs_for_stop + k]));
					eold[size_t(s) * p->eigs_for_stop + k] = th;
				}
			}
			const bool last = jj == maxn_s[size_t(s)] - 1;
			if ((dmax < p->tolerance && jj >= p->min_steps) || last) {
				j_stop[size_t(s)] = jj;
				act[size_t(s)]    = 0;
				--n_active;
				changed = true;
			}
		}
		if (changed
		    && (e = cudaMemcpyAsync(w->active, act.data(), size_t(S) * sizeof(int), cudaMemcpyHostToDevice, st)))
			return status(h, e, "update active sectors");
	}
	for (int s = 0; s < S; ++s)
		if (act[size_t(s)])
			j_stop[size_t(s)] = maxn_s[size_t(s)] - 1;
	// final scalars: entries up to each sector's stopping step no longer change
	if ((e = cudaStreamSynchronize(st))
	    || (e = dmrgpp::download_sync(w->host, w->alpha, nsc * sizeof(double), h->stream))
	    || (e = dmrgpp::download_sync(w->host + nsc, w->beta, (nsc + size_t(S)) * sizeof(double), h->stream)))
		return status(h, e, "read alpha/beta");

	// Ritz pairs per sector (LanczosSolver.h:76-84): lowest eigenvalue of the
	// (j_stop + 1)-dimensional tridiagonal and its eigenvector
	const double*       ah = w->host;
	const double*       bh = w->host + nsc;
	// sector s's coefficients at s * ldp: the layout of w->r, whose row length
	// is that of the (possibly larger) work buffers kept from an earlier solve
	const size_t        ncoef = size_t(S) * size_t(ldp);
	std::vector<double> coef(ncoef, 0.0);
	std::vector<int>    ncols(static_cast<size_t>(S));
	for (int s = 0; s < S; ++s) {
		if (skip[size_t(s)]) { // no part in this solve: no coefficients, z = 0 there
			energies[s]      = std::numeric_limits<double>::quiet_NaN();
			ncols[size_t(s)] = 0;
			if (steps_taken)
				steps_taken[s] = 0;
			continue;
		}
		const size_t n = j_stop[size_t(s)] + 1;
		d.resize(n);
		off.resize(n);
		for (size_t q = 0; q < n; ++q) {
			d[q]   = ah[q * size_t(S) + size_t(s)];
			off[q] = bh[(q + 1) * size_t(S) + size_t(s)];
		}
		energies[s] = tridiag_kth_lowest(int(n), d.data(), off.data(), 1);
		tridiag_inverse_iteration(int(n), d.data(), off.data(), energies[s],
		                          coef.data() + size_t(s) * size_t(ldp));
		ncols[size_t(s)] = int(n);
		if (steps_taken)
			steps_taken[s] = j_stop[size_t(s)];
	}
	if ((e = cudaMemcpyAsync(w->r, coef.data(), ncoef * sizeof(double), cudaMemcpyHostToDevice, st))
	    || (e = cudaMemcpyAsync(w->ncols, ncols.data(), size_t(S) * sizeof(int), cudaMemcpyHostToDevice, st)))
		return status(h, e, "upload Ritz coefficients");
	k_g_basis_combine<<<grid, kThreads, 0, st>>>(w->z, w->V, D, w->ncols, w->r, ldp, w->chunks, nch,
	                                             nullptr);
	if ((e = cudaMemcpyAsync(z, w->z, D * sizeof(double),
	                         on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st))
	    || (e = cudaStreamSynchronize(st)))
		return status(h, e, "Ritz vectors");
	return DMRGPP_OK;
}

// ---------------------------------------------------------------------------
// FP64 refinement of every sector of a group handle: the outer iteration of
// dmrgpp_refine_lowest (lanczos.cu) per sector, all sectors in lockstep.  Each
// outer step normalises psi, forms the FP64 Rayleigh quotients and residuals
// with one FP64 group H*x, and solves every unconverged sector's projected
// correction equation (I - psi psi^T)(H - theta)(I - psi psi^T) t = -r by
// conjugate gradients whose matvecs are the handle's (mixed) group launches;
// the per-sector CG scalars live on the device and a sector's CG stops on the
// device (converged, or a non-positive pAp), so the host reads one flag array
// per burst of 8 iterations.  No counterpart in the reference.
// ---------------------------------------------------------------------------
extern "C" int dmrgpp_refine_lowest_group(dmrgpp_kron_handle h, double* psi, int max_outer,
                                          double tolerance, int inner_iterations,
                                          double inner_tolerance, double* energies, int* converged,
                                          dmrgpp_refine_stats* stats)
{
	DMRGPP_TRACE("dmrgpp_refine_lowest_group");
	if (h && h->complex_sector)
		return dmrgpp::handle_fail(h, DMRGPP_NOT_SUPPORTED, "the device eigensolvers take real sectors");
	using namespace dmrgpp;
	if (!h)
		return DMRGPP_INVALID_ARG;
	if (!psi || !energies)
		return handle_fail(h, DMRGPP_INVALID_ARG, "null argument");
	if (max_outer < 0 || inner_iterations < 1)
		return handle_fail(h, DMRGPP_INVALID_ARG, "max_outer must be >= 0 and inner_iterations >= 1");
	const int    S = int(h->sector_start.size()) - 1;
	const size_t D = size_t(h->plan.dim());

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

	if (int rc = ensure_group_work(h, 1))
		return rc;
	GroupWork*         w  = h->group;
	const cudaStream_t st = h->stream;
	cudaError_t        e;
	if (!w->rv) {
		if ((e = dmrgpp::dev_malloc(&w->rv, 7 * D * sizeof(double)))
		    || (e = dmrgpp::dev_malloc(&w->rsc, 8 * size_t(S) * sizeof(double)))
		    || (e = dmrgpp::dev_malloc(&w->rpsc, 6 * size_t(S) * sizeof(double)))
		    || (e = dmrgpp::dev_malloc(&w->rpart, 3 * size_t(std::max(w->nch, 1)) * sizeof(double)))
		    || (e = dmrgpp::dev_malloc(&w->rint, 2 * size_t(S) * sizeof(int)))
		    || (e = cudaHostAlloc(&w->rhost, 2 * size_t(S) * (sizeof(double) + sizeof(int)), 0)))
			return status(h, e, "group refinement allocation");
	}
	const int nch   = w->nch;
	const int grid  = std::max(1, std::min(nch, kGrid));
	const int sgrid = (S + kThreads - 1) / kThreads;
	double*   hpsi  = w->rv;
	double*   r     = w->rv + D;
	double*   t     = w->rv + 2 * D;
	double*   res   = w->rv + 3 * D;
	double*   pv    = w->rv + 4 * D;
	double*   Aq    = w->rv + 5 * D;
	double*   theta = w->rsc;
	double*   rnorm = w->rsc + S;
	double*   nrm   = w->rsc + 2 * S;
	double*   ua    = w->rsc + 3 * S;
	double*   pAp   = w->rsc + 4 * S;
	double*   rr[2] = { w->rsc + 5 * S, w->rsc + 6 * S };
	double*   b0    = w->rsc + 7 * S;
	int*      outer = w->rint;
	int*      cg    = w->rint + S;
	double*   th_h  = w->rhost;
	double*   rn_h  = w->rhost + S;
	int*      cg_h  = reinterpret_cast<int*>(w->rhost + 2 * S);

	auto dot = [&](const double* x, const double* y, double* out, const int* act, int root) {
		k_g_dot<<<grid, kThreads, 0, st>>>(x, y, w->chunks, nch, act, w->partial);
		k_g_finish<<<S, kThreads, 0, st>>>(w->partial, w->seg_chunk, act, out, root);
	};
	// Jacobi corrections (dmrgpp_set_correction_preconditioner)
	const bool jac  = h->correction_precond == DMRGPP_PRECOND_JACOBI && h->d_diag;
	double*    wv   = w->rv + 6 * D;
	double*    uw   = w->rpsc;
	double*    sums = w->rpsc + S; // 3 x S
	double*    rho[2] = { w->rpsc + 4 * S, w->rpsc + 5 * S };
	auto pcg_sums = [&]() {
		k_g_pcg_sums<<<grid, kThreads, 0, st>>>(res, h->d_diag, theta, psi, wv, w->chunks, nch, cg, w->rpart);
		for (int q = 0; q < 3; ++q)
			k_g_finish<<<S, kThreads, 0, st>>>(w->rpart + size_t(q) * nch, w->seg_chunk, cg, sums + size_t(q) * S, 0);
	};
	// the FP64 group H*x skips converged sectors while this runs
	struct MaskOff {
		dmrgpp_kron_handle h;
		int                user;
		~MaskOff()
		{
			h->sector_active = nullptr;
			h->precision     = user;
		}
	} mask_off { h, h->precision };

	std::vector<int> act(size_t(S), 1), done(size_t(S), 0), stall(size_t(S), 0);
	std::vector<double> th(size_t(S), 0.0), rn(size_t(S), 0.0),
	    best(size_t(S), std::numeric_limits<double>::infinity());
	if ((e = cudaMemcpyAsync(outer, act.data(), size_t(S) * sizeof(int), cudaMemcpyHostToDevice, st)))
		return status(h, e, "group refinement start");
	dmrgpp_refine_stats s {};
	int                 n_active = S;
	for (int it = 0; it <= max_outer && n_active > 0; ++it) {
		// normalise, FP64 Rayleigh quotients and residuals of the active sectors
		dot(psi, psi, nrm, outer, 0);
		k_g_scale<<<grid, kThreads, 0, st>>>(psi, psi, nrm, 0, w->chunks, nch, outer);
		h->precision     = DMRGPP_FP64;
		h->sector_active = outer;
		int rc           = kron_apply_device(h, psi, hpsi);
		h->precision     = mask_off.user;
		h->sector_active = nullptr;
		if (rc)
			return rc;
		++s.fp64_matvecs;
		dot(psi, hpsi, theta, outer, 0);
		k_g_residual<<<grid, kThreads, 0, st>>>(hpsi, psi, theta, r, w->chunks, nch, outer, w->partial);
		k_g_finish<<<S, kThreads, 0, st>>>(w->partial, w->seg_chunk, outer, rnorm, 1);
		if ((e = cudaMemcpyAsync(th_h, theta, 2 * size_t(S) * sizeof(double), cudaMemcpyDeviceToHost, st))
		    || (e = cudaStreamSynchronize(st)))
			return status(h, e, "group refinement Rayleigh quotients");
		if (h->err_host && *reinterpret_cast<volatile int*>(h->err_host))
			return handle_fail(h, DMRGPP_TIMEOUT, "H*x kernel wait gave up during the group refinement");
		bool changed = false;
		for (int q = 0; q < S; ++q) {
			if (!act[size_t(q)])
				continue;
			th[size_t(q)] = th_h[q];
			rn[size_t(q)] = rn_h[q];
			if (rn_h[q] <= tolerance * std::max(1.0, std::fabs(th_h[q]))) {
				act[size_t(q)]  = 0;
				done[size_t(q)] = 1;
				--n_active;
				changed = true;
				continue;
			}
			// a sector whose residual has not halved over two outer steps
			// is failing (its start lies above the first excitation, where
			// the projected correction equation is indefinite): it stops
			// here, unconverged, instead of holding the lockstep launches
			if (rn_h[q] < 0.5 * best[size_t(q)]) {
				best[size_t(q)]  = rn_h[q];
				stall[size_t(q)] = 0;
			} else if (++stall[size_t(q)] >= 2) {
				act[size_t(q)] = 0;
				--n_active;
				changed = true;
			}
		}
		s.outer_iterations = size_t(it);
		if (n_active == 0 || it == max_outer)
			break;
		if (changed
		    && (e = cudaMemcpyAsync(outer, act.data(), size_t(S) * sizeof(int), cudaMemcpyHostToDevice, st)))
			return status(h, e, "group refinement update");
		// correction solves: t = 0, res = -(I - psi psi^T) r, p = res
		if ((e = cudaMemsetAsync(t, 0, D * sizeof(double), st))
		    || (e = cudaMemsetAsync(res, 0, D * sizeof(double), st)))
			return status(h, e, "group refinement clear");
		k_g_axpy<<<grid, kThreads, 0, st>>>(res, r, nullptr, -1.0, w->chunks, nch, outer);
		dot(psi, res, ua, outer, 0);
		k_g_axpy<<<grid, kThreads, 0, st>>>(res, psi, ua, -1.0, w->chunks, nch, outer);
		if ((e = cudaMemcpyAsync(pv, res, D * sizeof(double), cudaMemcpyDeviceToDevice, st)))
			return status(h, e, "group refinement copy");
		k_g_dot<<<grid, kThreads, 0, st>>>(res, res, w->chunks, nch, outer, w->partial);
		k_g_finish<<<S, kThreads, 0, st>>>(w->partial, w->seg_chunk, outer, rr[0], 0);
		k_g_finish<<<S, kThreads, 0, st>>>(w->partial, w->seg_chunk, outer, b0, 1);
		k_g_cg_start<<<sgrid, kThreads, 0, st>>>(b0, outer, cg, S);
		if (jac) { // Jacobi: wv = K^-1 psi, <psi, wv>, then p = z0 and rho0 = <res, z0>
			k_g_pcg_setup<<<grid, kThreads, 0, st>>>(psi, h->d_diag, theta, wv, w->chunks, nch, cg, w->rpart);
			k_g_finish<<<S, kThreads, 0, st>>>(w->rpart, w->seg_chunk, cg, uw, 0);
			pcg_sums();
			// first = 1: rho is not read, the other half of its double buffer stands in
			k_g_pcg_direction<<<grid, kThreads, 0, st>>>(pv, res, h->d_diag, theta, wv, uw, sums, S, rho[1],
			                                             rho[0], 1, w->chunks, nch, w->seg_chunk, cg);
		}
		int cur = 0, inner = 0;
		while (inner < inner_iterations) {
			const int burst = std::min(8, inner_iterations - inner);
			for (int q = 0; q < burst; ++q, ++inner) {
				// Aq = P (H - theta) p
				h->sector_active = cg;
				rc               = kron_apply_device(h, pv, Aq);
				h->sector_active = nullptr;
				if (rc)
					return rc;
				++s.inner_matvecs;
				k_g_axpy<<<grid, kThreads, 0, st>>>(Aq, pv, theta, -1.0, w->chunks, nch, cg);
				dot(psi, Aq, ua, cg, 0);
				k_g_axpy<<<grid, kThreads, 0, st>>>(Aq, psi, ua, -1.0, w->chunks, nch, cg);
				dot(pv, Aq, pAp, cg, 0);
				// alpha = rr / pAp (plain) or rho / pAp (Jacobi); |res|^2 for the check
				k_g_cg_update<<<grid, kThreads, 0, st>>>(t, res, pv, Aq, jac ? rho[cur] : rr[cur], pAp,
				                                         w->chunks, nch, cg, w->partial);
				k_g_finish<<<S, kThreads, 0, st>>>(w->partial, w->seg_chunk, cg, rr[cur ^ 1], 0);
				k_g_cg_check<<<sgrid, kThreads, 0, st>>>(pAp, rr[cur ^ 1], b0, inner_tolerance, cg, S);
				if (jac) {
					pcg_sums();
					k_g_pcg_direction<<<grid, kThreads, 0, st>>>(pv, res, h->d_diag, theta, wv, uw, sums, S,
					                                             rho[cur], rho[cur ^ 1], 0, w->chunks, nch,
					                                             w->seg_chunk, cg);
				} else {
					k_g_cg_direction<<<grid, kThreads, 0, st>>>(pv, res, rr[cur ^ 1], rr[cur], w->chunks, nch,
					                                            cg);
				}
				cur ^= 1;
			}
			if ((e = cudaGetLastError()))
				return status(h, e, "group refinement launch");
			if ((e = cudaMemcpyAsync(cg_h, cg, size_t(S) * sizeof(int), cudaMemcpyDeviceToHost, st))
			    || (e = cudaStreamSynchronize(st)))
				return status(h, e, "group refinement correction solves");
			bool any = false;
			for (int q = 0; q < S && !any; ++q)
				any = cg_h[q] != 0;
			if (!any)
				break;
		}
		// psi += t (t = 0 outside the active sectors)
		k_g_axpy<<<grid, kThreads, 0, st>>>(psi, t, nullptr, 1.0, w->chunks, nch, outer);
	}
	if ((e = cudaStreamSynchronize(st)))
		return status(h, e, "group refinement");
	s.converged = 1;
	for (int q = 0; q < S; ++q) {
		energies[q] = th[size_t(q)];
		if (converged)
			converged[q] = done[size_t(q)];
		s.residual_norm = std::max(s.residual_norm, rn[size_t(q)]);
		if (!done[size_t(q)])
			s.converged = 0;
	}
	if (stats)
		*stats = s;
	return s.converged ? DMRGPP_OK
	                   : handle_fail(h, DMRGPP_NOT_CONVERGED, "group refinement: a sector did not converge");
}

// ---------------------------------------------------------------------------
// Davidson for every sector of a group handle, all sectors in lockstep: the
// iteration of dmrgpp_davidson_lowest (lanczos.cu) per sector with the
// handle's matvecs.  Every iteration orthonormalises each active sector's
// correction against its basis (two classical Gram-Schmidt passes), applies H
// to the new columns of all sectors in one group launch, adds a column to
// each sector's projected matrix (read to the host), takes the lowest Ritz
// pair of every sector on the host, forms the Ritz vectors, residuals and
// their norms on the device, stops the sectors whose residual met the
// tolerance, and forms the next corrections (none, Jacobi, or the learned
// one with each sector's own Ritz value and residual norm).  Since every
// active sector adds one column per iteration, all restart together.  No
// counterpart in the reference.
// ---------------------------------------------------------------------------
extern "C" int dmrgpp_davidson_lowest_group(dmrgpp_kron_handle h, const dmrgpp_davidson_params* p,
                                            const double* init, int on_device, double* energies,
                                            double* z, int* converged, dmrgpp_davidson_stats* stats)
{
	DMRGPP_TRACE("dmrgpp_davidson_lowest_group");
	if (h && h->complex_sector)
		return dmrgpp::handle_fail(h, DMRGPP_NOT_SUPPORTED, "the device eigensolvers take real sectors");
	using namespace dmrgpp;
	if (!h)
		return DMRGPP_INVALID_ARG;
	if (!p || !init || !energies || !z)
		return handle_fail(h, DMRGPP_INVALID_ARG, "null argument");
	if (p->max_subspace < 2 || p->max_subspace > 128 || p->max_iterations < 1)
		return handle_fail(h, DMRGPP_INVALID_ARG, "max_subspace must be in [2, 128] for a group");
	if (p->preconditioner == DMRGPP_PRECOND_MLP && !p->mlp)
		return handle_fail(h, DMRGPP_INVALID_ARG, "learned preconditioner selected without a network");
	const int    S    = int(h->sector_start.size()) - 1;
	const size_t D    = size_t(h->plan.dim());
	const int    mmax = int(p->max_subspace);

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

	if (int rc = ensure_group_work(h, mmax))
		return rc;
	GroupWork*         w  = h->group;
	const cudaStream_t st = h->stream;
	cudaError_t        e;
	const int          ldp = w->cols;
	if (w->dmax < mmax) {
		dmrgpp::dev_free(w->dV);
		dmrgpp::dev_free(w->dW);
		w->dV = w->dW = nullptr;
		w->dmax       = 0;
		if ((e = dmrgpp::dev_malloc(&w->dV, D * size_t(mmax) * sizeof(double)))
		    || (e = dmrgpp::dev_malloc(&w->dW, D * size_t(mmax) * sizeof(double))))
			return status(h, e, "group Davidson basis allocation");
		w->dmax = mmax;
	}
	if (!w->dvec
	    && ((e = dmrgpp::dev_malloc(&w->dvec, 4 * D * sizeof(double)))
	        || (e = dmrgpp::dev_malloc(&w->dsc, 3 * size_t(S) * sizeof(double)))
	        || (e = dmrgpp::dev_malloc(&w->dcoef, size_t(S) * size_t(ldp) * sizeof(double)))))
		return status(h, e, "group Davidson allocation");
	const int nch  = w->nch;
	const int grid = std::max(1, std::min(nch, kGrid));
	auto      Vc   = [&](int c) { return w->dV + size_t(c) * D; };
	auto      Wc   = [&](int c) { return w->dW + size_t(c) * D; };
	double*   u    = w->dvec;
	double*   hu   = w->dvec + D;
	double*   r    = w->dvec + 2 * D;
	double*   t    = w->dvec + 3 * D;
	double*   th_d = w->dsc;
	double*   rn_d = w->dsc + S;
	double*   nrm  = w->dsc + 2 * S;
	double*   hbuf = w->host; // pinned, at least 2 * nseg * cols doubles

	// the group H*x skips converged sectors while this runs
	h->sector_active = w->active;
	struct MaskOff {
		dmrgpp_kron_handle h;
		~MaskOff() { h->sector_active = nullptr; }
	} mask_off { h };

	std::vector<int> act(size_t(S), 1), done(size_t(S), 0);
	std::vector<long long> dim_s(static_cast<size_t>(S));
	for (int q = 0; q < S; ++q)
		dim_s[size_t(q)] = h->sector_start[size_t(q) + 1] - h->sector_start[size_t(q)];
	if ((e = cudaMemcpyAsync(w->active, act.data(), size_t(S) * sizeof(int), cudaMemcpyHostToDevice, st))
	    || (e = cudaMemcpyAsync(t, init, D * sizeof(double),
	                            on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st)))
		return status(h, e, "group Davidson start");

	const size_t        mm = size_t(mmax);
	std::vector<double> G(size_t(S) * mm * mm, 0.0);
	std::vector<double> th(size_t(S), 0.0), rn(size_t(S), 0.0), coef(size_t(S) * size_t(ldp), 0.0);
	std::vector<int>    ncols(size_t(S), 0);
	dmrgpp_davidson_stats s {};
	const bool          mixed    = h->precision != DMRGPP_FP64;
	int                 n_active = S;
	int                 k        = 0;
	auto dot = [&](const double* x, const double* y, double* out) {
		k_g_dot<<<grid, kThreads, 0, st>>>(x, y, w->chunks, nch, w->active, w->partial);
		k_g_finish<<<S, kThreads, 0, st>>>(w->partial, w->seg_chunk, w->active, out, 0);
	};
	for (size_t it = 0; it < p->max_iterations && n_active > 0; ++it) {
		// orthonormalise the corrections against the bases and append them
		for (int pass = 0; pass < (k > 0 ? 2 : 0); ++pass) {
			k_g_basis_dots<<<grid, kThreads, 0, st>>>(w->dV, D, k, t, w->chunks, nch, w->active,
			                                          w->partial, ldp);
			k_g_basis_reduce<<<S, kThreads, 0, st>>>(w->partial, ldp, k, w->seg_chunk, w->active, w->r);
			k_g_basis_subtract<<<grid, kThreads, 0, st>>>(t, w->dV, D, k, w->r, ldp, w->chunks, nch,
			                                              w->active, w->partial);
		}
		if (k == 0)
			dot(t, t, nrm);
		else
			k_g_finish<<<S, kThreads, 0, st>>>(w->partial, w->seg_chunk, w->active, nrm, 0);
		k_g_scale<<<grid, kThreads, 0, st>>>(t, Vc(k), nrm, 0, w->chunks, nch, w->active);
		if (int rc = kron_apply_device(h, Vc(k), Wc(k)))
			return rc;
		if (mixed)
			++s.mixed_matvecs;
		else
			++s.fp64_matvecs;
		// new column of every sector's projected matrix
		k_g_basis_dots<<<grid, kThreads, 0, st>>>(w->dV, D, k + 1, Wc(k), w->chunks, nch, w->active,
		                                          w->partial, ldp);
		k_g_basis_reduce<<<S, kThreads, 0, st>>>(w->partial, ldp, k + 1, w->seg_chunk, w->active, w->r);
		if ((e = cudaMemcpyAsync(hbuf, w->r, size_t(S) * size_t(ldp) * sizeof(double),
		                         cudaMemcpyDeviceToHost, st))
		    || (e = cudaStreamSynchronize(st)))
			return status(h, e, "group Davidson projection");
		if (h->err_host && *reinterpret_cast<volatile int*>(h->err_host))
			return handle_fail(h, DMRGPP_TIMEOUT, "H*x kernel wait gave up during the group Davidson");
		// Rayleigh-Ritz per active sector
		for (int q = 0; q < S; ++q) {
			if (!act[size_t(q)])
				continue;
			double*       Gq  = G.data() + size_t(q) * mm * mm;
			const double* col = hbuf + size_t(q) * size_t(ldp);
			for (int i = 0; i <= k; ++i) {
				Gq[size_t(i) + size_t(k) * mm] = col[i];
				Gq[size_t(k) + size_t(i) * mm] = col[i];
			}
		}
		++k;
		// lowest pair of every active sector's k x k projected matrix, on the
		// host's cores (each sector writes only its own entries)
		parallel_for(size_t(S), [&](size_t q) {
			if (!act[q])
				return;
			const double*       Gq = G.data() + q * mm * mm;
			std::vector<double> Gk(size_t(k) * size_t(k));
			for (int j = 0; j < k; ++j)
				for (int i = 0; i < k; ++i)
					Gk[size_t(i) + size_t(j) * size_t(k)] = Gq[size_t(i) + size_t(j) * mm];
			sym_lowest(k, Gk.data(), &th[q], coef.data() + q * size_t(ldp));
			ncols[q] = k;
		});
		if ((e = cudaMemcpyAsync(w->dcoef, coef.data(), coef.size() * sizeof(double), cudaMemcpyHostToDevice, st))
		    || (e = cudaMemcpyAsync(th_d, th.data(), size_t(S) * sizeof(double), cudaMemcpyHostToDevice, st))
		    || (e = cudaMemcpyAsync(w->ncols, ncols.data(), size_t(S) * sizeof(int), cudaMemcpyHostToDevice, st)))
			return status(h, e, "group Davidson Ritz coefficients");
		k_g_basis_combine<<<grid, kThreads, 0, st>>>(u, w->dV, D, w->ncols, w->dcoef, ldp, w->chunks, nch,
		                                             w->active);
		k_g_basis_combine<<<grid, kThreads, 0, st>>>(hu, w->dW, D, w->ncols, w->dcoef, ldp, w->chunks, nch,
		                                             w->active);
		k_g_residual<<<grid, kThreads, 0, st>>>(hu, u, th_d, r, w->chunks, nch, w->active, w->partial);
		k_g_finish<<<S, kThreads, 0, st>>>(w->partial, w->seg_chunk, w->active, rn_d, 1);
		if ((e = cudaMemcpyAsync(hbuf, rn_d, size_t(S) * sizeof(double), cudaMemcpyDeviceToHost, st))
		    || (e = cudaStreamSynchronize(st)))
			return status(h, e, "group Davidson residuals");
		++s.iterations;
		bool changed = false;
		for (int q = 0; q < S; ++q) {
			if (!act[size_t(q)])
				continue;
			rn[size_t(q)] = hbuf[q];
			// converged, or the basis spans the whole sector (the pair is exact)
			if (hbuf[q] <= p->tolerance * std::max(1.0, std::fabs(th[size_t(q)])) || k >= dim_s[size_t(q)]) {
				act[size_t(q)]  = 0;
				done[size_t(q)] = 1;
				--n_active;
				changed = true;
			}
		}
		if (n_active == 0)
			break;
		if (changed
		    && (e = cudaMemcpyAsync(w->active, act.data(), size_t(S) * sizeof(int), cudaMemcpyHostToDevice, st)))
			return status(h, e, "group Davidson update");
		if (k == mmax) {
			// restart every active sector from its Ritz pair: V = [u], W = [H u]
			dot(u, u, nrm);
			k_g_scale<<<grid, kThreads, 0, st>>>(u, Vc(0), nrm, 0, w->chunks, nch, w->active);
			k_g_scale<<<grid, kThreads, 0, st>>>(hu, Wc(0), nrm, 0, w->chunks, nch, w->active);
			for (int q = 0; q < S; ++q)
				if (act[size_t(q)])
					G[size_t(q) * mm * mm] = th[size_t(q)];
			k = 1;
			++s.restarts;
		}
		// corrections
		if (p->preconditioner == DMRGPP_PRECOND_JACOBI) {
			k_g_jacobi<<<grid, kThreads, 0, st>>>(r, h->d_diag, th_d, p->denominator_floor, t, w->chunks, nch,
			                                      w->active);
		} else if (p->preconditioner == DMRGPP_PRECOND_MLP) {
			if (int rc = mlp_precondition_group(static_cast<dmrgpp_mlp_handle>(p->mlp), h->d_diag, r,
			                                    w->sec_start, th_d, rn_d, S, t, D, st))
				return handle_fail(h, rc, "learned preconditioner failed");
		} else if ((e = cudaMemcpyAsync(t, r, D * sizeof(double), cudaMemcpyDeviceToDevice, st))) {
			return status(h, e, "group Davidson correction");
		}
		if ((e = cudaGetLastError()))
			return status(h, e, "group Davidson launch");
	}
	// the Ritz vectors are normalised by construction (orthonormal bases, unit coefficients)
	if ((e = cudaMemcpyAsync(z, u, D * sizeof(double), on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
	                         st))
	    || (e = cudaStreamSynchronize(st)))
		return status(h, e, "group Davidson Ritz vectors");
	s.converged = 1;
	for (int q = 0; q < S; ++q) {
		energies[q] = th[size_t(q)];
		if (converged)
			converged[q] = done[size_t(q)];
		s.residual_norm = std::max(s.residual_norm, rn[size_t(q)]);
		if (!done[size_t(q)])
			s.converged = 0;
	}
	if (stats)
		*stats = s;
	return s.converged ? DMRGPP_OK
	                   : handle_fail(h, DMRGPP_NOT_CONVERGED, "group Davidson: a sector did not converge");
}
