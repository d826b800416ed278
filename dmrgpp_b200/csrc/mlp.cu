// Learned Davidson preconditioner: a small MLP trained on the GPU by the
// project's own forward and backward kernels (no counterpart in the
// reference, which has no Davidson solver).
//
// Per element e of a sector vector, with s = max(1, |theta|),
// rms = |r| / sqrt(n), f0 = (d_e - theta)/s, f1 = r_e / rms:
//   features x_e = [f0, f1, f1 f0 / (f0^2 + 0.05^2), 1 / (1 + (f0 / 0.05)^2)]
//   h1 = tanh(W1 x + b1), h2 = tanh(W2 h1 + b2), o = w3 . h2 + b3
//   correction t_e = o * rms / s
// (the third feature makes the diagonal (Jacobi) correction -r/(d-theta) a
// linear function of the inputs).  Training minimises the mean squared error
// between o and the scaled exact correction t*_e * s / rms.
//
// Parameters are kept in FP32 (master copy, Adam state).  Training runs its
// contractions in one tiled FP32 GEMM kernel whose reduction order is fixed,
// so it is bitwise reproducible.  Inference (the preconditioner applied in
// a solve) uses BF16 copies of the weights with FP32 accumulation, by
// default in one fused tcgen05 kernel (mlp_infer_tc_kernel):
//   per tile of 128 elements, 4 warps compute the features and layer 1 on
//   the CUDA cores and write h1 as BF16 into a ring of 64-unit chunks in the
//   128-byte-swizzled K-major layout; one thread issues the layer-2 MMAs
//   (kind::f16, BF16 x BF16 -> FP32, M = 128, N = 256, K = 16) against W2
//   kept in shared memory for the whole launch, into one of two TMEM
//   accumulators (2 x 256 columns); 4 epilogue warps read the accumulator
//   row by row (tcgen05.ld), apply bias and tanh and reduce with w3.
// The per-element work is 2 x 256 tanh and 66k MACs, so the fused kernel is
// bound by the tanh (SFU) throughput, not by the tensor cores or HBM.
// The earlier CUDA-core inference (BF16 weights widened to FP32, h1 kept in
// FP32) stays selectable (dmrgpp_mlp_set_inference).
#include "devmem.h"
#include "trace.h"
#include "dmrgpp_kron.h"
#include "mlp.h"
#include "tc_common.cuh"

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

namespace dmrgpp {
namespace {

constexpr int   F  = kMlpFeatures;
constexpr int   H  = kMlpWidth;
constexpr float kDelta = 0.05f;

// parameter offsets (floats)
constexpr size_t kW1 = 0;
constexpr size_t kB1 = kW1 + size_t(H) * F;
constexpr size_t kW2 = kB1 + H;
constexpr size_t kB2 = kW2 + size_t(H) * H;
constexpr size_t kW3 = kB2 + H;
constexpr size_t kB3 = kW3 + H;
constexpr size_t kNumParams = kB3 + 1;

} // namespace
} // namespace dmrgpp

struct dmrgpp_mlp_s {
	int            device  = 0;
	float*         params  = nullptr; // FP32 master
	float*         grads   = nullptr;
	float*         adam_m  = nullptr;
	float*         adam_v  = nullptr;
	int            adam_t  = 0;
	__nv_bfloat16* wbf     = nullptr; // BF16 copy of all parameters (inference)
	float*         pinf    = nullptr; // the BF16 copy widened to FP32
	bool           bf_dirty = true;
	int            cap     = 0;       // rows of the training / inference buffers
	float*         x       = nullptr; // cap x F
	float*         h1      = nullptr; // cap x H
	float*         h2      = nullptr; // cap x H
	float*         out     = nullptr; // cap
	float*         gout    = nullptr; // cap
	float*         dz      = nullptr; // cap x H
	float*         dz1     = nullptr; // cap x H
	double*        loss    = nullptr; // device scalar
	double*        partial = nullptr;
	unsigned*      ctr     = nullptr;
	int            last_rows = 0;
	int            inference = DMRGPP_MLP_TENSOR_CORES;
	int*           err_host  = nullptr; // mapped word: a tensor-core launch gave up
	int*           err_dev   = nullptr;
	std::string    err;
};

namespace dmrgpp {
namespace {

thread_local std::string g_mlp_error;

int mlp_fail(dmrgpp_mlp_handle m, int status, const std::string& msg)
{
	if (m)
		m->err = msg;
	else
		g_mlp_error = msg;
	return status;
}

int mlp_cuda(dmrgpp_mlp_handle m, cudaError_t e, const char* where)
{
	return mlp_fail(m, e == cudaErrorMemoryAllocation ? DMRGPP_OOM : DMRGPP_CUDA_ERROR,
	                std::string(where) + ": " + cudaGetErrorString(e));
}

__device__ __forceinline__ void features(double d, double r, double theta, double s, double rms,
                                         float* x)
{
	const float f0 = float((d - theta) / s);
	const float f1 = rms > 0 ? float(r / rms) : 0.f;
	x[0]           = f0;
	x[1]           = f1;
	x[2]           = f1 * f0 / (f0 * f0 + kDelta * kDelta);
	const float q  = f0 / kDelta;
	x[3]           = 1.f / (1.f + q * q);
}

__global__ void k_features(const double* __restrict__ d, const double* __restrict__ r, double theta,
                           double s, double rms, size_t n, float* __restrict__ x)
{
	for (size_t e = blockIdx.x * size_t(blockDim.x) + threadIdx.x; e < n;
	     e += size_t(gridDim.x) * blockDim.x)
		features(d[e], r[e], theta, s, rms, x + e * F);
}

// Per-sector Ritz values and residual norms of a group of sectors (device
// arrays; start has nsec + 1 entries).  start == NULL: one sector, the
// scalars passed beside it.
struct SectorScalars {
	const long long* start;
	const double*    theta;
	const double*    rnorm;
	int              nsec;
};

struct RowScalars {
	double theta, s, rms, scale;
};

// The scalars of element e: the single-sector ones, or those of the sector
// holding e (binary search over the sector starts), formed as the host
// forms them for one sector: s = max(1, |theta|), rms = |r| / sqrt(n_s).
__device__ __forceinline__ RowScalars row_scalars(const SectorScalars& g, const RowScalars& one, long long e)
{
	if (!g.start)
		return one;
	int lo = 0, hi = g.nsec;
	while (hi - lo > 1) {
		const int mid = (lo + hi) >> 1;
		if (g.start[mid] <= e)
			lo = mid;
		else
			hi = mid;
	}
	RowScalars      v;
	const long long n = g.start[lo + 1] - g.start[lo];
	v.theta           = g.theta[lo];
	v.s               = fmax(1.0, fabs(v.theta));
	v.rms             = g.rnorm[lo] / sqrt(double(n > 0 ? n : 1));
	v.scale           = v.rms / v.s;
	return v;
}

// features of rows e0 .. e0 + n of a group
__global__ void k_features_group(const double* __restrict__ d, const double* __restrict__ r,
                                 SectorScalars g, long long e0, size_t n, float* __restrict__ x)
{
	const RowScalars none {};
	for (size_t e = blockIdx.x * size_t(blockDim.x) + threadIdx.x; e < n;
	     e += size_t(gridDim.x) * blockDim.x) {
		const RowScalars v = row_scalars(g, none, e0 + (long long)e);
		features(d[e], r[e], v.theta, v.s, v.rms, x + e * F);
	}
}

// C (M x N, row-major, ldc) = op(A) * op(B) (+ C if accumulate); op(A) is
// M x K, op(B) is K x N.  TA: A stored K x M (row-major) instead of M x K.
// TB: B stored N x K instead of K x N.  64 x 64 tiles, k-steps of 16, each
// of 256 threads owns a 4 x 4 block; the k order is fixed.
template <bool TA, bool TB>
__global__ void __launch_bounds__(256)
k_sgemm(int M, int N, int K, const float* __restrict__ A, int lda, const float* __restrict__ B,
        int ldb, float* __restrict__ C, int ldc, int accumulate)
{
	__shared__ float As[16][64 + 4];
	__shared__ float Bs[16][64 + 4];
	const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
	const int m0 = blockIdx.y * 64, n0 = blockIdx.x * 64;
	float     acc[4][4] = {};
	for (int k0 = 0; k0 < K; k0 += 16) {
		for (int q = threadIdx.x; q < 16 * 64; q += 256) {
			const int kk = q / 64, mm = q % 64;
			const int gm = m0 + mm, gk = k0 + kk;
			float     v  = 0.f;
			if (gm < M && gk < K)
				v = TA ? A[size_t(gk) * lda + gm] : A[size_t(gm) * lda + gk];
			As[kk][mm] = v;
			const int gn = n0 + mm;
			float     w  = 0.f;
			if (gn < N && gk < K)
				w = TB ? B[size_t(gn) * ldb + gk] : B[size_t(gk) * ldb + gn];
			Bs[kk][mm] = w;
		}
		__syncthreads();
#pragma unroll
		for (int kk = 0; kk < 16; ++kk) {
			float a[4], b[4];
#pragma unroll
			for (int i = 0; i < 4; ++i) {
				a[i] = As[kk][ty * 4 + i];
				b[i] = Bs[kk][tx * 4 + i];
			}
#pragma unroll
			for (int i = 0; i < 4; ++i)
#pragma unroll
				for (int j = 0; j < 4; ++j)
					acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
		}
		__syncthreads();
	}
#pragma unroll
	for (int i = 0; i < 4; ++i)
#pragma unroll
		for (int j = 0; j < 4; ++j) {
			const int gm = m0 + ty * 4 + i, gn = n0 + tx * 4 + j;
			if (gm < M && gn < N) {
				float* c = C + size_t(gm) * ldc + gn;
				*c       = accumulate ? *c + acc[i][j] : acc[i][j];
			}
		}
}

template <bool TA, bool TB>
void sgemm(int M, int N, int K, const float* A, int lda, const float* B, int ldb, float* C, int ldc,
           bool accumulate, cudaStream_t st)
{
	dim3 grid((N + 63) / 64, (M + 63) / 64);
	k_sgemm<TA, TB><<<grid, 256, 0, st>>>(M, N, K, A, lda, B, ldb, C, ldc, accumulate ? 1 : 0);
}

// Z (rows x H) += bias; Z = tanh(Z)
__global__ void k_bias_tanh(float* __restrict__ Z, const float* __restrict__ b, size_t rows)
{
	for (size_t q = blockIdx.x * size_t(blockDim.x) + threadIdx.x; q < rows * H;
	     q += size_t(gridDim.x) * blockDim.x)
		Z[q] = tanhf(Z[q] + b[q % H]);
}

// out[b] = h2[b,:] . w3 + b3  (one warp per row)
__global__ void k_head(const float* __restrict__ h2, const float* __restrict__ w3, const float* b3,
                       float* __restrict__ out, int rows)
{
	const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
	if (warp >= rows)
		return;
	float s = 0.f;
	for (int j = lane; j < H; j += 32)
		s = fmaf(h2[size_t(warp) * H + j], w3[j], s);
	for (int o = 16; o > 0; o >>= 1)
		s += __shfl_down_sync(0xffffffffu, s, o);
	if (lane == 0)
		out[warp] = s + b3[0];
}

// loss = sum w_b (o_b - y_b)^2 / rows, gout_b = 2 w_b (o_b - y_b) / rows
__global__ void k_mse(const float* __restrict__ o, const float* __restrict__ y,
                      const float* __restrict__ wgt, int rows, float* __restrict__ gout,
                      double* loss, double* partial, unsigned* ctr)
{
	__shared__ double red[8];
	double            s = 0.0;
	for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < rows; b += gridDim.x * blockDim.x) {
		const float wb = wgt ? wgt[b] : 1.f;
		const float d  = o[b] - y[b];
		gout[b]        = 2.f * wb * d / float(rows);
		s += double(wb) * double(d) * double(d);
	}
	for (int off = 16; off > 0; off >>= 1)
		s += __shfl_down_sync(0xffffffffu, s, off);
	if ((threadIdx.x & 31) == 0)
		red[threadIdx.x >> 5] = s;
	__syncthreads();
	if (threadIdx.x == 0) {
		double t = 0.0;
		for (int w = 0; w < int(blockDim.x >> 5); ++w)
			t += red[w];
		partial[blockIdx.x] = t;
		__threadfence();
		if (atomicAdd(ctr, 1u) == gridDim.x - 1) {
			__threadfence();
			double tot = 0.0;
			for (int b = 0; b < int(gridDim.x); ++b)
				tot += __ldcg(partial + b);
			*loss = tot / double(rows);
			*ctr  = 0u;
		}
	}
}

// dz = (gout[b] * w3[j]) * (1 - h2^2)
__global__ void k_head_back(const float* __restrict__ gout, const float* __restrict__ w3,
                            const float* __restrict__ h2, float* __restrict__ dz, size_t rows)
{
	for (size_t q = blockIdx.x * size_t(blockDim.x) + threadIdx.x; q < rows * H;
	     q += size_t(gridDim.x) * blockDim.x) {
		const float h = h2[q];
		dz[q]         = gout[q / H] * w3[q % H] * (1.f - h * h);
	}
}

// dz *= (1 - h^2)
__global__ void k_tanh_back(float* __restrict__ dz, const float* __restrict__ h, size_t n)
{
	for (size_t q = blockIdx.x * size_t(blockDim.x) + threadIdx.x; q < n;
	     q += size_t(gridDim.x) * blockDim.x)
		dz[q] *= 1.f - h[q] * h[q];
}

// g[j] = sum_b M[b, j] (fixed order), cols columns of a rows x cols matrix
__global__ void k_colsum(const float* __restrict__ Mx, int rows, int cols, float* __restrict__ g)
{
	const int j = blockIdx.x * blockDim.x + threadIdx.x;
	if (j >= cols)
		return;
	float s = 0.f;
	for (int b = 0; b < rows; ++b)
		s += Mx[size_t(b) * cols + j];
	g[j] = s;
}

__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, size_t n, float lr, float b1, float b2, float eps,
                       float c1, float c2)
{
	for (size_t q = blockIdx.x * size_t(blockDim.x) + threadIdx.x; q < n;
	     q += size_t(gridDim.x) * blockDim.x) {
		const float gq = g[q];
		m[q]           = b1 * m[q] + (1.f - b1) * gq;
		v[q]           = b2 * v[q] + (1.f - b2) * gq * gq;
		p[q] -= lr * (m[q] / c1) / (sqrtf(v[q] / c2) + eps);
	}
}

__global__ void k_to_bf16(const float* __restrict__ p, __nv_bfloat16* __restrict__ q, size_t n)
{
	for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n;
	     i += size_t(gridDim.x) * blockDim.x)
		q[i] = __float2bfloat16_rn(p[i]);
}

__global__ void k_from_bf16(const __nv_bfloat16* __restrict__ q, float* __restrict__ p, size_t n)
{
	for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n;
	     i += size_t(gridDim.x) * blockDim.x)
		p[i] = __bfloat162float(q[i]);
}

// t_e = o_e * rms / s
__global__ void k_scale_out(const float* __restrict__ o, double scale, double* __restrict__ t, size_t n)
{
	for (size_t e = blockIdx.x * size_t(blockDim.x) + threadIdx.x; e < n;
	     e += size_t(gridDim.x) * blockDim.x)
		t[e] = double(o[e]) * scale;
}

__global__ void k_scale_out_group(const float* __restrict__ o, SectorScalars g, long long e0,
                                  double* __restrict__ t, size_t n)
{
	const RowScalars none {};
	for (size_t e = blockIdx.x * size_t(blockDim.x) + threadIdx.x; e < n;
	     e += size_t(gridDim.x) * blockDim.x)
		t[e] = double(o[e]) * row_scalars(g, none, e0 + (long long)e).scale;
}

// ------------------------------------------------ tensor-core inference
constexpr int kTcRows    = 128;                 // elements per tile = TMEM lanes
constexpr int kTcSlots   = 4;                   // ring of h1 chunks (64 units each)
constexpr int kTcThreads = 288;                 // layer-1 warps 0-3, epilogue 4-7, MMA 8
constexpr int kW2Bytes   = H * H * 2;           // BF16 W2, 128 KB
constexpr int kSlotBytes = kTcRows * 128;       // 128 rows x 64 BF16
constexpr int kTcSmem    = kW2Bytes + kTcSlots * kSlotBytes + 1024;

struct MlpTcArgs {
	const double*        diag;
	const double*        r;
	double*              t;
	long long            n;
	int                  ntiles;
	RowScalars           one; // one sector: theta, s, rms, scale = rms / s
	SectorScalars        g;   // a group of sectors (g.start != NULL): per-row scalars
	const float*         p;  // parameters: BF16 values widened to FP32
	const __nv_bfloat16* w2; // BF16 W2 (row j = hidden unit j of layer 2)
	int*                 error;
};

// kind::f16: D = F32, A = B = BF16, both K-major, M = 128, N = 256
__device__ __forceinline__ unsigned idesc_bf16_128x256()
{
	return (1u << 4) | (1u << 7) | (1u << 10) | (unsigned(256 >> 3) << 17) | (unsigned(128 >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(unsigned d, uint64_t a, uint64_t b, unsigned idesc, unsigned acc)
{
	asm volatile("{\n\t.reg .pred p;\n\t"
	             "setp.ne.b32 p, %4, 0;\n\t"
	             "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
	             "l"(a), "l"(b), "r"(idesc), "r"(acc)
	             : "memory");
}

__device__ __forceinline__ float tanh_sfu(float x)
{
	float y;
	asm("tanh.approx.f32 %0, %1;\n" : "=f"(y) : "f"(x));
	return y;
}

// generic-proxy shared-memory writes -> visible to the tensor cores
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

// byte offset of 16-byte unit u (0..7) of a 128-byte row in the
// 128-byte-swizzled K-major layout (8-row atoms of 1024 bytes)
__device__ __forceinline__ unsigned swz(int row, int u)
{
	return unsigned(row) * 128u + unsigned((u ^ (row & 7)) * 16);
}

__device__ __forceinline__ unsigned bf16x2(float lo, float hi)
{
	const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
	return *reinterpret_cast<const unsigned*>(&v);
}

__device__ __forceinline__ void mlp_give_up(volatile int* abort, int* error)
{
	*abort = 1;
	atomicExch(error, 2);
}

__global__ void __launch_bounds__(kTcThreads, 1) mlp_infer_tc_kernel(const __grid_constant__ MlpTcArgs a)
{
	using namespace tc;
	extern __shared__ unsigned char smem_raw[];
	__shared__ float                           sW1[H * F], sb1[H], sb2[H], sw3[H];
	__shared__ float                           sb3;
	__shared__ __align__(8) unsigned long long bars[2 * kTcSlots + 5];
	__shared__ unsigned                        tmem_slot;
	__shared__ volatile int                    abort_flag;

	const unsigned raw   = smem_addr(smem_raw);
	const unsigned base  = (raw + 1023u) & ~1023u; // W2, then the ring
	unsigned char* basep = smem_raw + (base - raw);
	const unsigned full0 = smem_addr(&bars[0]), empty0 = smem_addr(&bars[kTcSlots]);
	const unsigned accf0 = smem_addr(&bars[2 * kTcSlots]), acce0 = smem_addr(&bars[2 * kTcSlots + 2]);
	const unsigned drain = smem_addr(&bars[2 * kTcSlots + 4]);
	const int      warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

	for (int i = threadIdx.x; i < H * F; i += kTcThreads)
		sW1[i] = a.p[kW1 + i];
	for (int i = threadIdx.x; i < H; i += kTcThreads) {
		sb1[i] = a.p[kB1 + i];
		sb2[i] = a.p[kB2 + i];
		sw3[i] = a.p[kW3 + i];
	}
	if (threadIdx.x == 0)
		sb3 = a.p[kB3];
	// W2 as the B operand (N = 256 rows j, K = 256): K-chunk c holds units
	// 64c .. 64c+63 of every row, 32 KB per chunk
	const uint4* w2g = reinterpret_cast<const uint4*>(a.w2);
	for (int u = threadIdx.x; u < H * H / 8; u += kTcThreads) {
		const int j = u >> 5, q = u & 31;
		*reinterpret_cast<uint4*>(basep + (q >> 3) * (H * 128) + swz(j, q & 7)) = w2g[u];
	}
	fence_async_smem();
	if (warp == 8) {
		asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
		                 smem_addr(&tmem_slot)),
		             "r"(512u)
		             : "memory");
		asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
	}
	if (threadIdx.x == 0) {
		abort_flag = 0;
		for (int q = 0; q < kTcSlots; ++q) {
			mbar_init(full0 + 8 * q, 4); // one arrival per layer-1 warp
			mbar_init(empty0 + 8 * q, 1);
		}
		for (int b = 0; b < 2; ++b) {
			mbar_init(accf0 + 8 * b, 1);
			mbar_init(acce0 + 8 * b, 4); // one arrival per epilogue warp
		}
		mbar_init(drain, 1);
		asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
	}
	tc_fence_before();
	__syncthreads();
	tc_fence_after();
	const unsigned tmem = tmem_slot;
	const unsigned ring = base + kW2Bytes;

	if (warp < 4) {
		// layer 1: thread = element row of the tile
		const int row = threadIdx.x;
		unsigned  g   = 0;
		bool      ok  = true;
		for (int tile = blockIdx.x; tile < a.ntiles && ok; tile += gridDim.x) {
			const long long e    = (long long)tile * kTcRows + row;
			float           x[F] = { 0.f, 0.f, 0.f, 0.f };
			if (e < a.n) {
				const RowScalars v = row_scalars(a.g, a.one, e);
				features(a.diag[e], a.r[e], v.theta, v.s, v.rms, x);
			}
			for (int c = 0; c < H / 64; ++c) {
				const unsigned slot = g % kTcSlots;
				if (g >= kTcSlots)
					ok = __all_sync(0xffffffffu, mbar_wait(empty0 + 8 * slot, ((g / kTcSlots) - 1) & 1, &abort_flag));
				if (!ok)
					break;
				unsigned char* dst = basep + kW2Bytes + slot * kSlotBytes;
#pragma unroll
				for (int u = 0; u < 8; ++u) {
					unsigned w[4];
#pragma unroll
					for (int q = 0; q < 4; ++q) {
						const int j0 = c * 64 + u * 8 + 2 * q;
						float     h[2];
#pragma unroll
						for (int k = 0; k < 2; ++k) {
							const float* wr = sW1 + (j0 + k) * F;
							h[k] = tanh_sfu(fmaf(wr[3], x[3], fmaf(wr[2], x[2], fmaf(wr[1], x[1], fmaf(wr[0], x[0], sb1[j0 + k])))));
						}
						w[q] = bf16x2(h[0], h[1]);
					}
					*reinterpret_cast<uint4*>(dst + swz(row, u)) = make_uint4(w[0], w[1], w[2], w[3]);
				}
				fence_async_smem();
				__syncwarp();
				if (lane == 0)
					mbar_arrive(full0 + 8 * slot);
				++g;
			}
		}
		if (!ok && lane == 0)
			mlp_give_up(&abort_flag, a.error);
	} else if (warp < 8) {
		// epilogue: TMEM lanes 32 (warp % 4) ..
		const int quarter = warp & 3, row = quarter * 32 + lane;
		unsigned  tcount  = 0;
		bool      ok      = true;
		for (int tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x) {
			const unsigned b = tcount & 1;
			ok               = __all_sync(0xffffffffu, mbar_wait(accf0 + 8 * b, (tcount >> 1) & 1, &abort_flag));
			if (!ok)
				break;
			tc_fence_after();
			float o = 0.f;
			for (int c0 = 0; c0 < H; c0 += 32) {
				float v[32];
				tmem_ld32(tmem + (unsigned(quarter * 32) << 16) + b * 256u + unsigned(c0), v);
#pragma unroll
				for (int i = 0; i < 32; ++i)
					o = fmaf(sw3[c0 + i], tanh_sfu(v[i] + sb2[c0 + i]), o);
			}
			tc_fence_before();
			__syncwarp();
			if (lane == 0)
				mbar_arrive(acce0 + 8 * b);
			const long long e = (long long)tile * kTcRows + row;
			if (e < a.n)
				a.t[e] = double(o + sb3) * row_scalars(a.g, a.one, e).scale;
			++tcount;
		}
		if (!ok && lane == 0)
			mlp_give_up(&abort_flag, a.error);
	} else if (lane == 0) {
		// layer-2 MMAs
		const unsigned idesc  = idesc_bf16_128x256();
		unsigned       g      = 0, tcount = 0;
		bool           ok     = true, issued = false;
		for (int tile = blockIdx.x; tile < a.ntiles && ok; tile += gridDim.x) {
			const unsigned b = tcount & 1;
			if (tcount >= 2 && !mbar_wait(acce0 + 8 * b, ((tcount >> 1) - 1) & 1, &abort_flag)) {
				ok = false;
				break;
			}
			tc_fence_after();
			const unsigned d = tmem + b * 256u;
			for (int c = 0; c < H / 64; ++c) {
				const unsigned slot = g % kTcSlots;
				if (!mbar_wait(full0 + 8 * slot, (g / kTcSlots) & 1, &abort_flag)) {
					ok = false;
					break;
				}
				tc_fence_after();
#pragma unroll
				for (int ks = 0; ks < 4; ++ks) // K = 16 BF16 = 32 bytes per MMA
					mma_bf16(d, smem_desc(ring + slot * kSlotBytes + ks * 32),
					         smem_desc(base + c * (H * 128) + ks * 32), idesc, (c | ks) != 0);
				mma_commit(empty0 + 8 * slot);
				issued = true;
				++g;
			}
			if (!ok)
				break;
			mma_commit(accf0 + 8 * b);
			++tcount;
		}
		if (!ok)
			mlp_give_up(&abort_flag, a.error);
		if (issued) {
			mma_commit(drain);
			if (!mbar_wait(drain, 0, nullptr))
				mlp_give_up(&abort_flag, a.error);
		}
	}
	__syncwarp();
	tc_fence_before();
	__syncthreads();
	tc_fence_after();
	if (warp == 8)
		asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(512u)
		             : "memory");
}

int grid_for(size_t n, int threads = 256)
{
	size_t b = (n + threads - 1) / threads;
	return int(b < 148 * 16 ? (b > 0 ? b : 1) : 148 * 16);
}

int ensure_rows(dmrgpp_mlp_handle m, int rows)
{
	if (rows <= m->cap)
		return DMRGPP_OK;
	cudaFree(m->x);
	cudaFree(m->h1);
	cudaFree(m->h2);
	cudaFree(m->out);
	cudaFree(m->gout);
	cudaFree(m->dz);
	cudaFree(m->dz1);
	m->x = m->h1 = m->h2 = m->out = m->gout = m->dz = m->dz1 = nullptr;
	m->cap                                                   = 0;
	cudaError_t e;
	const size_t r = size_t(rows);
	if ((e = cudaMalloc(&m->x, r * F * sizeof(float))) || (e = cudaMalloc(&m->h1, r * H * sizeof(float)))
	    || (e = cudaMalloc(&m->h2, r * H * sizeof(float))) || (e = cudaMalloc(&m->out, r * sizeof(float)))
	    || (e = cudaMalloc(&m->gout, r * sizeof(float))) || (e = cudaMalloc(&m->dz, r * H * sizeof(float)))
	    || (e = cudaMalloc(&m->dz1, r * H * sizeof(float))))
		return mlp_cuda(m, e, "MLP row buffers");
	m->cap = rows;
	return DMRGPP_OK;
}

// FP32 forward of `rows` feature rows x (rows x F) with parameter set P;
// fills m->h1, m->h2, m->out
void forward(dmrgpp_mlp_handle m, const float* P, const float* x, int rows, cudaStream_t st)
{
	sgemm<false, true>(rows, H, F, x, F, P + kW1, F, m->h1, H, false, st);
	k_bias_tanh<<<grid_for(size_t(rows) * H), 256, 0, st>>>(m->h1, P + kB1, size_t(rows));
	sgemm<false, true>(rows, H, H, m->h1, H, P + kW2, H, m->h2, H, false, st);
	k_bias_tanh<<<grid_for(size_t(rows) * H), 256, 0, st>>>(m->h2, P + kB2, size_t(rows));
	k_head<<<(rows * 32 + 255) / 256, 256, 0, st>>>(m->h2, P + kW3, P + kB3, m->out, rows);
}

} // namespace

namespace {

// t = learned correction of r; one sector (g.start == NULL: theta, rnorm) or
// a group of sectors (per-sector scalars in g)
int precondition(dmrgpp_mlp_handle m, const double* diag, const double* r, double theta, double rnorm,
                 const SectorScalars& g, double* t, size_t n, cudaStream_t st)
{
	if (!m)
		return DMRGPP_INVALID_ARG;
	RowScalars one;
	one.theta = theta;
	one.s     = std::max(1.0, std::fabs(theta));
	one.rms   = rnorm / std::sqrt(double(n > 0 ? n : 1));
	one.scale = one.rms / one.s;
	if (m->bf_dirty) {
		k_to_bf16<<<grid_for(kNumParams), 256, 0, st>>>(m->params, m->wbf, kNumParams);
		m->bf_dirty = false;
	}
	// inference weights: BF16 values widened to FP32 (the network as it ships)
	k_from_bf16<<<grid_for(kNumParams), 256, 0, st>>>(m->wbf, m->pinf, kNumParams);
	const float* pinf = m->pinf;
	if (m->inference == DMRGPP_MLP_TENSOR_CORES) {
		if (*reinterpret_cast<volatile int*>(m->err_host)) {
			*m->err_host = 0;
			return mlp_fail(m, DMRGPP_TIMEOUT, "an earlier tensor-core MLP launch gave up waiting");
		}
		if (n == 0)
			return DMRGPP_OK;
		static thread_local int attr_device = -1;
		int                     dev = 0, sms = 0;
		cudaError_t             e   = cudaGetDevice(&dev);
		if (!e && attr_device != dev) {
			e = cudaFuncSetAttribute(mlp_infer_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem);
			if (!e)
				attr_device = dev;
		}
		if (!e)
			e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
		if (e)
			return mlp_cuda(m, e, "MLP tensor-core kernel attributes");
		MlpTcArgs a;
		a.diag   = diag;
		a.r      = r;
		a.t      = t;
		a.n      = (long long)n;
		a.ntiles = int((n + kTcRows - 1) / kTcRows);
		a.one    = one;
		a.g      = g;
		a.p      = pinf;
		a.w2     = m->wbf + kW2;
		a.error  = m->err_dev;
		mlp_infer_tc_kernel<<<unsigned(std::min(a.ntiles, sms)), kTcThreads, kTcSmem, st>>>(a);
		e = cudaGetLastError();
		return e == cudaSuccess ? DMRGPP_OK : mlp_cuda(m, e, "MLP tensor-core inference");
	}
	const int chunk = 1 << 16;
	if (int rc = ensure_rows(m, int(std::min<size_t>(n, chunk))))
		return rc;
	for (size_t e0 = 0; e0 < n; e0 += chunk) {
		const int rows = int(std::min<size_t>(chunk, n - e0));
		if (g.start)
			k_features_group<<<grid_for(size_t(rows)), 256, 0, st>>>(diag + e0, r + e0, g, (long long)e0,
			                                                        size_t(rows), m->x);
		else
			k_features<<<grid_for(size_t(rows)), 256, 0, st>>>(diag + e0, r + e0, one.theta, one.s,
			                                                  one.rms, size_t(rows), m->x);
		forward(m, pinf, m->x, rows, st);
		if (g.start)
			k_scale_out_group<<<grid_for(size_t(rows)), 256, 0, st>>>(m->out, g, (long long)e0, t + e0,
			                                                         size_t(rows));
		else
			k_scale_out<<<grid_for(size_t(rows)), 256, 0, st>>>(m->out, one.scale, t + e0, size_t(rows));
	}
	cudaError_t e = cudaGetLastError();
	return e == cudaSuccess ? DMRGPP_OK : mlp_cuda(m, e, "MLP inference");
}

} // namespace

int mlp_precondition(dmrgpp_mlp_handle m, const double* diag, const double* r, double theta,
                     double rnorm, double* t, size_t n, cudaStream_t st)
{
	return precondition(m, diag, r, theta, rnorm, SectorScalars {}, t, n, st);
}

int mlp_precondition_group(dmrgpp_mlp_handle m, const double* diag, const double* r,
                           const long long* sector_start, const double* theta, const double* rnorm,
                           int nsec, double* t, size_t n, cudaStream_t st)
{
	if (nsec < 1 || !sector_start || !theta || !rnorm)
		return mlp_fail(m, DMRGPP_INVALID_ARG, "group preconditioner: null sector arrays");
	const SectorScalars g { sector_start, theta, rnorm, nsec };
	return precondition(m, diag, r, 0.0, 0.0, g, t, n, st);
}

} // namespace dmrgpp

extern "C" {

size_t dmrgpp_mlp_num_params(void) { return dmrgpp::kNumParams; }

const char* dmrgpp_mlp_last_error(dmrgpp_mlp_handle m) { return m ? m->err.c_str() : dmrgpp::g_mlp_error.c_str(); }

int dmrgpp_mlp_create(unsigned long long seed, dmrgpp_mlp_handle* out)
{
	using namespace dmrgpp;
	if (!out)
		return mlp_fail(nullptr, DMRGPP_INVALID_ARG, "null output");
	*out                = nullptr;
	dmrgpp_mlp_handle m = new dmrgpp_mlp_s();
	cudaGetDevice(&m->device);
	// Glorot-uniform weights, zero biases, from a seeded host generator
	std::vector<float>               p(kNumParams, 0.f);
	std::mt19937_64                  rng(seed);
	auto                             fill = [&](size_t off, int fan_in, int fan_out, size_t count) {
                const float a = std::sqrt(6.f / float(fan_in + fan_out));
                std::uniform_real_distribution<float> u(-a, a);
                for (size_t i = 0; i < count; ++i)
                        p[off + i] = u(rng);
	};
	fill(kW1, F, H, size_t(H) * F);
	fill(kW2, H, H, size_t(H) * H);
	fill(kW3, H, 1, size_t(H));
	cudaError_t e;
	if ((e = cudaMalloc(&m->params, kNumParams * sizeof(float)))
	    || (e = cudaMalloc(&m->grads, kNumParams * sizeof(float)))
	    || (e = cudaMalloc(&m->adam_m, kNumParams * sizeof(float)))
	    || (e = cudaMalloc(&m->adam_v, kNumParams * sizeof(float)))
	    || (e = cudaMalloc(&m->wbf, kNumParams * sizeof(__nv_bfloat16)))
	    || (e = cudaMalloc(&m->pinf, kNumParams * sizeof(float)))
	    || (e = cudaMalloc(&m->loss, sizeof(double)))
	    || (e = cudaMalloc(&m->partial, 4096 * sizeof(double)))
	    || (e = cudaMalloc(&m->ctr, sizeof(unsigned))) || (e = cudaMemset(m->ctr, 0, sizeof(unsigned)))
	    || (e = cudaMemset(m->adam_m, 0, kNumParams * sizeof(float)))
	    || (e = cudaMemset(m->adam_v, 0, kNumParams * sizeof(float)))
	    || (e = cudaMemcpy(m->params, p.data(), kNumParams * sizeof(float), cudaMemcpyHostToDevice))
	    // the MLP's kernels run on callers' streams, which may be non-blocking
	    // (not ordered with these legacy-stream writes): finish them here
	    || (e = cudaDeviceSynchronize())
	    || (e = error_word_alloc(&m->err_host, &m->err_dev))) {
		const int rc = mlp_cuda(nullptr, e, "MLP create");
		dmrgpp_mlp_destroy(m);
		return rc;
	}
	*out = m;
	return DMRGPP_OK;
}

int dmrgpp_mlp_destroy(dmrgpp_mlp_handle m)
{
	if (!m)
		return DMRGPP_OK;
	cudaDeviceSynchronize();
	cudaFree(m->params);
	cudaFree(m->grads);
	cudaFree(m->adam_m);
	cudaFree(m->adam_v);
	cudaFree(m->wbf);
	cudaFree(m->pinf);
	cudaFree(m->loss);
	cudaFree(m->partial);
	cudaFree(m->ctr);
	cudaFree(m->x);
	cudaFree(m->h1);
	cudaFree(m->h2);
	cudaFree(m->out);
	cudaFree(m->gout);
	cudaFree(m->dz);
	cudaFree(m->dz1);
	dmrgpp::error_word_free(m->err_host);
	delete m;
	return DMRGPP_OK;
}

int dmrgpp_mlp_set_inference(dmrgpp_mlp_handle m, int mode)
{
	if (!m)
		return dmrgpp::mlp_fail(nullptr, DMRGPP_INVALID_ARG, "null handle");
	if (mode != DMRGPP_MLP_TENSOR_CORES && mode != DMRGPP_MLP_CUDA_CORES)
		return dmrgpp::mlp_fail(m, DMRGPP_INVALID_ARG, "unknown inference mode");
	m->inference = mode;
	return DMRGPP_OK;
}

int dmrgpp_mlp_get_params(dmrgpp_mlp_handle m, float* host, size_t n)
{
	if (!m || !host || n != dmrgpp::kNumParams)
		return DMRGPP_INVALID_ARG;
	// kernels on callers' (possibly non-blocking) streams finish first
	return cudaDeviceSynchronize() == cudaSuccess
	        && cudaMemcpy(host, m->params, n * sizeof(float), cudaMemcpyDeviceToHost) == cudaSuccess
	    ? DMRGPP_OK
	    : DMRGPP_CUDA_ERROR;
}

int dmrgpp_mlp_set_params(dmrgpp_mlp_handle m, const float* host, size_t n)
{
	if (!m || !host || n != dmrgpp::kNumParams)
		return DMRGPP_INVALID_ARG;
	m->bf_dirty = true;
	m->adam_t   = 0;
	// no kernel on a caller's stream may still use the old values, and the
	// next one must see the new ones
	if (cudaDeviceSynchronize() != cudaSuccess)
		return DMRGPP_CUDA_ERROR;
	cudaMemset(m->adam_m, 0, n * sizeof(float));
	cudaMemset(m->adam_v, 0, n * sizeof(float));
	return cudaMemcpy(m->params, host, n * sizeof(float), cudaMemcpyHostToDevice) == cudaSuccess
	        && cudaDeviceSynchronize() == cudaSuccess
	    ? DMRGPP_OK
	    : DMRGPP_CUDA_ERROR;
}

int dmrgpp_mlp_get_grads(dmrgpp_mlp_handle m, float* host, size_t n)
{
	if (!m || !host || n != dmrgpp::kNumParams)
		return DMRGPP_INVALID_ARG;
	return cudaDeviceSynchronize() == cudaSuccess
	        && cudaMemcpy(host, m->grads, n * sizeof(float), cudaMemcpyDeviceToHost) == cudaSuccess
	    ? DMRGPP_OK
	    : DMRGPP_CUDA_ERROR;
}

int dmrgpp_mlp_features(const double* diag, const double* r, double theta, double rnorm, size_t n,
                        float* x, void* stream)
{
	if (!diag || !r || !x)
		return DMRGPP_INVALID_ARG;
	const double s   = std::max(1.0, std::fabs(theta));
	const double rms = rnorm / std::sqrt(double(n > 0 ? n : 1));
	dmrgpp::k_features<<<dmrgpp::grid_for(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(
	    diag, r, theta, s, rms, n, x);
	return cudaGetLastError() == cudaSuccess ? DMRGPP_OK : DMRGPP_CUDA_ERROR;
}

int dmrgpp_mlp_forward(dmrgpp_mlp_handle m, const float* x, int rows, float* out, void* stream)
{
	DMRGPP_TRACE("dmrgpp_mlp_forward");
	using namespace dmrgpp;
	if (!m || !x || rows < 1)
		return DMRGPP_INVALID_ARG;
	cudaStream_t st = static_cast<cudaStream_t>(stream);
	if (int rc = ensure_rows(m, rows))
		return rc;
	forward(m, m->params, x, rows, st);
	m->last_rows = rows;
	if (out && cudaMemcpyAsync(out, m->out, size_t(rows) * sizeof(float), cudaMemcpyDeviceToDevice, st))
		return mlp_fail(m, DMRGPP_CUDA_ERROR, "copy output");
	return cudaGetLastError() == cudaSuccess ? DMRGPP_OK : mlp_fail(m, DMRGPP_CUDA_ERROR, "forward");
}

int dmrgpp_mlp_backward(dmrgpp_mlp_handle m, const float* x, const float* y, const float* weight,
                        double* loss, void* stream)
{
	DMRGPP_TRACE("dmrgpp_mlp_backward");
	using namespace dmrgpp;
	if (!m || !x || !y || m->last_rows < 1)
		return DMRGPP_INVALID_ARG;
	cudaStream_t st   = static_cast<cudaStream_t>(stream);
	const int    rows = m->last_rows;
	const float* P    = m->params;
	float*       G    = m->grads;
	const int    nbm  = std::min(4096, (rows + 255) / 256);
	k_mse<<<nbm, 256, 0, st>>>(m->out, y, weight, rows, m->gout, m->loss, m->partial, m->ctr);
	// head: dw3 = h2^T gout, db3 = sum gout
	sgemm<true, false>(H, 1, rows, m->h2, H, m->gout, 1, G + kW3, 1, false, st);
	k_colsum<<<1, 32, 0, st>>>(m->gout, rows, 1, G + kB3);
	// layer 2: dz2 = gout w3 (1 - h2^2); dW2 = dz2^T h1; db2 = colsum dz2
	k_head_back<<<grid_for(size_t(rows) * H), 256, 0, st>>>(m->gout, P + kW3, m->h2, m->dz, size_t(rows));
	sgemm<true, false>(H, H, rows, m->dz, H, m->h1, H, G + kW2, H, false, st);
	k_colsum<<<(H + 255) / 256, 256, 0, st>>>(m->dz, rows, H, G + kB2);
	// layer 1: dz1 = (dz2 W2) (1 - h1^2); dW1 = dz1^T x; db1 = colsum dz1
	sgemm<false, false>(rows, H, H, m->dz, H, P + kW2, H, m->dz1, H, false, st);
	k_tanh_back<<<grid_for(size_t(rows) * H), 256, 0, st>>>(m->dz1, m->h1, size_t(rows) * H);
	sgemm<true, false>(H, F, rows, m->dz1, H, x, F, G + kW1, F, false, st);
	k_colsum<<<(H + 255) / 256, 256, 0, st>>>(m->dz1, rows, H, G + kB1);
	if (loss && cudaMemcpyAsync(loss, m->loss, sizeof(double), cudaMemcpyDeviceToHost, st))
		return mlp_fail(m, DMRGPP_CUDA_ERROR, "read loss");
	if (cudaStreamSynchronize(st) != cudaSuccess)
		return mlp_fail(m, DMRGPP_CUDA_ERROR, "backward");
	return DMRGPP_OK;
}

int dmrgpp_mlp_adam_step(dmrgpp_mlp_handle m, float lr, void* stream)
{
	DMRGPP_TRACE("dmrgpp_mlp_adam_step");
	using namespace dmrgpp;
	if (!m)
		return DMRGPP_INVALID_ARG;
	m->adam_t++;
	const float b1 = 0.9f, b2 = 0.999f;
	const float c1 = 1.f - std::pow(b1, float(m->adam_t)), c2 = 1.f - std::pow(b2, float(m->adam_t));
	k_adam<<<grid_for(kNumParams), 256, 0, static_cast<cudaStream_t>(stream)>>>(
	    m->params, m->grads, m->adam_m, m->adam_v, kNumParams, lr, b1, b2, 1e-8f, c1, c2);
	m->bf_dirty = true;
	return cudaGetLastError() == cudaSuccess ? DMRGPP_OK : DMRGPP_CUDA_ERROR;
}

int dmrgpp_mlp_precondition(dmrgpp_mlp_handle m, const double* diag, const double* r, double theta,
                            double rnorm, double* t, size_t n, void* stream)
{
	DMRGPP_TRACE("dmrgpp_mlp_precondition");
	return dmrgpp::mlp_precondition(m, diag, r, theta, rnorm, t, n, static_cast<cudaStream_t>(stream));
}

int dmrgpp_mlp_precondition_group(dmrgpp_mlp_handle m, const double* diag, const double* r,
                                  const long long* sector_start, const double* theta,
                                  const double* rnorm, int nsectors, double* t, size_t n, void* stream)
{
	DMRGPP_TRACE("dmrgpp_mlp_precondition_group");
	return dmrgpp::mlp_precondition_group(m, diag, r, sector_start, theta, rnorm, nsectors, t, n,
	                                      static_cast<cudaStream_t>(stream));
}

} // extern "C"
