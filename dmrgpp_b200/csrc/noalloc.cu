// dmrgpp_kron_apply_noalloc: one-shot H*x that performs no device allocation.
//
// Who needs it: callers that must not call cudaMalloc -- code that runs while
// another component owns all device memory through its own allocator, code
// that may only enqueue work on a stream it was handed, or a host runtime
// that forbids allocation after its start-up phase.  dmrgpp_kron_create
// allocates the packed operators, the pass-1 buffer and the launch lists with
// cudaMalloc; this entry point instead places all three in one file-scope
// device array of fixed size, g_noalloc_scratch, which the CUDA module
// reserves when the library is loaded on a device and keeps until the process
// exits.
//
// The same planning (build_kron_plan) and the same grouped-GEMM kernels as
// dmrgpp_kron_create + dmrgpp_kron_apply are used; only the home of the
// scratch differs.
#include "dmrgpp_kron.h"
#include "kron_gemm.cuh"
#include "kron_plan.h"

#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <string>
#include <vector>

namespace {

constexpr size_t kScratchBytes = DMRGPP_NOALLOC_SCRATCH_BYTES;
constexpr int    kMaxDevices   = 64;

// The scratch.  In host code this name is only a stand-in for the device
// array: its device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) double g_noalloc_scratch[kScratchBytes / sizeof(double)];

std::mutex  g_setup_mutex;
double*     g_scratch_ptr[kMaxDevices] = {};
bool        g_kernels_ready[kMaxDevices] = {};
thread_local std::string g_noalloc_error;

int noalloc_fail(int status, const std::string& msg)
{
	g_noalloc_error = msg;
	return status;
}

// Once per device, with that device current: the array's device address and
// the kernels' shared-memory attribute.
cudaError_t setup_device(int dev, double** out)
{
	std::lock_guard<std::mutex> lock(g_setup_mutex);
	if (!g_scratch_ptr[dev]) {
		void*       p = nullptr;
		cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
		if (e != cudaSuccess)
			return e;
		g_scratch_ptr[dev] = static_cast<double*>(p);
	}
	if (!g_kernels_ready[dev]) {
		cudaError_t e = dmrgpp::init_grouped_dgemm();
		if (e != cudaSuccess)
			return e;
		g_kernels_ready[dev] = true;
	}
	*out = g_scratch_ptr[dev];
	return cudaSuccess;
}

} // namespace

extern "C" {

const char* dmrgpp_kron_noalloc_last_error(void) { return g_noalloc_error.c_str(); }

int dmrgpp_kron_apply_noalloc(const dmrgpp_kron_desc* d, const double* x, double* y)
{
	if (!d)
		return noalloc_fail(DMRGPP_INVALID_ARG, "null descriptor");
	if (!x || !y)
		return noalloc_fail(DMRGPP_INVALID_ARG, "null vector");
	if (d->precision != DMRGPP_FP64)
		return noalloc_fail(DMRGPP_NOT_SUPPORTED, "only FP64 is available without allocation");
	if (!d->left_patch_size || !d->right_patch_size)
		return noalloc_fail(DMRGPP_INVALID_ARG, "null patch-size array");

	size_t maxs = 0;
	for (size_t p = 0; p < d->npatches; ++p) {
		maxs = d->left_patch_size[p] > maxs ? d->left_patch_size[p] : maxs;
		maxs = d->right_patch_size[p] > maxs ? d->right_patch_size[p] : maxs;
	}
	const int           tile = maxs <= 192 ? 32 : 64;
	dmrgpp::KronPlan    plan;
	dmrgpp::PackBuffer  pack;
	std::string         msg = dmrgpp::build_kron_plan(d->noperator,
                                              d->npatches,
                                              d->left_patch_size,
                                              d->right_patch_size,
                                              d->Amatrix,
                                              d->ld_Amatrix,
                                              d->Bmatrix,
                                              d->ld_Bmatrix,
                                              tile,
                                              tile,
                                              plan,
                                              &pack);
	if (!msg.empty())
		return noalloc_fail(DMRGPP_INVALID_ARG, msg);

	// scratch layout: [packed operators | BX | segments and tiles]
	const size_t ops_bytes  = size_t(plan.op_elems) * sizeof(double);
	const size_t bx_bytes   = size_t(plan.bx_elems) * sizeof(double);
	const size_t seg_bytes  = (plan.seg1.size() + plan.seg2.size()) * sizeof(dmrgpp::GemmSeg);
	const size_t tile_bytes = (plan.tile1.size() + plan.tile2.size()) * sizeof(dmrgpp::GemmTile);
	const size_t need       = ops_bytes + bx_bytes + seg_bytes + tile_bytes;
	if (need > kScratchBytes)
		return noalloc_fail(DMRGPP_INVALID_ARG,
		                    "sector needs " + std::to_string(need)
		                        + " bytes of scratch; the static scratch of "
		                          "dmrgpp_kron_apply_noalloc holds "
		                        + std::to_string(kScratchBytes) + " bytes");

	int prev = -1;
	if (cudaGetDevice(&prev) != cudaSuccess)
		return noalloc_fail(DMRGPP_CUDA_ERROR, "no CUDA device");
	const int dev = d->device >= 0 ? d->device : prev;
	if (dev >= kMaxDevices)
		return noalloc_fail(DMRGPP_INVALID_ARG, "device ordinal out of range");
	if (dev != prev && cudaSetDevice(dev) != cudaSuccess)
		return noalloc_fail(DMRGPP_CUDA_ERROR, "cudaSetDevice failed");
	auto restore = [&](int rc) {
		if (dev != prev)
			cudaSetDevice(prev);
		return rc;
	};

	// The operator and list uploads read host memory that this call frees
	// before it returns; a capture would record copies from freed memory.
	cudaStream_t                stream = static_cast<cudaStream_t>(d->stream);
	cudaStreamCaptureStatus     cap    = cudaStreamCaptureStatusNone;
	cudaError_t                 e      = cudaStreamIsCapturing(stream, &cap);
	if (e != cudaSuccess)
		return restore(noalloc_fail(DMRGPP_CUDA_ERROR,
		                            std::string("stream query: ") + cudaGetErrorString(e)));
	if (cap != cudaStreamCaptureStatusNone)
		return restore(noalloc_fail(DMRGPP_NOT_SUPPORTED,
		                            "the stream is being captured: this call uploads from host "
		                            "memory that it frees before returning"));

	double* base = nullptr;
	e            = setup_device(dev, &base);
	if (e != cudaSuccess)
		return restore(noalloc_fail(DMRGPP_CUDA_ERROR,
		                            std::string("scratch set-up: ") + cudaGetErrorString(e)));

	double*      ops    = base;
	double*      bx     = base + plan.op_elems;
	auto*        segs   = reinterpret_cast<dmrgpp::GemmSeg*>(bx + plan.bx_elems);
	auto*        tiles  = reinterpret_cast<dmrgpp::GemmTile*>(
                reinterpret_cast<unsigned char*>(segs) + seg_bytes);

	// host staging of the lists, then pageable-memory copies: each returns
	// once its source has been read, so the host vectors may go out of scope
	std::vector<unsigned char> lists(seg_bytes + tile_bytes);
	unsigned char*             p = lists.data();
	auto put = [&](const void* src, size_t n) {
		if (n)
			memcpy(p, src, n);
		p += n;
	};
	put(plan.seg1.data(), plan.seg1.size() * sizeof(dmrgpp::GemmSeg));
	put(plan.seg2.data(), plan.seg2.size() * sizeof(dmrgpp::GemmSeg));
	put(plan.tile1.data(), plan.tile1.size() * sizeof(dmrgpp::GemmTile));
	put(plan.tile2.data(), plan.tile2.size() * sizeof(dmrgpp::GemmTile));

	// Every byte read by the passes is written first in this call (operators
	// and lists by these copies, BX rows by pass 1, y by pass 2), so nothing
	// left by an earlier call needs clearing.
	if (ops_bytes && (e = cudaMemcpyAsync(ops, pack.data(), ops_bytes, cudaMemcpyHostToDevice, stream)))
		return restore(noalloc_fail(DMRGPP_CUDA_ERROR,
		                            std::string("operator upload: ") + cudaGetErrorString(e)));
	if (!lists.empty()
	    && (e = cudaMemcpyAsync(segs, lists.data(), lists.size(), cudaMemcpyHostToDevice, stream)))
		return restore(noalloc_fail(DMRGPP_CUDA_ERROR,
		                            std::string("list upload: ") + cudaGetErrorString(e)));

	const dmrgpp::GemmSeg*  seg1  = segs;
	const dmrgpp::GemmSeg*  seg2  = segs + plan.seg1.size();
	const dmrgpp::GemmTile* tile1 = tiles;
	const dmrgpp::GemmTile* tile2 = tiles + plan.tile1.size();
	dmrgpp::GemmArgs        a1 { ops, x, bx, seg1, tile1, int(plan.tile1.size()) };
	if ((e = dmrgpp::launch_grouped_dgemm(a1, plan.bm, plan.bn, stream)))
		return restore(noalloc_fail(DMRGPP_CUDA_ERROR,
		                            std::string("pass 1: ") + cudaGetErrorString(e)));
	dmrgpp::GemmArgs a2 { bx, ops, y, seg2, tile2, int(plan.tile2.size()) };
	if ((e = dmrgpp::launch_grouped_dgemm(a2, plan.bm, plan.bn, stream)))
		return restore(noalloc_fail(DMRGPP_CUDA_ERROR,
		                            std::string("pass 2: ") + cudaGetErrorString(e)));
	return restore(DMRGPP_OK);
}

} // extern "C"
