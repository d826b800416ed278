// Patch-wise wave-function transformation on the device (dmrgpp_wft_* in
// dmrgpp_kron.h, plan in wft_plan.h): two grouped FP64 GEMM launches per
// apply, on the FP64 tensor pipe (kron_gemm.cuh).
#include "devmem.h"
#include "trace.h"
#include "dmrgpp_kron.h"
#include "kron_gemm.cuh"
#include "wft_plan.h"

#include <cuda_runtime.h>

#include <cstring>
#include <new>
#include <string>
#include <vector>

struct dmrgpp_wft_s {
	int                 device = 0;
	cudaStream_t        stream = nullptr;
	dmrgpp::WftPlan     plan;
	double*             d_ops  = nullptr; // packed WR and WL^T blocks
	double*             d_t    = nullptr; // pass-A result T
	double*             d_x    = nullptr; // staging for host-pointer applies
	double*             d_y    = nullptr;
	void*               d_lists = nullptr;
	dmrgpp::GemmSeg*    segA = nullptr;
	dmrgpp::GemmSeg*    segB = nullptr;
	dmrgpp::GemmTile*   tileA = nullptr;
	dmrgpp::GemmTile*   tileB = nullptr;
	std::string         err;
};

namespace {

thread_local std::string g_wft_error;

int wft_fail(dmrgpp_wft_handle h, int status, const std::string& msg)
{
	(h ? h->err : g_wft_error) = msg;
	return status;
}

int wft_cuda(dmrgpp_wft_handle h, cudaError_t e, const char* where)
{
	return wft_fail(h, e == cudaErrorMemoryAllocation ? DMRGPP_OOM : DMRGPP_CUDA_ERROR,
	                std::string(where) + ": " + cudaGetErrorString(e));
}

struct Device {
	int  prev = -1;
	bool ok   = false;
	explicit Device(int dev)
	{
		ok = cudaGetDevice(&prev) == cudaSuccess && (dev == prev || cudaSetDevice(dev) == cudaSuccess);
	}
	~Device()
	{
		int cur = -1;
		if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev)
			cudaSetDevice(prev);
	}
};

void wft_release(dmrgpp_wft_handle h)
{
	cudaDeviceSynchronize();
	dmrgpp::dev_free(h->d_ops);
	dmrgpp::dev_free(h->d_t);
	dmrgpp::dev_free(h->d_x);
	dmrgpp::dev_free(h->d_y);
	dmrgpp::dev_free(h->d_lists);
	h->d_ops = h->d_t = h->d_x = h->d_y = nullptr;
	h->d_lists                          = nullptr;
}

int enqueue(dmrgpp_wft_handle h, const double* x, double* y)
{
	const auto&       P = h->plan;
	dmrgpp::GemmArgs  a {};
	a.A      = h->d_ops;
	a.B      = x;
	a.C      = h->d_t;
	a.segs   = h->segA;
	a.tiles  = h->tileA;
	a.ntiles = int(P.tileA.size());
	cudaError_t e = dmrgpp::launch_grouped_dgemm(a, P.bm, P.bn, h->stream);
	if (e == cudaSuccess) {
		a.A      = h->d_t;
		a.B      = h->d_ops;
		a.C      = y;
		a.segs   = h->segB;
		a.tiles  = h->tileB;
		a.ntiles = int(P.tileB.size());
		e        = dmrgpp::launch_grouped_dgemm(a, P.bm, P.bn, h->stream);
	}
	return e == cudaSuccess ? DMRGPP_OK : wft_cuda(h, e, "transformation launch");
}

} // namespace

extern "C" {

int dmrgpp_wft_create(const dmrgpp_wft_desc* d, dmrgpp_wft_handle* out)
{
	DMRGPP_TRACE("dmrgpp_wft_create");
	if (!out)
		return wft_fail(nullptr, DMRGPP_INVALID_ARG, "null output handle");
	*out = nullptr;
	if (!d)
		return wft_fail(nullptr, DMRGPP_INVALID_ARG, "null descriptor");
	dmrgpp_wft_handle h = new (std::nothrow) dmrgpp_wft_s();
	if (!h)
		return wft_fail(nullptr, DMRGPP_OOM, "host allocation failed");
	std::vector<double> packed;
	std::string         msg = dmrgpp::build_wft_plan(*d, h->plan, &packed);
	if (!msg.empty()) {
		delete h;
		return wft_fail(nullptr, DMRGPP_INVALID_ARG, msg);
	}
	if (d->device >= 0)
		h->device = d->device;
	else if (cudaGetDevice(&h->device) != cudaSuccess) {
		delete h;
		return wft_fail(nullptr, DMRGPP_CUDA_ERROR, "no CUDA device");
	}
	Device g(h->device);
	h->stream   = static_cast<cudaStream_t>(d->stream);
	auto bail   = [&](cudaError_t e, const char* where) {
                const int rc = wft_cuda(nullptr, e, where);
                wft_release(h);
                delete h;
                return rc;
	};
	if (!g.ok)
		return bail(cudaErrorInvalidDevice, "cudaSetDevice");
	const auto& P = h->plan;
	cudaError_t e;
	if ((e = dmrgpp::init_grouped_dgemm()))
		return bail(e, "kernel attributes");
	auto bytes = [](long long n) { return size_t(n > 0 ? n : 1) * sizeof(double); };
	if ((e = dmrgpp::dev_malloc(&h->d_ops, bytes(P.op_elems))) || (e = dmrgpp::dev_malloc(&h->d_t, bytes(P.t_elems)))
	    || (e = dmrgpp::dev_malloc(&h->d_x, bytes(P.dim_in()))) || (e = dmrgpp::dev_malloc(&h->d_y, bytes(P.dim_out()))))
		return bail(e, "device allocation");
	if (P.op_elems > 0
	    && (e = dmrgpp::upload_sync(h->d_ops, packed.data(), size_t(P.op_elems) * sizeof(double), h->stream)))
		return bail(e, "upload transformation blocks");
	// the four launch lists in one allocation, 16-byte aligned parts
	std::vector<unsigned char> lists;
	std::vector<size_t>        offs;
	auto add = [&](const void* src, size_t n) {
		offs.push_back(lists.size());
		lists.resize(lists.size() + ((n + 15) / 16) * 16);
		if (n)
			std::memcpy(lists.data() + offs.back(), src, n);
	};
	add(P.segA.data(), P.segA.size() * sizeof(dmrgpp::GemmSeg));
	add(P.segB.data(), P.segB.size() * sizeof(dmrgpp::GemmSeg));
	add(P.tileA.data(), P.tileA.size() * sizeof(dmrgpp::GemmTile));
	add(P.tileB.data(), P.tileB.size() * sizeof(dmrgpp::GemmTile));
	if ((e = dmrgpp::dev_malloc(&h->d_lists, lists.empty() ? 16 : lists.size())))
		return bail(e, "device allocation (lists)");
	if (!lists.empty() && (e = dmrgpp::upload_sync(h->d_lists, lists.data(), lists.size(), h->stream)))
		return bail(e, "upload lists");
	unsigned char* base = static_cast<unsigned char*>(h->d_lists);
	h->segA  = reinterpret_cast<dmrgpp::GemmSeg*>(base + offs[0]);
	h->segB  = reinterpret_cast<dmrgpp::GemmSeg*>(base + offs[1]);
	h->tileA = reinterpret_cast<dmrgpp::GemmTile*>(base + offs[2]);
	h->tileB = reinterpret_cast<dmrgpp::GemmTile*>(base + offs[3]);
	*out     = h;
	return DMRGPP_OK;
}

int dmrgpp_wft_apply(dmrgpp_wft_handle h, const double* x, double* y, int on_device)
{
	DMRGPP_TRACE("dmrgpp_wft_apply");
	if (!h)
		return wft_fail(nullptr, DMRGPP_INVALID_ARG, "null handle");
	if (!x || !y)
		return wft_fail(h, DMRGPP_INVALID_ARG, "null vector");
	Device g(h->device);
	if (!g.ok)
		return wft_cuda(h, cudaErrorInvalidDevice, "cudaSetDevice");
	const size_t din = size_t(h->plan.dim_in()), dout = size_t(h->plan.dim_out());
	cudaError_t  e;
	if (on_device)
		return enqueue(h, x, y);
	if ((e = cudaMemcpyAsync(h->d_x, x, din * sizeof(double), cudaMemcpyHostToDevice, h->stream)))
		return wft_cuda(h, e, "copy x to device");
	if (int rc = enqueue(h, h->d_x, h->d_y))
		return rc;
	if ((e = cudaMemcpyAsync(y, h->d_y, dout * sizeof(double), cudaMemcpyDeviceToHost, h->stream))
	    || (e = cudaStreamSynchronize(h->stream)))
		return wft_cuda(h, e, "copy y to host");
	return DMRGPP_OK;
}

int dmrgpp_wft_dims(dmrgpp_wft_handle h, size_t* dim_in, size_t* dim_out)
{
	if (!h || !dim_in || !dim_out)
		return wft_fail(h, DMRGPP_INVALID_ARG, "null argument");
	*dim_in  = size_t(h->plan.dim_in());
	*dim_out = size_t(h->plan.dim_out());
	return DMRGPP_OK;
}

int dmrgpp_wft_flops(dmrgpp_wft_handle h, double* flops)
{
	if (!h || !flops)
		return wft_fail(h, DMRGPP_INVALID_ARG, "null argument");
	*flops = h->plan.flops;
	return DMRGPP_OK;
}

int dmrgpp_wft_destroy(dmrgpp_wft_handle h)
{
	if (!h)
		return DMRGPP_OK;
	Device g(h->device);
	wft_release(h);
	delete h;
	return DMRGPP_OK;
}

const char* dmrgpp_wft_last_error(dmrgpp_wft_handle h) { return h ? h->err.c_str() : g_wft_error.c_str(); }

} // extern "C"
