// C ABI of the Kronecker H*x engine (include/dmrgpp_kron.h).
#include "dmrgpp_kron.h"
#include "kron_gemm.cuh"
#include "kron_plan.h"

#include <cuda_runtime.h>

#include <cstring>
#include <new>
#include <string>
#include <vector>

#define DMRGPP_VERSION_STRING "dmrgpp-b200 0.1"

struct dmrgpp_kron_s {
	int                 device     = 0;
	cudaStream_t        stream     = nullptr;
	int                 precision  = DMRGPP_FP64;
	dmrgpp::KronPlan    plan;
	double*             d_ops   = nullptr; // packed Bstack_j and A^T blocks
	double*             d_bx    = nullptr; // pass-1 output (scratch)
	double*             d_x     = nullptr; // staging for host-pointer applies
	double*             d_y     = nullptr;
	dmrgpp::GemmSeg*    d_seg1  = nullptr;
	dmrgpp::GemmSeg*    d_seg2  = nullptr;
	dmrgpp::GemmTile*   d_tile1 = nullptr;
	dmrgpp::GemmTile*   d_tile2 = nullptr;
	void*               d_lists = nullptr; // one allocation behind the four lists
	std::string         err;
};

namespace {

thread_local std::string g_create_error;

// Restores the caller's current device on scope exit.
struct DeviceGuard {
	int  prev = -1;
	bool ok   = true;
	explicit DeviceGuard(int dev)
	{
		if (cudaGetDevice(&prev) != cudaSuccess) {
			ok = false;
			return;
		}
		if (dev >= 0 && dev != prev)
			ok = cudaSetDevice(dev) == cudaSuccess;
	}
	~DeviceGuard()
	{
		int cur = -1;
		if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev)
			cudaSetDevice(prev);
	}
};

int fail(dmrgpp_kron_handle h, int status, const std::string& msg)
{
	if (h)
		h->err = msg;
	else
		g_create_error = msg;
	return status;
}

int cuda_fail(dmrgpp_kron_handle h, cudaError_t e, const char* where)
{
	const int status = (e == cudaErrorMemoryAllocation) ? DMRGPP_OOM : DMRGPP_CUDA_ERROR;
	return fail(h, status, std::string(where) + ": " + cudaGetErrorString(e));
}

void release(dmrgpp_kron_handle h)
{
	if (!h)
		return;
	cudaFree(h->d_ops);
	cudaFree(h->d_bx);
	cudaFree(h->d_x);
	cudaFree(h->d_y);
	cudaFree(h->d_lists);
	h->d_ops = h->d_bx = h->d_x = h->d_y = nullptr;
	h->d_lists                           = nullptr;
	h->stream                            = nullptr;
}

// Tile shape for a sector: small sectors need small tiles to fill the SMs.
void pick_tile(const dmrgpp_kron_desc* d, int& bm, int& bn)
{
	size_t maxs = 0;
	for (size_t p = 0; p < d->npatches; ++p) {
		maxs = d->left_patch_size[p] > maxs ? d->left_patch_size[p] : maxs;
		maxs = d->right_patch_size[p] > maxs ? d->right_patch_size[p] : maxs;
	}
	if (maxs <= 192) {
		bm = bn = 32;
	} else {
		bm = bn = 64;
	}
}

int check_desc(const dmrgpp_kron_desc* d)
{
	if (!d)
		return fail(nullptr, DMRGPP_INVALID_ARG, "null descriptor");
	if (d->precision != DMRGPP_FP64 && d->precision != DMRGPP_SPLIT_BF16
	    && d->precision != DMRGPP_TF32X3)
		return fail(nullptr, DMRGPP_INVALID_ARG, "unknown precision mode");
	if (!d->left_patch_size || !d->right_patch_size)
		return fail(nullptr, DMRGPP_INVALID_ARG, "null patch-size array");
	return DMRGPP_OK;
}

} // namespace

extern "C" {

const char* dmrgpp_version(void) { return DMRGPP_VERSION_STRING; }

const char* dmrgpp_kron_last_error(dmrgpp_kron_handle h)
{
	return h ? h->err.c_str() : g_create_error.c_str();
}

int dmrgpp_kron_plan_info_get(const dmrgpp_kron_desc* d, dmrgpp_kron_plan_info* info)
{
	if (int rc = check_desc(d))
		return rc;
	if (!info)
		return fail(nullptr, DMRGPP_INVALID_ARG, "null info");
	int bm, bn;
	pick_tile(d, bm, bn);
	dmrgpp::KronPlan plan;
	std::string      msg = dmrgpp::build_kron_plan(d->noperator,
                                              d->npatches,
                                              d->left_patch_size,
                                              d->right_patch_size,
                                              d->Amatrix,
                                              d->ld_Amatrix,
                                              d->Bmatrix,
                                              d->ld_Bmatrix,
                                              bm,
                                              bn,
                                              plan,
                                              nullptr);
	if (!msg.empty())
		return fail(nullptr, DMRGPP_INVALID_ARG, msg);
	info->ntriples       = plan.triples.size();
	info->dim            = size_t(plan.dim());
	info->f_alg          = plan.f_alg;
	info->operator_bytes = size_t(plan.op_elems) * sizeof(double);
	info->bx_bytes       = size_t(plan.bx_elems) * sizeof(double);
	info->pass1_tiles    = plan.tile1.size();
	info->pass2_tiles    = plan.tile2.size();
	return DMRGPP_OK;
}

int dmrgpp_kron_create(const dmrgpp_kron_desc* d, dmrgpp_kron_handle* out)
{
	if (!out)
		return fail(nullptr, DMRGPP_INVALID_ARG, "null output handle");
	*out = nullptr;
	if (int rc = check_desc(d))
		return rc;
	if (d->precision != DMRGPP_FP64)
		return fail(nullptr, DMRGPP_NOT_SUPPORTED, "precision mode not built into this library");

	dmrgpp_kron_handle h = new (std::nothrow) dmrgpp_kron_s();
	if (!h)
		return fail(nullptr, DMRGPP_OOM, "host allocation failed");
	h->precision = d->precision;

	int bm, bn;
	pick_tile(d, bm, bn);
	std::vector<double> pack;
	std::string         msg = dmrgpp::build_kron_plan(d->noperator,
                                              d->npatches,
                                              d->left_patch_size,
                                              d->right_patch_size,
                                              d->Amatrix,
                                              d->ld_Amatrix,
                                              d->Bmatrix,
                                              d->ld_Bmatrix,
                                              bm,
                                              bn,
                                              h->plan,
                                              &pack);
	if (!msg.empty()) {
		delete h;
		return fail(nullptr, DMRGPP_INVALID_ARG, msg);
	}

	if (d->device >= 0) {
		h->device = d->device;
	} else if (cudaGetDevice(&h->device) != cudaSuccess) {
		delete h;
		return fail(nullptr, DMRGPP_CUDA_ERROR, "no CUDA device");
	}
	DeviceGuard g(h->device);
	auto        bail = [&](cudaError_t e, const char* where) {
                int rc = cuda_fail(nullptr, e, where);
                release(h);
                delete h;
                return rc;
	};
	if (!g.ok)
		return bail(cudaErrorInvalidDevice, "cudaSetDevice");

	cudaError_t e = dmrgpp::init_grouped_dgemm();
	if (e != cudaSuccess)
		return bail(e, "kernel attributes");
	// NULL is the CUDA default stream, as for cuBLAS handles
	h->stream = static_cast<cudaStream_t>(d->stream);

	const auto&  P   = h->plan;
	const size_t dim = size_t(P.dim());
	if ((e = cudaMalloc(&h->d_ops, size_t(P.op_elems ? P.op_elems : 1) * sizeof(double))))
		return bail(e, "cudaMalloc(operators)");
	if ((e = cudaMalloc(&h->d_bx, size_t(P.bx_elems ? P.bx_elems : 1) * sizeof(double))))
		return bail(e, "cudaMalloc(BX)");
	if ((e = cudaMalloc(&h->d_x, dim * sizeof(double))))
		return bail(e, "cudaMalloc(x)");
	if ((e = cudaMalloc(&h->d_y, dim * sizeof(double))))
		return bail(e, "cudaMalloc(y)");

	const size_t nseg  = P.seg1.size() + P.seg2.size();
	const size_t ntile = P.tile1.size() + P.tile2.size();
	const size_t bytes = nseg * sizeof(dmrgpp::GemmSeg) + ntile * sizeof(dmrgpp::GemmTile);
	if ((e = cudaMalloc(&h->d_lists, bytes ? bytes : 16)))
		return bail(e, "cudaMalloc(lists)");
	std::vector<unsigned char> lists(bytes);
	unsigned char*             p = lists.data();
	auto put = [&](const void* src, size_t n) {
		if (n)
			std::memcpy(p, src, n);
		void* dev = static_cast<unsigned char*>(h->d_lists) + (p - lists.data());
		p += n;
		return dev;
	};
	h->d_seg1  = (dmrgpp::GemmSeg*)put(P.seg1.data(), P.seg1.size() * sizeof(dmrgpp::GemmSeg));
	h->d_seg2  = (dmrgpp::GemmSeg*)put(P.seg2.data(), P.seg2.size() * sizeof(dmrgpp::GemmSeg));
	h->d_tile1 = (dmrgpp::GemmTile*)put(P.tile1.data(), P.tile1.size() * sizeof(dmrgpp::GemmTile));
	h->d_tile2 = (dmrgpp::GemmTile*)put(P.tile2.data(), P.tile2.size() * sizeof(dmrgpp::GemmTile));
	if (bytes && (e = cudaMemcpy(h->d_lists, lists.data(), bytes, cudaMemcpyHostToDevice)))
		return bail(e, "upload lists");
	if (!pack.empty()
	    && (e = cudaMemcpy(h->d_ops, pack.data(), pack.size() * sizeof(double), cudaMemcpyHostToDevice)))
		return bail(e, "upload operators");
	*out = h;
	return DMRGPP_OK;
}

int dmrgpp_kron_destroy(dmrgpp_kron_handle h)
{
	if (!h)
		return DMRGPP_OK;
	DeviceGuard g(h->device);
	cudaStreamSynchronize(h->stream);
	release(h);
	delete h;
	return DMRGPP_OK;
}

int dmrgpp_kron_dim(dmrgpp_kron_handle h, size_t* dim)
{
	if (!h || !dim)
		return fail(h, DMRGPP_INVALID_ARG, "null argument");
	*dim = size_t(h->plan.dim());
	return DMRGPP_OK;
}

int dmrgpp_kron_flops(dmrgpp_kron_handle h, double* f)
{
	if (!h || !f)
		return fail(h, DMRGPP_INVALID_ARG, "null argument");
	*f = h->plan.f_alg;
	return DMRGPP_OK;
}

int dmrgpp_kron_apply(dmrgpp_kron_handle h, const double* x, double* y, int on_device)
{
	if (!h)
		return fail(nullptr, DMRGPP_INVALID_ARG, "null handle");
	if (!x || !y)
		return fail(h, DMRGPP_INVALID_ARG, "null vector");
	DeviceGuard g(h->device);
	if (!g.ok)
		return cuda_fail(h, cudaErrorInvalidDevice, "cudaSetDevice");
	const auto&   P   = h->plan;
	const size_t  dim = size_t(P.dim());
	const double* X   = on_device ? x : h->d_x;
	double*       Y   = on_device ? y : h->d_y;
	cudaError_t   e;
	if (!on_device
	    && (e = cudaMemcpyAsync(h->d_x, x, dim * sizeof(double), cudaMemcpyHostToDevice, h->stream)))
		return cuda_fail(h, e, "copy x to device");

	dmrgpp::GemmArgs a1 { h->d_ops, X, h->d_bx, h->d_seg1, h->d_tile1, int(P.tile1.size()) };
	if ((e = dmrgpp::launch_grouped_dgemm(a1, P.bm, P.bn, h->stream)))
		return cuda_fail(h, e, "pass 1 launch");
	dmrgpp::GemmArgs a2 { h->d_bx, h->d_ops, Y, h->d_seg2, h->d_tile2, int(P.tile2.size()) };
	if ((e = dmrgpp::launch_grouped_dgemm(a2, P.bm, P.bn, h->stream)))
		return cuda_fail(h, e, "pass 2 launch");

	if (!on_device) {
		if ((e = cudaMemcpyAsync(y, h->d_y, dim * sizeof(double), cudaMemcpyDeviceToHost, h->stream)))
			return cuda_fail(h, e, "copy y to host");
		if ((e = cudaStreamSynchronize(h->stream)))
			return cuda_fail(h, e, "apply");
	}
	return DMRGPP_OK;
}

} // extern "C"
