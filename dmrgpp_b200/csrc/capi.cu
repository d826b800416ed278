// C ABI of the Kronecker H*x engine (include/dmrgpp_kron.h).
#include "dmrgpp_kron.h"
#include "trace.h"
#include "kron_gemm.cuh"
#include "kron_fused.cuh"
#include "kron_persistent.cuh"
#include "kron_plan.h"
#include "devmem.h"
#include "handle.h"
#include "tc_gemm.cuh"

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <thread>
#include <climits>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#define DMRGPP_VERSION_STRING "dmrgpp-b200 0.1"



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
	// nothing of the handle may still run: its memory and error word are reused
	cudaDeviceSynchronize();
	dmrgpp::release_lanczos(h);
	dmrgpp::release_davidson(h);
	dmrgpp::release_group(h);
	dmrgpp::dev_free(h->d_diag);
	h->d_diag = nullptr;
	dmrgpp::dev_free(h->d_cx);
	h->d_cx = nullptr;
	dmrgpp::dev_free(h->m_ops_hi);
	dmrgpp::dev_free(h->m_ops_lo);
	dmrgpp::dev_free(h->m_xs_hi);
	dmrgpp::dev_free(h->m_xs_lo);
	dmrgpp::dev_free(h->m_bxs_hi);
	dmrgpp::dev_free(h->m_bxs_lo);
	dmrgpp::dev_free(h->m_xmap);
	dmrgpp::dev_free(h->m_lists);
	dmrgpp::dev_free(h->m_partial);
	dmrgpp::dev_free(h->m_arrive);
	h->m_partial = nullptr;
	h->m_arrive  = nullptr;
	h->m_ops_hi = h->m_ops_lo = h->m_xs_hi = h->m_xs_lo = h->m_bxs_hi = h->m_bxs_lo = nullptr;
	h->m_xmap   = nullptr;
	h->m_lists  = nullptr;
	h->m_tsec1 = h->m_tsec2 = nullptr;
	h->mixed_ready = false;
	dmrgpp::dev_free(h->d_ops);
	dmrgpp::dev_free(h->d_bx);
	dmrgpp::dev_free(h->d_x);
	dmrgpp::dev_free(h->d_y);
	dmrgpp::dev_free(h->d_lists);
	dmrgpp::dev_free(h->d_ctr);
	dmrgpp::dev_free(h->d_part);
	dmrgpp::dev_free(h->d_flists);
	h->d_flists = nullptr;
	h->d_fitems = nullptr;
	h->d_funits = nullptr;
	dmrgpp::error_word_free(h->err_host);
	h->err_host = h->err_dev = nullptr;
	h->d_ctr                 = nullptr;
	h->d_part                = nullptr;
	h->d_ops = h->d_bx = h->d_x = h->d_y = nullptr;
	h->d_lists                           = nullptr;
	h->stream                            = nullptr;
}

// Tile shape for a sector: small sectors need small tiles to fill the SMs.
void pick_tile_sizes(size_t np, const size_t* l, const size_t* r, int& bm, int& bn)
{
	size_t maxs = 0;
	for (size_t p = 0; p < np; ++p) {
		maxs = l[p] > maxs ? l[p] : maxs;
		maxs = r[p] > maxs ? r[p] : maxs;
	}
	if (maxs <= 192) {
		bm = bn = 32;
	} else {
		bm = bn = 64;
	}
}

void pick_tile(const dmrgpp_kron_desc* d, int& bm, int& bn)
{
	pick_tile_sizes(d->npatches, d->left_patch_size, d->right_patch_size, bm, bn);
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no
// direct libcuda dependency)
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
	static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
	if (!fn) {
		void*                           p = nullptr;
		cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
		if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess
		    && q == cudaDriverEntryPointSuccess)
			fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
	}
	return fn;
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

// After the stream has drained: a wait inside a kernel that gave up (the
// persistent kernel leaves its counters dirty); report it and restore a
// clean state.
int check_error_word(dmrgpp_kron_handle h)
{
	if (!h->err_host || *reinterpret_cast<volatile int*>(h->err_host) == 0)
		return DMRGPP_OK;
	*h->err_host      = 0;
	const size_t nctr = 3 + h->plan.np + size_t(h->plan.n_split_tiles);
	cudaMemsetAsync(h->d_ctr, 0, nctr * sizeof(unsigned), h->stream);
	if (h->m_arrive)
		cudaMemsetAsync(h->m_arrive, 0, size_t(std::max(h->plan.mixed.n_split_tiles, 1)) * sizeof(unsigned),
		                h->stream);
	cudaStreamSynchronize(h->stream);
	return fail(h, DMRGPP_TIMEOUT, "a bounded wait in an H*x kernel gave up; result invalid");
}

} // namespace

namespace dmrgpp {

int handle_fail(dmrgpp_kron_handle h, int status, const std::string& msg)
{
	return fail(h, status, msg);
}

int mixed_apply_device(dmrgpp_kron_handle h, const double* X, double* Y, const StepIO* io)
{
	const MixedPlan& mp = h->plan.mixed;
	cudaError_t      e;
	if ((e = tc_split_x(X, h->m_xmap, h->m_xs_hi, h->m_xs_lo, h->plan.dim(), h->stream, io)))
		return cuda_fail(h, e, "x split launch");
	TcArgs a1 {};
	const CUtensorMap* tm = reinterpret_cast<const CUtensorMap*>(h->m_tmap);
	a1.A_hi   = tm[0];
	a1.A_lo   = tm[1];
	a1.B_hi   = tm[2];
	a1.B_lo   = tm[3];
	a1.C_hi_map = tm[8];
	a1.C_lo_map = tm[9];
	a1.C_hi   = h->m_bxs_hi;
	a1.C_lo   = h->m_bxs_lo;
	a1.segs   = h->m_seg1;
	a1.tiles  = h->m_tile1;
	a1.ntiles = int(mp.tile1.size());
	a1.grid   = h->m_grid1;
	a1.test_unarmed = h->test_stall;
	a1.starts = h->m_starts1;
	a1.error  = h->err_dev;
	a1.tile_sector   = h->m_tsec1;
	a1.sector_active = h->m_tsec1 ? h->sector_active : nullptr;
	if ((e = tc_launch(a1, mp.bn, true, h->stream)))
		return cuda_fail(h, e, "tensor-core pass 1 launch");
	TcArgs a2 {};
	a2.A_hi   = tm[4];
	a2.A_lo   = tm[5];
	a2.B_hi   = tm[6];
	a2.B_lo   = tm[7];
	a2.Cd     = Y;
	a2.io     = io;
	a2.segs   = h->m_seg2;
	a2.tiles  = h->m_tile2;
	a2.ntiles = int(mp.tile2.size());
	a2.grid   = h->m_grid2;
	a2.starts = h->m_starts2;
	a2.tile_sector   = h->m_tsec2;
	a2.sector_active = h->m_tsec2 ? h->sector_active : nullptr;
	a2.partial = h->m_partial;
	a2.arrive  = h->m_arrive;
	a2.error  = h->err_dev;
	if ((e = tc_launch(a2, mp.bn, false, h->stream)))
		return cuda_fail(h, e, "tensor-core pass 2 launch");
	return DMRGPP_OK;
}

int kron_apply_device(dmrgpp_kron_handle h, const double* X, double* Y, const StepIO* io)
{
	if (h->precision == DMRGPP_TF32X3)
		return mixed_apply_device(h, X, Y, io);
	const auto& P = h->plan;
	cudaError_t e;
	if (h->cfg >= kNumTileCfgs) {
		dmrgpp::FusedArgs fa {};
		fa.ops           = h->d_ops;
		fa.x             = X;
		fa.y             = Y;
		fa.items         = h->d_fitems;
		fa.units         = h->d_funits;
		fa.sector_active = h->sector_active;
		fa.io            = io;
		fa.n_items       = int(P.fitems.size());
		fa.max_clusters  = h->fused_clusters;
		if ((e = dmrgpp::launch_fused(fa, h->cfg - kNumTileCfgs, h->stream)))
			return cuda_fail(h, e, "fused H*x launch");
		return DMRGPP_OK;
	}
	dmrgpp::PersistentArgs pa {};
	pa.ops           = h->d_ops;
	pa.x             = X;
	pa.bx            = h->d_bx;
	pa.y             = Y;
	pa.partial       = h->d_part;
	pa.seg1          = h->d_seg1;
	pa.pseg2         = h->d_pseg2;
	pa.items         = h->d_items;
	pa.n1_of_j       = h->d_n1;
	pa.work_counter  = h->d_ctr;
	pa.done          = h->d_ctr + 3;
	pa.arrive        = h->d_ctr + 3 + P.np;
	pa.test_extra_wait = h->test_stall;
	pa.error         = h->err_dev;
	pa.item_sector   = h->d_item_sector;
	pa.sector_active = h->sector_active;
	pa.io            = io;
	pa.n_items       = int(P.items.size());
	pa.np            = int(P.np);
	pa.n_split_tiles = P.n_split_tiles;
	if ((e = dmrgpp::launch_persistent(pa, h->cfg, h->grid, h->stream)))
		return cuda_fail(h, e, "H*x launch");
	return DMRGPP_OK;

}

void mixed_host_plan(dmrgpp_kron_handle h, int sms, MixedHost& out)
{
	size_t maxs = 0;
	for (size_t p = 0; p < h->plan.np; ++p)
		maxs = std::max<size_t>(maxs, size_t(std::max(h->plan.l[p], h->plan.r[p])));
	const int bn = maxs > 96 ? 128 : 64;
	// operators: packed on the device from the FP64 copy (mixed_pack_jobs)
	out.msg = build_mixed_plan(h->plan, bn, nullptr, nullptr, &out.xmap, sms);
	if (!out.msg.empty())
		return;
	if (validation_requested()) { // debug mode: bounds of the layout before any launch
		const std::string v = validate_mixed_plan(h->plan);
		if (!v.empty()) {
			out.msg = "schedule check: " + v;
			return;
		}
	}
	MixedPlan& mp = h->plan.mixed;
	out.grid1     = balance_tiles(mp.tile1, mp.seg1, sms, out.starts1);
	out.grid2     = balance_tiles(mp.tile2, mp.seg2, sms, out.starts2);
	out.jobs      = mixed_pack_jobs(h->plan);
	out.ready     = true;
}

int build_mixed(dmrgpp_kron_handle h, MixedHost& host)
{
	if (!host.ready)
		return fail(h, DMRGPP_INVALID_ARG, host.msg);
	cudaError_t      e;
	const MixedPlan& mp = h->plan.mixed;
	if ((e = tc_init()) != cudaSuccess)
		return cuda_fail(h, e, "tensor-core kernel attributes");
	const std::vector<int>& xmap    = host.xmap;
	const std::vector<int>& starts1 = host.starts1;
	const std::vector<int>& starts2 = host.starts2;
	h->m_grid1                      = host.grid1;
	h->m_grid2                      = host.grid2;
	auto fbytes = [](long long n) { return size_t(n > 0 ? n : 1) * sizeof(float); };
	if ((e = dmrgpp::dev_malloc(&h->m_ops_hi, fbytes(mp.ops_elems))) || (e = dmrgpp::dev_malloc(&h->m_ops_lo, fbytes(mp.ops_elems)))
	    || (e = dmrgpp::dev_malloc(&h->m_xs_hi, fbytes(mp.xs_elems))) || (e = dmrgpp::dev_malloc(&h->m_xs_lo, fbytes(mp.xs_elems)))
	    || (e = dmrgpp::dev_malloc(&h->m_bxs_hi, fbytes(mp.bxs_elems)))
	    || (e = dmrgpp::dev_malloc(&h->m_bxs_lo, fbytes(mp.bxs_elems)))
	    || (e = dmrgpp::dev_malloc(&h->m_xmap, size_t(std::max<long long>(h->plan.dim(), 1)) * sizeof(int))))
		return cuda_fail(h, e, "device allocation (mixed-precision buffers)");
	// K-split pass-2 tiles: FP32 partial slots and self-resetting counters
	if ((e = dmrgpp::dev_malloc(&h->m_partial, fbytes(mp.split_slots * 128 * mp.bn)))
	    || (e = dmrgpp::dev_malloc(&h->m_arrive, size_t(std::max(mp.n_split_tiles, 1)) * sizeof(unsigned)))
	    || (e = dmrgpp::clear_async(h->m_arrive, size_t(std::max(mp.n_split_tiles, 1)) * sizeof(unsigned), h->stream)))
		return cuda_fail(h, e, "device allocation (split-K partials)");
	// K padding must read as zero
	if ((e = dmrgpp::clear_async(h->m_xs_hi, fbytes(mp.xs_elems), h->stream)) || (e = dmrgpp::clear_async(h->m_xs_lo, fbytes(mp.xs_elems), h->stream))
	    || (e = dmrgpp::clear_async(h->m_bxs_hi, fbytes(mp.bxs_elems), h->stream))
	    || (e = dmrgpp::clear_async(h->m_bxs_lo, fbytes(mp.bxs_elems), h->stream)))
		return cuda_fail(h, e, "clear mixed-precision buffers");
	{
		const std::vector<PackJob>& jobs   = host.jobs;
		PackJob*                    d_jobs = nullptr;
		if ((e = dmrgpp::clear_async(h->m_ops_hi, fbytes(mp.ops_elems), h->stream)) || (e = dmrgpp::clear_async(h->m_ops_lo, fbytes(mp.ops_elems), h->stream))
		    || (e = dmrgpp::dev_malloc(&d_jobs, std::max<size_t>(jobs.size(), 1) * sizeof(PackJob)))
		    || (e = dmrgpp::upload_sync(d_jobs, jobs.data(), jobs.size() * sizeof(PackJob), h->stream))
		    || (e = tc_pack_ops(h->d_ops, h->m_ops_hi, h->m_ops_lo, d_jobs, int(jobs.size()), h->stream))
		    || (e = cudaStreamSynchronize(h->stream))) {
			dmrgpp::dev_free(d_jobs);
			return cuda_fail(h, e, "pack mixed-precision operators");
		}
		dmrgpp::dev_free(d_jobs);
	}
	{
		// the operand buffers as 2-D tensors [row][32 floats], 128-byte
		// swizzle: pass 1 A = operators (128-row boxes), B = x split (bn);
		// pass 2 A = BX split (128), B = operators (bn); hi and lo each;
		// then the BX split with 32-row boxes for pass 1's stores
		PFN_cuTensorMapEncodeTiled_v12000 encode = tensor_map_encoder();
		if (!encode)
			return fail(h, DMRGPP_NOT_SUPPORTED, "cuTensorMapEncodeTiled is not available");
		CUtensorMap* tm = reinterpret_cast<CUtensorMap*>(h->m_tmap);
		struct Spec {
			float*    buf;
			long long elems;
			int       box;
		} spec[10] = { { h->m_ops_hi, mp.ops_elems, mp.bm }, { h->m_ops_lo, mp.ops_elems, mp.bm },
		               { h->m_xs_hi, mp.xs_elems, mp.bn },   { h->m_xs_lo, mp.xs_elems, mp.bn },
		               { h->m_bxs_hi, mp.bxs_elems, mp.bm }, { h->m_bxs_lo, mp.bxs_elems, mp.bm },
		               { h->m_ops_hi, mp.ops_elems, mp.bn }, { h->m_ops_lo, mp.ops_elems, mp.bn },
		               { h->m_bxs_hi, mp.bxs_elems, 32 },    { h->m_bxs_lo, mp.bxs_elems, 32 } };
		for (int q = 0; q < 10; ++q) {
			const cuuint64_t dims[2]    = { 32, cuuint64_t(std::max<long long>(spec[q].elems / 32, 1)) };
			const cuuint64_t strides[1] = { 128 };
			const cuuint32_t box[2]     = { 32, cuuint32_t(spec[q].box) };
			const cuuint32_t es[2]      = { 1, 1 };
			const CUresult   r = encode(&tm[q], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, spec[q].buf, dims, strides,
                                          box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                          CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
			if (r != CUDA_SUCCESS)
				return fail(h, DMRGPP_CUDA_ERROR,
				            "tensor map " + std::to_string(q) + " rejected (code " + std::to_string(int(r)) + ")");
		}
	}
	if (!xmap.empty()
	    && (e = dmrgpp::upload_sync(h->m_xmap, xmap.data(), xmap.size() * sizeof(int), h->stream)))
		return cuda_fail(h, e, "upload x map");
	std::vector<unsigned char> lists;
	std::vector<size_t>        offs;
	auto add = [&](const void* src, size_t n) {
		offs.push_back(lists.size());
		lists.resize(lists.size() + ((n + 15) / 16) * 16);
		if (n)
			std::memcpy(lists.data() + offs.back(), src, n);
	};
	add(mp.seg1.data(), mp.seg1.size() * sizeof(GemmSeg));
	add(mp.seg2.data(), mp.seg2.size() * sizeof(GemmSeg));
	add(mp.tile1.data(), mp.tile1.size() * sizeof(GemmTile));
	add(mp.tile2.data(), mp.tile2.size() * sizeof(GemmTile));
	add(starts1.data(), starts1.size() * sizeof(int));
	add(starts2.data(), starts2.size() * sizeof(int));
	// group handles: the sector of every tile (pass 1: its input patch; pass
	// 2: its output patch), so that stopped sectors' tiles can be skipped
	const bool group = h->sector_start.size() > 2;
	if (group) {
		auto sector_of = [&](long long off) {
			return int(std::upper_bound(h->sector_start.begin(), h->sector_start.end(), off)
			           - h->sector_start.begin())
			    - 1;
		};
		std::vector<int> t1(mp.tile1.size()), t2(mp.tile2.size());
		for (size_t q = 0; q < t1.size(); ++q)
			t1[q] = sector_of(h->plan.xy_start[size_t(mp.seg1[size_t(mp.tile1[q].seg_begin)].dep)]);
		for (size_t q = 0; q < t2.size(); ++q)
			t2[q] = sector_of(mp.tile2[q].c_off);
		add(t1.data(), t1.size() * sizeof(int));
		add(t2.data(), t2.size() * sizeof(int));
	}
	if ((e = dmrgpp::dev_malloc(&h->m_lists, lists.empty() ? 16 : lists.size())))
		return cuda_fail(h, e, "device allocation (mixed lists)");
	auto at    = [&](int i) { return static_cast<unsigned char*>(h->m_lists) + offs[i]; };
	h->m_seg1  = reinterpret_cast<GemmSeg*>(at(0));
	h->m_seg2  = reinterpret_cast<GemmSeg*>(at(1));
	h->m_tile1 = reinterpret_cast<GemmTile*>(at(2));
	h->m_tile2 = reinterpret_cast<GemmTile*>(at(3));
	h->m_starts1 = reinterpret_cast<int*>(at(4));
	h->m_starts2 = reinterpret_cast<int*>(at(5));
	h->m_tsec1   = group ? reinterpret_cast<int*>(at(6)) : nullptr;
	h->m_tsec2   = group ? reinterpret_cast<int*>(at(7)) : nullptr;
	if (!lists.empty()
	    && (e = dmrgpp::upload_sync(h->m_lists, lists.data(), lists.size(), h->stream)))
		return cuda_fail(h, e, "upload mixed lists");
	h->mixed_ready = true;
	return DMRGPP_OK;
}

// Fused form: schedule for configuration fcfg, its tiles' work cut into about
// parts_per_sm rounds of parts for every co-resident CTA.
int configure_fused(dmrgpp_kron_handle h, int fcfg, int parts_per_sm)
{
	cudaError_t e = fused_init(fcfg, &h->fused_clusters);
	if (e == cudaSuccess && h->fused_clusters < 1)
		e = cudaErrorInvalidConfiguration;
	if (e != cudaSuccess)
		return cuda_fail(h, e, "fused kernel attributes");
	KronPlan&        P = h->plan;
	const FusedShape s = fused_shape(fcfg);
	std::vector<int> sector_of_patch;
	if (h->sector_start.size() > 2) {
		sector_of_patch.resize(P.np);
		for (size_t i = 0; i < P.np; ++i)
			sector_of_patch[i] = int(std::upper_bound(h->sector_start.begin(), h->sector_start.end(),
			                                          P.xy_start[i])
			                         - h->sector_start.begin())
			    - 1;
	}
	build_fused_schedule(P, s.bm, s.bn, s.cw, s.cluster, parts_per_sm, h->fused_clusters * s.cluster,
	                     sector_of_patch.empty() ? nullptr : &sector_of_patch);
	if (validation_requested()) { // debug mode: bounds of the work list before any launch
		const std::string v = validate_fused_schedule(P, s.bm, s.bn, s.cluster);
		if (!v.empty())
			return fail(h, DMRGPP_INVALID_ARG, "schedule check: " + v);
	}
	if (P.fitems.size() > size_t(INT_MAX) || P.funits.size() > size_t(INT_MAX))
		return fail(h, DMRGPP_INVALID_ARG, "sector too large for the fused form");
	const size_t ib = P.fitems.size() * sizeof(FusedItem), ub = P.funits.size() * sizeof(FusedUnit);
	dmrgpp::dev_free(h->d_flists);
	h->d_flists = nullptr;
	h->d_fitems = nullptr;
	h->d_funits = nullptr;
	if ((e = dmrgpp::dev_malloc(&h->d_flists, std::max<size_t>(ib + ub, 16))))
		return cuda_fail(h, e, "device allocation (fused lists)");
	h->d_fitems = static_cast<FusedItem*>(h->d_flists);
	h->d_funits = reinterpret_cast<FusedUnit*>(static_cast<unsigned char*>(h->d_flists) + ib);
	if ((ib && (e = dmrgpp::upload_sync(h->d_fitems, P.fitems.data(), ib, h->stream)))
	    || (ub && (e = dmrgpp::upload_sync(h->d_funits, P.funits.data(), ub, h->stream))))
		return cuda_fail(h, e, "upload fused lists");
	h->cfg           = kNumTileCfgs + fcfg;
	h->items_per_cta = parts_per_sm;
	return DMRGPP_OK;
}

int configure_schedule(dmrgpp_kron_handle h, int cfg, int items_per_cta)
{
	if (cfg >= kNumTileCfgs)
		return configure_fused(h, cfg - kNumTileCfgs, items_per_cta);
	int         grid = 0, tile = 0, bk = 0;
	cudaError_t e    = persistent_config(cfg, &grid, &tile, &bk);
	if (e != cudaSuccess)
		return cuda_fail(h, e, "persistent kernel attributes");
	KronPlan& P = h->plan;
	if (tile != P.bm || P.tile1.size() + P.tile2.size() == 0)
		build_tile_lists(P, tile, tile);
	build_persistent_schedule(P, bk, grid, items_per_cta);
	if (validation_requested()) { // debug mode: bounds of the work list before any launch
		const std::string v = validate_persistent_schedule(P, tile);
		if (!v.empty())
			return fail(h, DMRGPP_INVALID_ARG, "schedule check: " + v);
	}
	h->cfg           = cfg;
	h->grid          = grid;
	h->tile          = tile;
	h->items_per_cta = items_per_cta;

	// every list in one allocation, each chunk on a 16-byte boundary
	std::vector<unsigned char> lists;
	std::vector<size_t>        offs;
	auto add = [&](const void* src, size_t n) {
		offs.push_back(lists.size());
		lists.resize(lists.size() + ((n + 15) / 16) * 16);
		if (n)
			std::memcpy(lists.data() + offs.back(), src, n);
	};
	add(P.seg1.data(), P.seg1.size() * sizeof(GemmSeg));
	add(P.seg2.data(), P.seg2.size() * sizeof(GemmSeg));
	add(P.tile1.data(), P.tile1.size() * sizeof(GemmTile));
	add(P.tile2.data(), P.tile2.size() * sizeof(GemmTile));
	add(P.items.data(), P.items.size() * sizeof(KronItem));
	add(P.pseg2.data(), P.pseg2.size() * sizeof(GemmSeg));
	add(P.n1_of_j.data(), P.n1_of_j.size() * sizeof(int));
	// sector of every item (a pass-1 item: its input patch; pass 2: its output)
	std::vector<int> item_sector(P.items.size(), 0);
	if (h->sector_start.size() > 2) {
		auto sector_of = [&](long long off) {
			return int(std::upper_bound(h->sector_start.begin(), h->sector_start.end(), off)
			           - h->sector_start.begin())
			    - 1;
		};
		for (size_t q = 0; q < P.items.size(); ++q) {
			const KronItem& w = P.items[q];
			item_sector[q]    = w.kind == 0 ? sector_of(P.xy_start[size_t(w.producer)]) : sector_of(w.c_off);
		}
	}
	add(item_sector.data(), item_sector.size() * sizeof(int));
	dmrgpp::dev_free(h->d_lists);
	dmrgpp::dev_free(h->d_ctr);
	dmrgpp::dev_free(h->d_part);
	h->d_lists = nullptr;
	h->d_ctr   = nullptr;
	h->d_part  = nullptr;
	if ((e = dmrgpp::dev_malloc(&h->d_lists, lists.empty() ? 16 : lists.size())))
		return cuda_fail(h, e, "device allocation (lists)");
	auto at    = [&](int i) { return static_cast<unsigned char*>(h->d_lists) + offs[i]; };
	h->d_seg1  = reinterpret_cast<GemmSeg*>(at(0));
	h->d_seg2  = reinterpret_cast<GemmSeg*>(at(1));
	h->d_tile1 = reinterpret_cast<GemmTile*>(at(2));
	h->d_tile2 = reinterpret_cast<GemmTile*>(at(3));
	h->d_items = reinterpret_cast<KronItem*>(at(4));
	h->d_pseg2 = reinterpret_cast<GemmSeg*>(at(5));
	h->d_n1    = reinterpret_cast<int*>(at(6));
	h->d_item_sector = reinterpret_cast<int*>(at(7));
	if (!lists.empty()
	    && (e = dmrgpp::upload_sync(h->d_lists, lists.data(), lists.size(), h->stream)))
		return cuda_fail(h, e, "upload lists");

	const size_t nctr = 3 + P.np + size_t(P.n_split_tiles);
	if ((e = dmrgpp::dev_malloc(&h->d_ctr, nctr * sizeof(unsigned))))
		return cuda_fail(h, e, "device allocation (counters)");
	if ((e = dmrgpp::clear_async(h->d_ctr, nctr * sizeof(unsigned), h->stream)))
		return cuda_fail(h, e, "clear counters");
	const size_t part_elems = size_t(P.partial_slots) * size_t(tile) * size_t(tile);
	if ((e = dmrgpp::dev_malloc(&h->d_part, (part_elems ? part_elems : 1) * sizeof(double))))
		return cuda_fail(h, e, "device allocation (partials)");
	return DMRGPP_OK;
}

} // namespace dmrgpp

namespace {

// Device side of a new handle whose plan (with host blocks) is built: device
// buffers, persistent schedule, diagonal, and the TF32x3 form if requested.
// Frees h on failure.
using Clock = std::chrono::steady_clock;

double seconds_since(Clock::time_point t0)
{
	return std::chrono::duration<double>(Clock::now() - t0).count();
}

// t0: when create started (before the plan); the plan's time is recorded by
// the caller in h->setup_times[DMRGPP_SETUP_PLAN]
int finish_create(dmrgpp_kron_handle h, int device, void* stream, int bm, Clock::time_point t0,
                  dmrgpp_kron_handle* out)
{
	// (h->crs, when set, points at the caller's CRS operators until the upload)
	if (device >= 0) {
		h->device = device;
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
	h->stream = static_cast<cudaStream_t>(stream);

	auto         tp  = Clock::now();
	const auto&  P   = h->plan;
	const size_t dim = size_t(P.dim());
	if ((e = dmrgpp::dev_malloc(&h->d_ops, size_t(P.op_elems ? P.op_elems : 1) * sizeof(double))))
		return bail(e, "device allocation (operators)");
	if ((e = dmrgpp::dev_malloc(&h->d_bx, size_t(P.bx_elems ? P.bx_elems : 1) * sizeof(double))))
		return bail(e, "device allocation (BX)");
	if ((e = dmrgpp::dev_malloc(&h->d_x, dim * sizeof(double))))
		return bail(e, "device allocation (x)");
	if ((e = dmrgpp::dev_malloc(&h->d_y, dim * sizeof(double))))
		return bail(e, "device allocation (y)");

	if ((e = dmrgpp::error_word_alloc(&h->err_host, &h->err_dev)))
		return bail(e, "error word");
	if (int rc = dmrgpp::configure_schedule(h, bm == 32 ? 0 : 2, 2)) {
		const std::string why = h->err;
		release(h);
		delete h;
		return fail(nullptr, rc, why);
	}
	// the TF32x3 form's host planning (reads the plan, writes plan.mixed)
	// runs on its own thread while the operators are uploaded
	dmrgpp::MixedHost mixed_host;
	std::thread       mixed_thread;
	if (h->precision == DMRGPP_TF32X3) {
		int sms = 0;
		if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device)))
			return bail(e, "SM count");
		mixed_thread = std::thread([h, sms, &mixed_host] { dmrgpp::mixed_host_plan(h, sms, mixed_host); });
	}
	auto join_mixed = [&] {
		if (mixed_thread.joinable())
			mixed_thread.join();
	};
	auto abandon = [&](int rc) { // the thread reads h: join it before h goes
		join_mixed();
		const std::string why = h->err;
		release(h);
		delete h;
		return fail(nullptr, rc, why);
	};
	h->setup_times[DMRGPP_SETUP_ALLOC] = seconds_since(tp);
	tp                                 = Clock::now();
	if (int rc = h->crs ? dmrgpp::upload_operators_crs(h)
	                    : dmrgpp::upload_operators(h, &h->setup_times[DMRGPP_SETUP_UPLOAD_FILL]))
		return abandon(rc);
	h->crs = nullptr;
	h->setup_times[DMRGPP_SETUP_UPLOAD] = seconds_since(tp);
	tp                                  = Clock::now();
	if (int rc = dmrgpp::upload_diagonal(h))
		return abandon(rc);
	h->setup_times[DMRGPP_SETUP_DIAGONAL] = seconds_since(tp);
	tp                                    = Clock::now();
	if (h->precision == DMRGPP_TF32X3) {
		join_mixed();
		if (int rc = dmrgpp::build_mixed(h, mixed_host))
			return abandon(rc);
		h->setup_times[DMRGPP_SETUP_MIXED] = seconds_since(tp);
	}
	h->setup_times[DMRGPP_SETUP_TOTAL] = seconds_since(t0);
	// the caller's host blocks are not referenced after create
	h->plan.blocks.clear();
	h->plan.blocks.shrink_to_fit();
	*out = h;
	return DMRGPP_OK;
}

} // namespace

extern "C" {

const char* dmrgpp_version(void) { return DMRGPP_VERSION_STRING; }

const char* dmrgpp_kron_last_error(dmrgpp_kron_handle h)
{
	return h ? h->err.c_str() : g_create_error.c_str();
}

int dmrgpp_kron_setup_profile(dmrgpp_kron_handle h, double* t, size_t n)
{
	if (!h || (!t && n))
		return fail(h, DMRGPP_INVALID_ARG, "null argument");
	if (n > DMRGPP_SETUP_NPHASES)
		return fail(h, DMRGPP_INVALID_ARG, "at most DMRGPP_SETUP_NPHASES phases");
	for (size_t q = 0; q < n; ++q)
		t[q] = h->setup_times[q];
	return DMRGPP_OK;
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
	DMRGPP_TRACE("dmrgpp_kron_create");
	if (!out)
		return fail(nullptr, DMRGPP_INVALID_ARG, "null output handle");
	*out = nullptr;
	if (int rc = check_desc(d))
		return rc;
	if (d->precision == DMRGPP_SPLIT_BF16)
		return fail(nullptr, DMRGPP_NOT_SUPPORTED, "split-BF16 is not built into this library");

	dmrgpp_kron_handle h = new (std::nothrow) dmrgpp_kron_s();
	if (!h)
		return fail(nullptr, DMRGPP_OOM, "host allocation failed");
	h->precision = d->precision;

	const auto t0 = Clock::now();
	int        bm, bn;
	pick_tile(d, bm, bn);
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
                                              nullptr);
	if (!msg.empty()) {
		delete h;
		return fail(nullptr, DMRGPP_INVALID_ARG, msg);
	}
	h->sector_start                   = { 0, h->plan.dim() };
	h->setup_times[DMRGPP_SETUP_PLAN] = seconds_since(t0);
	return finish_create(h, d->device, d->stream, bm, t0, out);
}

int dmrgpp_kron_create_crs(const dmrgpp_kron_crs_desc* d, dmrgpp_kron_handle* out)
{
	DMRGPP_TRACE("dmrgpp_kron_create_crs");
	if (!out)
		return fail(nullptr, DMRGPP_INVALID_ARG, "null output handle");
	*out = nullptr;
	if (!d)
		return fail(nullptr, DMRGPP_INVALID_ARG, "null descriptor");
	if (d->precision != DMRGPP_FP64 && d->precision != DMRGPP_SPLIT_BF16 && d->precision != DMRGPP_TF32X3)
		return fail(nullptr, DMRGPP_INVALID_ARG, "unknown precision mode");
	if (d->precision == DMRGPP_SPLIT_BF16)
		return fail(nullptr, DMRGPP_NOT_SUPPORTED, "split-BF16 is not built into this library");
	const auto                    t0 = Clock::now();
	dmrgpp::CrsSource             src;
	std::vector<dmrgpp::Triple>   triples;
	std::vector<dmrgpp::BlockRef> blocks;
	double                        f_alg = 0.0;
	std::string                   msg   = dmrgpp::crs_triples(d, src, triples, blocks, f_alg);
	if (!msg.empty())
		return fail(nullptr, DMRGPP_INVALID_ARG, msg);
	dmrgpp_kron_handle h = new (std::nothrow) dmrgpp_kron_s();
	if (!h)
		return fail(nullptr, DMRGPP_OOM, "host allocation failed");
	h->precision = d->precision;
	int bm, bn;
	pick_tile_sizes(d->npatches, d->left_patch_size, d->right_patch_size, bm, bn);
	msg = dmrgpp::build_kron_plan_triples(d->noperator, d->npatches, d->left_patch_size, d->right_patch_size,
	                                      std::move(triples), std::move(blocks), f_alg, bm, bn, h->plan,
	                                      nullptr);
	if (!msg.empty()) {
		delete h;
		return fail(nullptr, DMRGPP_INVALID_ARG, msg);
	}
	h->sector_start                   = { 0, h->plan.dim() };
	h->setup_times[DMRGPP_SETUP_PLAN] = seconds_since(t0);
	h->crs                            = &src; // read by finish_create's upload only
	return finish_create(h, d->device, d->stream, bm, t0, out);
}

int dmrgpp_kron_create_complex(const dmrgpp_kron_desc* d, dmrgpp_kron_handle* out)
{
	DMRGPP_TRACE("dmrgpp_kron_create_complex");
	if (!out)
		return fail(nullptr, DMRGPP_INVALID_ARG, "null output handle");
	*out = nullptr;
	if (int rc = check_desc(d))
		return rc;
	if (d->precision == DMRGPP_SPLIT_BF16)
		return fail(nullptr, DMRGPP_NOT_SUPPORTED, "split-BF16 is not built into this library");
	if (d->noperator == 0 || d->npatches == 0)
		return fail(nullptr, DMRGPP_INVALID_ARG, "noperator and npatches must be >= 1");
	const size_t np = d->npatches, K = d->noperator, np2 = 2 * np, K2 = 2 * K;
	if (np2 > size_t(INT_MAX))
		return fail(nullptr, DMRGPP_INVALID_ARG, "too many patches");
	// real embedding: patch p holds Re x_p, patch p + np holds Im x_p; with
	// A = Ar + i Ai and B = Br + i Bi, A (x) B = (Ar(x)Br - Ai(x)Bi) + i (Ar(x)Bi + Ai(x)Br):
	//   (i, j), (i+np, j+np):  Ar(x)Br, (-Ai)(x)Bi
	//   (i, j+np):             (-Ar)(x)Bi, (-Ai)(x)Br
	//   (i+np, j):             Ar(x)Bi, Ai(x)Br
	// each complex term k becomes real terms 2k and 2k+1 of every quadrant
	std::vector<size_t>        l2(np2), r2(np2);
	std::vector<const double*> A2(np2 * np2 * K2, nullptr), B2(np2 * np2 * K2, nullptr);
	std::vector<size_t>        ldA2(np2 * np2 * K2, 0), ldB2(np2 * np2 * K2, 0);
	for (size_t p = 0; p < np; ++p) {
		l2[p] = l2[p + np] = d->left_patch_size[p];
		r2[p] = r2[p + np] = d->right_patch_size[p];
	}
	std::vector<std::vector<double>> store;
	auto part = [&](const double* z, size_t ld, size_t rows, size_t cols, int im, double sign) {
		store.emplace_back(rows * cols);
		double* m = store.back().data();
		for (size_t c = 0; c < cols; ++c)
			for (size_t q = 0; q < rows; ++q)
				m[q + c * rows] = sign * z[2 * (q + c * ld) + size_t(im)];
		return static_cast<const double*>(m);
	};
	for (size_t k = 0; k < K; ++k)
		for (size_t j = 0; j < np; ++j)
			for (size_t i = 0; i < np; ++i) {
				const size_t t = i + j * np + k * np * np;
				if (!d->Amatrix[t] || !d->Bmatrix[t])
					continue;
				if (d->ld_Amatrix[t] < l2[i] || d->ld_Bmatrix[t] < r2[i])
					return fail(nullptr, DMRGPP_INVALID_ARG,
					            "leading dimension smaller than the block's rows at table entry "
					                + std::to_string(t));
				const size_t  li = l2[i], lj = l2[j], ri = r2[i], rj = r2[j];
				const double* Ar  = part(d->Amatrix[t], d->ld_Amatrix[t], li, lj, 0, 1.0);
				const double* Ai  = part(d->Amatrix[t], d->ld_Amatrix[t], li, lj, 1, 1.0);
				const double* nAr = part(d->Amatrix[t], d->ld_Amatrix[t], li, lj, 0, -1.0);
				const double* nAi = part(d->Amatrix[t], d->ld_Amatrix[t], li, lj, 1, -1.0);
				const double* Br  = part(d->Bmatrix[t], d->ld_Bmatrix[t], ri, rj, 0, 1.0);
				const double* Bi  = part(d->Bmatrix[t], d->ld_Bmatrix[t], ri, rj, 1, 1.0);
				auto set = [&](size_t I, size_t J, size_t kk, const double* a, const double* b) {
					const size_t u = I + J * np2 + kk * np2 * np2;
					A2[u]          = a;
					B2[u]          = b;
					ldA2[u]        = l2[I];
					ldB2[u]        = r2[I];
				};
				set(i, j, 2 * k, Ar, Br);
				set(i, j, 2 * k + 1, nAi, Bi);
				set(i + np, j + np, 2 * k, Ar, Br);
				set(i + np, j + np, 2 * k + 1, nAi, Bi);
				set(i, j + np, 2 * k, nAr, Bi);
				set(i, j + np, 2 * k + 1, nAi, Br);
				set(i + np, j, 2 * k, Ar, Bi);
				set(i + np, j, 2 * k + 1, Ai, Br);
			}
	dmrgpp_kron_desc e = *d;
	e.noperator        = K2;
	e.npatches         = np2;
	e.left_patch_size  = l2.data();
	e.right_patch_size = r2.data();
	e.Amatrix          = A2.data();
	e.ld_Amatrix       = ldA2.data();
	e.Bmatrix          = B2.data();
	e.ld_Bmatrix       = ldB2.data();
	dmrgpp_kron_handle h = nullptr;
	if (int rc = dmrgpp_kron_create(&e, &h))
		return rc;
	h->complex_sector = true;
	DeviceGuard       g(h->device);
	if (cudaError_t err = dmrgpp::dev_malloc(&h->d_cx, size_t(std::max<long long>(h->plan.dim(), 1)) * sizeof(double))) {
		dmrgpp_kron_destroy(h);
		return cuda_fail(nullptr, err, "device allocation (complex staging)");
	}
	*out = h;
	return DMRGPP_OK;
}

int dmrgpp_kron_is_complex(dmrgpp_kron_handle h, int* is_complex)
{
	if (!h || !is_complex)
		return fail(h, DMRGPP_INVALID_ARG, "null argument");
	*is_complex = h->complex_sector ? 1 : 0;
	return DMRGPP_OK;
}

int dmrgpp_kron_create_group(const dmrgpp_kron_desc* descs, size_t nsectors, dmrgpp_kron_handle* out)
{
	DMRGPP_TRACE("dmrgpp_kron_create_group");
	if (!out)
		return fail(nullptr, DMRGPP_INVALID_ARG, "null output handle");
	*out = nullptr;
	if (!descs || nsectors == 0)
		return fail(nullptr, DMRGPP_INVALID_ARG, "no sectors");
	for (size_t s = 0; s < nsectors; ++s) {
		if (int rc = check_desc(&descs[s]))
			return rc;
		if (descs[s].noperator == 0 || descs[s].npatches == 0)
			return fail(nullptr, DMRGPP_INVALID_ARG,
			            "sector " + std::to_string(s) + ": noperator and npatches must be >= 1");
		if (!descs[s].Amatrix || !descs[s].ld_Amatrix || !descs[s].Bmatrix || !descs[s].ld_Bmatrix)
			return fail(nullptr, DMRGPP_INVALID_ARG, "sector " + std::to_string(s) + ": null table");
		if (descs[s].precision != descs[0].precision || descs[s].device != descs[0].device
		    || descs[s].stream != descs[0].stream)
			return fail(nullptr, DMRGPP_INVALID_ARG,
			            "all sectors of a group need the same precision, device and stream");
	}
	if (descs[0].precision == DMRGPP_SPLIT_BF16)
		return fail(nullptr, DMRGPP_NOT_SUPPORTED, "split-BF16 is not built into this library");

	// the union: sector s's patches follow those of sectors 0..s-1; no block
	// connects two sectors, so the union's H is block-diagonal
	const auto                    t0 = Clock::now();
	std::vector<size_t>           l, r;
	std::vector<dmrgpp::Triple>   triples;
	std::vector<dmrgpp::BlockRef> blocks;
	std::vector<long long>        starts(1, 0);
	double                        f_alg = 0.0;
	size_t                        nop   = 0;
	for (size_t s = 0; s < nsectors; ++s) {
		const dmrgpp_kron_desc& d = descs[s];
		for (size_t p = 0; p < d.npatches; ++p)
			if (d.left_patch_size[p] < 1 || d.right_patch_size[p] < 1)
				return fail(nullptr, DMRGPP_INVALID_ARG,
				            "sector " + std::to_string(s) + " patch " + std::to_string(p)
				                + " has an empty left or right group");
		if (l.size() + d.npatches > size_t(INT_MAX))
			return fail(nullptr, DMRGPP_INVALID_ARG, "too many patches in the group");
		std::string msg = dmrgpp::collect_triples(d.noperator, d.npatches, d.left_patch_size,
		                                          d.right_patch_size, d.Amatrix, d.ld_Amatrix,
		                                          d.Bmatrix, d.ld_Bmatrix, int(l.size()), triples,
		                                          blocks, f_alg);
		if (!msg.empty())
			return fail(nullptr, DMRGPP_INVALID_ARG, "sector " + std::to_string(s) + ": " + msg);
		long long dim = 0;
		for (size_t p = 0; p < d.npatches; ++p) {
			l.push_back(d.left_patch_size[p]);
			r.push_back(d.right_patch_size[p]);
			dim += (long long)d.left_patch_size[p] * (long long)d.right_patch_size[p];
		}
		starts.push_back(starts.back() + dim);
		nop = std::max(nop, d.noperator);
	}

	dmrgpp_kron_handle h = new (std::nothrow) dmrgpp_kron_s();
	if (!h)
		return fail(nullptr, DMRGPP_OOM, "host allocation failed");
	h->precision = descs[0].precision;
	int bm, bn;
	pick_tile_sizes(l.size(), l.data(), r.data(), bm, bn);
	std::string msg = dmrgpp::build_kron_plan_triples(nop, l.size(), l.data(), r.data(),
	                                                  std::move(triples), std::move(blocks), f_alg,
	                                                  bm, bn, h->plan, nullptr);
	if (!msg.empty()) {
		delete h;
		return fail(nullptr, DMRGPP_INVALID_ARG, msg);
	}
	h->sector_start                   = std::move(starts);
	h->setup_times[DMRGPP_SETUP_PLAN] = seconds_since(t0);
	return finish_create(h, descs[0].device, descs[0].stream, bm, t0, out);
}

int dmrgpp_kron_group_sectors(dmrgpp_kron_handle h, size_t* nsectors, long long* offsets)
{
	if (!h || !nsectors)
		return fail(h, DMRGPP_INVALID_ARG, "null argument");
	*nsectors = h->sector_start.size() - 1;
	if (offsets)
		for (size_t s = 0; s < h->sector_start.size(); ++s)
			offsets[s] = h->sector_start[s];
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
	*dim = size_t(h->plan.dim()) / (h->complex_sector ? 2 : 1);
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
	DMRGPP_TRACE("dmrgpp_kron_apply");
	if (!h)
		return fail(nullptr, DMRGPP_INVALID_ARG, "null handle");
	if (!x || !y)
		return fail(h, DMRGPP_INVALID_ARG, "null vector");
	DeviceGuard g(h->device);
	if (!g.ok)
		return cuda_fail(h, cudaErrorInvalidDevice, "cudaSetDevice");
	if (h->complex_sector) {
		// interleaved complex x -> [Re; Im] -> real embedding -> interleaved y
		const size_t n = size_t(h->plan.dim()) / 2;
		cudaError_t  e;
		if (!on_device
		    && (e = cudaMemcpyAsync(h->d_cx, x, 2 * n * sizeof(double), cudaMemcpyHostToDevice, h->stream)))
			return cuda_fail(h, e, "copy x to device");
		if ((e = dmrgpp::complex_split(on_device ? x : h->d_cx, h->d_x, n, h->stream)))
			return cuda_fail(h, e, "complex split");
		if (int rc = dmrgpp::kron_apply_device(h, h->d_x, h->d_y))
			return rc;
		if ((e = dmrgpp::complex_join(h->d_y, on_device ? y : h->d_cx, n, h->stream)))
			return cuda_fail(h, e, "complex join");
		if (on_device)
			return DMRGPP_OK;
		if ((e = cudaMemcpyAsync(y, h->d_cx, 2 * n * sizeof(double), cudaMemcpyDeviceToHost, h->stream))
		    || (e = cudaStreamSynchronize(h->stream)))
			return cuda_fail(h, e, "copy y to host");
		return check_error_word(h);
	}
	const auto&   P   = h->plan;
	const size_t  dim = size_t(P.dim());
	const double* X   = on_device ? x : h->d_x;
	double*       Y   = on_device ? y : h->d_y;
	cudaError_t   e;
	if (!on_device
	    && (e = cudaMemcpyAsync(h->d_x, x, dim * sizeof(double), cudaMemcpyHostToDevice, h->stream)))
		return cuda_fail(h, e, "copy x to device");

	if (int rc = dmrgpp::kron_apply_device(h, X, Y))
		return rc;

	if (!on_device) {
		if ((e = cudaMemcpyAsync(y, h->d_y, dim * sizeof(double), cudaMemcpyDeviceToHost, h->stream)))
			return cuda_fail(h, e, "copy y to host");
		if ((e = cudaStreamSynchronize(h->stream)))
			return cuda_fail(h, e, "apply");
		return check_error_word(h);
	}
	return DMRGPP_OK;
}

int dmrgpp_kron_test_stall_dependency(dmrgpp_kron_handle h, int on)
{
	if (!h)
		return fail(nullptr, DMRGPP_INVALID_ARG, "null handle");
	h->test_stall = on ? 1 : 0;
	return DMRGPP_OK;
}

int dmrgpp_kron_set_precision(dmrgpp_kron_handle h, int precision)
{
	if (!h)
		return fail(nullptr, DMRGPP_INVALID_ARG, "null handle");
	if (precision == DMRGPP_FP64 || (precision == DMRGPP_TF32X3 && h->mixed_ready)) {
		h->precision = precision;
		return DMRGPP_OK;
	}
	return fail(h, DMRGPP_NOT_SUPPORTED,
	            "precision not available on this handle (create it with that precision)");
}

int dmrgpp_kron_get_precision(dmrgpp_kron_handle h, int* precision)
{
	if (!h || !precision)
		return fail(nullptr, DMRGPP_INVALID_ARG, "null handle or output");
	*precision = h->precision;
	return DMRGPP_OK;
}

int dmrgpp_kron_synchronize(dmrgpp_kron_handle h)
{
	if (!h)
		return fail(nullptr, DMRGPP_INVALID_ARG, "null handle");
	DeviceGuard g(h->device);
	cudaError_t e = cudaStreamSynchronize(h->stream);
	if (e != cudaSuccess)
		return cuda_fail(h, e, "synchronize");
	return check_error_word(h);
}

} // extern "C"
