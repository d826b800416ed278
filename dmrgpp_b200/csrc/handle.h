// Internal definition of a sector handle (opaque in include/dmrgpp_kron.h),
// shared by the C-ABI translation units.
#pragma once

#include "dmrgpp_kron.h"
#include "kron_plan.h"

#include <cuda_runtime.h>

#include <string>
#include <vector>

namespace dmrgpp {
struct LanczosWork;  // device buffers of the eigensolvers, created on first use
struct DavidsonWork;
struct GroupWork;
// The caller's CRS operators during dmrgpp_kron_create_crs (crs.cu), with the
// host-side maps the device scatter needs.
struct CrsSource {
	const dmrgpp_kron_crs_desc* desc = nullptr;
	std::vector<int> lpatch, lloc; // per left state: its patch (-1: none) and index in the group
	std::vector<int> rpatch, rloc; // per right state
	std::vector<int> tri_ptr;      // per (k, i) (k * np + i): range of tri_j / tri_t
	std::vector<int> tri_j, tri_t; // contributing input patches j (ascending) and their triples
};

// Block-presence scan of the CRS operators: validates d, fills src and the
// contributing (i, j, k) triples in (i, j, k) order with their algorithmic
// flops, as collect_triples does for dense tables.  Returns "" or the reason.
std::string crs_triples(const dmrgpp_kron_crs_desc* d, CrsSource& src, std::vector<Triple>& triples,
                        std::vector<BlockRef>& blocks, double& f_alg);
}

struct dmrgpp_kron_s {
	int                 device     = 0;
	cudaStream_t        stream     = nullptr;
	int                 precision  = DMRGPP_FP64;
	dmrgpp::KronPlan    plan;
	std::vector<long long> sector_start; // offsets of the group's sectors in x (one sector: {0, dim})
	double*             d_ops   = nullptr; // packed Bstack_j and A^T blocks
	double*             d_bx    = nullptr; // pass-1 output (scratch)
	double*             d_x     = nullptr; // staging for host-pointer applies
	double*             d_y     = nullptr;
	dmrgpp::GemmSeg*    d_seg1  = nullptr;
	dmrgpp::GemmSeg*    d_seg2  = nullptr;
	dmrgpp::GemmTile*   d_tile1 = nullptr;
	dmrgpp::GemmTile*   d_tile2 = nullptr;
	void*               d_lists = nullptr; // one allocation behind every list
	// persistent single-launch form
	int                 cfg     = 0;  // tile configuration (kron_persistent.cuh)
	int                 tile    = 32;
	int                 grid    = 0;
	int                 items_per_cta = 2;
	dmrgpp::KronItem*   d_items = nullptr;
	dmrgpp::GemmSeg*    d_pseg2 = nullptr;
	int*                d_n1    = nullptr;
	int*                d_item_sector = nullptr; // per persistent item: its sector
	const int*          sector_active = nullptr; // set by the group solver: skip stopped sectors
	unsigned*           d_ctr   = nullptr; // work counters, done[np], arrive[split tiles]
	double*             d_part  = nullptr; // split-K partial tiles
	// fused form (cfg >= kNumTileCfgs, kron_fused.cu): items and units
	void*               d_flists = nullptr;
	dmrgpp::FusedItem*  d_fitems = nullptr;
	dmrgpp::FusedUnit*  d_funits = nullptr;
	int                 fused_clusters = 0; // co-resident clusters of the fused configuration
	double              tuned_fp64_us   = -1.0; // last autotune: best FP64 apply (microseconds)
	double              tuned_tf32x3_us = -1.0; // and the TF32x3 apply (handles with that form)
	int*                err_host = nullptr; // mapped pinned word written by the kernel
	int*                err_dev  = nullptr;
	int                 test_stall = 0;     // dmrgpp_kron_test_stall_dependency
	double              setup_times[DMRGPP_SETUP_NPHASES] = {}; // dmrgpp_kron_setup_profile
	// complex sector (dmrgpp_kron_create_complex): the plan is its real
	// embedding with 2 np patches (real parts, then imaginary parts); user
	// vectors are interleaved complex of plan.dim() / 2 entries
	bool                complex_sector = false;
	double*             d_cx = nullptr;     // interleaved staging for host-pointer applies
	// mixed-precision (TF32x3 tensor-core) form, built when requested
	bool                mixed_ready = false;
	float*              m_ops_hi = nullptr; // packed operators, TF32 hi / lo
	float*              m_ops_lo = nullptr;
	float*              m_xs_hi  = nullptr; // x split, K-major, zero padding
	float*              m_xs_lo  = nullptr;
	float*              m_bxs_hi = nullptr; // pass-1 result split
	float*              m_bxs_lo = nullptr;
	int*                m_xmap   = nullptr; // sector vector -> x split offsets
	int                 m_grid1  = 0;       // persistent CTAs of tensor-core pass 1 / 2
	int                 m_grid2  = 0;
	int*                m_starts1 = nullptr; // per-CTA tile runs of pass 1 / 2
	int*                m_starts2 = nullptr;
	int*                m_tsec1 = nullptr;   // group handles: per tile of pass 1 / 2 its sector
	int*                m_tsec2 = nullptr;
	float*              m_partial = nullptr; // split-K partial tiles of pass 2
	unsigned*           m_arrive  = nullptr; // per split tile: parts done
	// CUtensorMap (128 bytes) of the operand buffers: pass 1 A hi/lo, B hi/lo,
	// pass 2 A hi/lo, B hi/lo, then the BX split hi/lo with 32-row boxes
	// (pass 1's stores); passed to the kernels by value
	alignas(64) unsigned char m_tmap[10][128] = {};
	void*               m_lists  = nullptr; // seg1, seg2, tile1, tile2
	dmrgpp::GemmSeg*    m_seg1 = nullptr;
	dmrgpp::GemmSeg*    m_seg2 = nullptr;
	dmrgpp::GemmTile*   m_tile1 = nullptr;
	dmrgpp::GemmTile*   m_tile2 = nullptr;
	dmrgpp::LanczosWork* lanczos = nullptr;
	double*             d_diag = nullptr; // diagonal of H (patch order)
	int                 correction_precond = 0; // dmrgpp_correction_solve: DMRGPP_PRECOND_NONE or _JACOBI
	dmrgpp::DavidsonWork* davidson = nullptr;
	dmrgpp::GroupWork*  group = nullptr;   // group Lanczos buffers (group_lanczos.cu)
	const dmrgpp::CrsSource* crs = nullptr; // create time only: build the blocks from CRS operators
	std::string         err;
};

namespace dmrgpp {

// Enqueues y = H x on h->stream (device pointers); no synchronisation.  With
// io, the kernels read x and y from io on the device instead (for captured,
// replayed solver steps).
int kron_apply_device(dmrgpp_kron_handle h, const double* x, double* y,
                      const dmrgpp::StepIO* io = nullptr);

// Copies the caller's blocks (h->plan.blocks) into the packed FP64 operators
// h->d_ops through pinned staging buffers and a placement kernel, and waits
// for it; seconds_fill (optional) receives the host time spent copying into
// the staging buffers.
int upload_operators(dmrgpp_kron_handle h, double* seconds_fill);

// Allocates h->d_diag and computes the diagonal of H on the device from the
// packed operators (after upload_operators); waits for it.
int upload_diagonal(dmrgpp_kron_handle h);

// Host planning of the TF32x3 tensor-core form: plan.mixed, the per-CTA
// tile runs, the x map and the device packing jobs.  Reads h->plan and
// writes only h->plan.mixed and out, so it may run on another thread while
// the FP64 operators are uploaded.
struct MixedHost {
	bool                 ready = false;
	std::string          msg;
	std::vector<int>     xmap, starts1, starts2;
	int                  grid1 = 0, grid2 = 0;
	std::vector<PackJob> jobs;
};
void mixed_host_plan(dmrgpp_kron_handle h, int sms, MixedHost& out);

// Uploads the TF32x3 form planned in host (create time only, after the FP64
// operators are on the device).
int build_mixed(dmrgpp_kron_handle h, MixedHost& host);

// Writes the packed operators of a handle made by dmrgpp_kron_create_crs from
// h->crs (crs.cu), in place of upload_operators.
int upload_operators_crs(dmrgpp_kron_handle h);

// (Re)builds and uploads the schedule of h for configuration cfg: the
// persistent two-pass form for cfg in 0..kNumTileCfgs-1 (items_per_cta work
// items per CTA), the fused form (kron_fused.cuh) for kNumTileCfgs + f
// (items_per_cta parts per SM).
int configure_schedule(dmrgpp_kron_handle h, int cfg, int items_per_cta);

// Records msg as the handle's last error and returns status.
int handle_fail(dmrgpp_kron_handle h, int status, const std::string& msg);

// Interleaved complex (re, im pairs) <-> real embedding [re parts; im parts]
// of n complex values, enqueued on stream (complex.cu).
cudaError_t complex_split(const double* interleaved, double* split, size_t n, cudaStream_t stream);
cudaError_t complex_join(const double* split, double* interleaved, size_t n, cudaStream_t stream);

// Releases the eigensolver buffers of a handle (lanczos.cu).
void release_lanczos(dmrgpp_kron_handle h);
void release_davidson(dmrgpp_kron_handle h);
void release_group(dmrgpp_kron_handle h);

} // namespace dmrgpp
