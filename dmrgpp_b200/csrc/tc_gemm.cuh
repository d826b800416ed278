// Mixed-precision (TF32x3) grouped GEMM on tcgen05 tensor cores (tc_gemm.cu).
#pragma once

#include "kron_plan.h"

#include <cuda.h>
#include <cuda_runtime.h>

namespace dmrgpp {

struct TcArgs {
	// the pass's operand buffers as 2-D TMA tensors [row][32 floats]
	// (kron_plan.h): A with 128-row boxes, B with BN-row boxes; hi and lo
	CUtensorMap A_hi, A_lo, B_hi, B_lo;
	// pass 1: the split output buffers (hi, lo) as the same 2-D tensors with
	// 32-row boxes, for the epilogue's tiled TMA stores
	CUtensorMap C_hi_map, C_lo_map;
	float*          C_hi; // pass 1: K-major split output
	float*          C_lo;
	double*         Cd;   // pass 2: FP64 column-major output
	const GemmSeg*  segs;
	const GemmTile* tiles;  // CTA b processes tiles [starts[b], starts[b+1])
	const int*      starts; // grid + 1 entries (balance_tiles)
	int             ntiles;
	int             grid;   // persistent CTAs, at most one per SM
	int*            error; // set to 2 when an mbarrier wait gave up
	const StepIO*   io;    // NULL, or pass 2 writes io->y instead of Cd
	float*          partial; // pass 2: 128 x BN FP32 partial tiles of split parts (slots)
	unsigned*       arrive;  // pass 2: per split output tile, parts done (self-resetting)
	int             test_unarmed; // test hook: CTA 0's producer leaves its first stage unarmed
	const int*      tile_sector;   // group handles: per tile its sector (else NULL)
	const int*      sector_active; // NULL, or per sector: 0 = skip its tiles (C left as is)
};

// Kernel attributes on the current device; call once per device.
cudaError_t tc_init();

// One grouped pass over a.ntiles tiles of 128 x bn (bn = 64 or 128) by
// a.grid persistent CTAs.
cudaError_t tc_launch(const TcArgs& a, int bn, bool pass1, cudaStream_t stream);

// Runs the jobs (device array) on stream; hi/lo must be zeroed beforehand.
cudaError_t tc_pack_ops(const double* ops, float* hi, float* lo, const PackJob* jobs, int njobs,
                        cudaStream_t stream);

// x (patch order, FP64; io->x instead when io is given) -> TF32 hi/lo parts at map[e].
cudaError_t tc_split_x(const double* x, const int* map, float* hi, float* lo, long long n,
                       cudaStream_t stream, const StepIO* io = nullptr);

} // namespace dmrgpp
