// Persistent single-launch form of the sector H*x (see kron_persistent.cu).
#pragma once

#include "kron_plan.h"

#include <cuda_runtime.h>

namespace dmrgpp {

struct PersistentArgs {
	const double*   ops;     // packed Bstack_j and A^T blocks
	const double*   x;       // sector vector in
	double*         bx;      // pass-1 results
	double*         y;       // sector vector out
	double*         partial; // split-K partial tiles
	const GemmSeg*  seg1;
	const GemmSeg*  pseg2;
	const KronItem* items;
	const int*      n1_of_j;
	unsigned*       work_counter; // [0] next item, [1] CTAs that left, [2] abort
	unsigned*       done;         // per input patch: finished pass-1 tiles
	unsigned*       arrive;       // per split tile: finished parts
	int*            error;        // set to nonzero when a wait gave up
	const int*      item_sector;   // per item: its sector (group handles)
	const int*      sector_active; // NULL, or per sector: 0 = skip its items (y left as is)
	const StepIO*   io;            // NULL, or x and y to read on the device (replaces x, y)
	int             n_items;
	int             np;
	int             n_split_tiles;
	int             test_extra_wait; // 0; >0 makes waits on patch 0 unsatisfiable (tests)
};

// Tile configurations (output tile, k-chunk, pipeline depth):
//   0: 32x32, k16, 4 stages   1: 32x32, k32, 3 stages
//   2: 64x64, k16, 3 stages   3: 64x64, k32, 3 stages
//   4: 32x32, k32, 4 stages   5: 32x32, k64, 3 stages
constexpr int kNumTileCfgs = 6;

// Sets kernel attributes of configuration cfg on the current device and
// returns its persistent grid (SMs x resident CTAs), tile edge and k-chunk.
cudaError_t persistent_config(int cfg, int* grid, int* tile, int* bk);

cudaError_t launch_persistent(const PersistentArgs& a, int cfg, int grid, cudaStream_t stream);

} // namespace dmrgpp
