// Fused form of the sector H*x for sectors of small patches (see
// kron_fused.cu): both passes of one output tile in one CTA, the tile's work
// split over the CTAs of a thread-block cluster and summed through
// distributed shared memory.
#pragma once

#include "kron_plan.h"

#include <cuda_runtime.h>

namespace dmrgpp {

struct FusedArgs {
	const double*    ops;   // packed Bstack_j and A^T blocks (the persistent form's layout)
	const double*    x;     // sector vector in
	double*          y;     // sector vector out
	const FusedItem* items; // one per CTA, cluster by cluster
	const FusedUnit* units;
	const int*       sector_active; // NULL, or per sector: 0 = skip (y left as is)
	const StepIO*    io;            // NULL, or x and y to read on the device
	int              n_items;       // cluster slots x cluster size
	int              max_clusters;  // co-resident clusters (fused_init); the grid holds at most this many
};

// Fused configurations (output rows BM, unit width CW in input columns,
// output columns BN, cluster size):
//   0: 32, 64, 128, 8     1: 32, 64, 128, 16
constexpr int kNumFusedCfgs = 2;

struct FusedShape {
	int bm, cw, bn, cluster;
};
FusedShape fused_shape(int fcfg);

// Sets the kernel attributes of configuration fcfg on the current device and
// returns how many of its clusters can be resident at once.
cudaError_t fused_init(int fcfg, int* clusters);

cudaError_t launch_fused(const FusedArgs& a, int fcfg, cudaStream_t stream);

} // namespace dmrgpp
