// FP64 grouped GEMM used by both Kronecker passes.
//
// One CTA computes one output tile C[m0:m0+BM, n0:n0+BN] of a column-major
// M x N matrix as the sum, over its K-segments, of A_s(M x K_s) * B_s(K_s x N)
// with both operands column-major (A M-contiguous, B K-contiguous).  Tiles of
// ragged size are handled by zero-filled copies.
//
// Arithmetic: FP64 tensor-core MMA (mma.sync m8n8k4 .f64), the FP64 tensor
// pipe of sm_100a (tcgen05 has no FP64 kind).  Operands are staged
// global -> shared with cp.async (zero-fill for out-of-range elements) in a
// STAGES-deep ring; every element is read from global memory once per tile.
#pragma once

#include "kron_plan.h"

#include <cuda_runtime.h>

namespace dmrgpp {

struct GemmArgs {
	const double*   A;     // base of all A operands of this pass
	const double*   B;     // base of all B operands of this pass
	double*         C;     // base of all outputs of this pass
	const GemmSeg*  segs;
	const GemmTile* tiles;
	int             ntiles;
};

// Raises the dynamic shared-memory limit of the kernels on the current
// device; call once per device before the first launch.
cudaError_t init_grouped_dgemm();

// Launches one grouped-GEMM pass over args.ntiles tiles of bm x bn.
cudaError_t launch_grouped_dgemm(const GemmArgs& args, int bm, int bn, cudaStream_t stream);

} // namespace dmrgpp
