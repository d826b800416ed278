// Host-side plan of the patch-wise wave-function transformation
// (dmrgpp_wft_* in dmrgpp_kron.h): for every output patch q with source
// input patch p,
//     T_q = WR_q * X_p          (pass A: r_out[q] x l_in[p], K = r_in[p])
//     Y_q = T_q * WL_q^T        (pass B: r_out[q] x l_out[q], K = l_in[p])
// as two grouped FP64 GEMMs (kron_gemm.cuh).  The transformation blocks are
// packed once: WR_q column-major r_out[q] x r_in[p] (the A operand of pass A)
// and WL_q^T column-major l_in[p] x l_out[q] (the B operand of pass B, K
// contiguous).  The reference applies the same two products per patch
// (BlockDiagWf.h:174-258, two GemmR calls).
#pragma once

#include "dmrgpp_kron.h"
#include "kron_plan.h"

#include <string>
#include <vector>

namespace dmrgpp {

struct WftPlan {
	size_t                 np_in = 0, np_out = 0;
	std::vector<long long> l_in, r_in, l_out, r_out, src;
	std::vector<long long> x_start, y_start; // np + 1 offsets of each layout
	std::vector<long long> wr_off, wlt_off, t_off; // per output patch (0 without a source)
	long long              op_elems = 0, t_elems = 0;
	double                 flops    = 0.0;
	int                    bm = 64, bn = 64;
	std::vector<GemmSeg>   segA, segB;
	std::vector<GemmTile>  tileA, tileB;
	long long dim_in() const { return x_start.empty() ? 0 : x_start.back(); }
	long long dim_out() const { return y_start.empty() ? 0 : y_start.back(); }
};

// Validates the descriptor and builds the plan; packed (optional) receives
// the packed transformation blocks (op_elems doubles).  Returns "" or the
// reason the descriptor is invalid.
std::string build_wft_plan(const dmrgpp_wft_desc& d, WftPlan& plan, std::vector<double>* packed);

} // namespace dmrgpp
