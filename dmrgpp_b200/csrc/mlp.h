// Learned Davidson preconditioner (mlp.cu): a per-element MLP
//   features(d_e - theta, r_e, theta, |r|) -> 256 -> 256 -> 1 (tanh hidden layers)
// mapping the sector diagonal, the residual and the Ritz value to the
// correction of the next Davidson step.
#pragma once

#include "dmrgpp_kron.h"

#include <cuda_runtime.h>

namespace dmrgpp {

constexpr int kMlpFeatures = 4;
constexpr int kMlpWidth    = 256;

// t = correction for residual r at Ritz value theta (|r| = rnorm), n elements.
int mlp_precondition(dmrgpp_mlp_handle m, const double* diag, const double* r, double theta,
                     double rnorm, double* t, size_t n, cudaStream_t stream);

// The same for the concatenated vectors of nsec sectors (device arrays:
// sector_start has nsec + 1 offsets, theta and rnorm one value per sector);
// every element sees its own sector's scalars.
int mlp_precondition_group(dmrgpp_mlp_handle m, const double* diag, const double* r,
                           const long long* sector_start, const double* theta, const double* rnorm,
                           int nsec, double* t, size_t n, cudaStream_t stream);

} // namespace dmrgpp
