// Interleaved complex vectors <-> the real embedding used by complex sectors
// (dmrgpp_kron_create_complex): [Re x (patch order); Im x (patch order)].
#include "handle.h"

namespace dmrgpp {
namespace {

// std::complex<double> is only 8-byte aligned: plain double accesses
__global__ void __launch_bounds__(256) split_kernel(const double* __restrict__ z, double* __restrict__ re,
                                                   double* __restrict__ im, size_t n)
{
	for (size_t e = blockIdx.x * size_t(256) + threadIdx.x; e < n; e += size_t(gridDim.x) * 256) {
		re[e] = z[2 * e];
		im[e] = z[2 * e + 1];
	}
}

__global__ void __launch_bounds__(256) join_kernel(const double* __restrict__ re, const double* __restrict__ im,
                                                  double* __restrict__ z, size_t n)
{
	for (size_t e = blockIdx.x * size_t(256) + threadIdx.x; e < n; e += size_t(gridDim.x) * 256) {
		z[2 * e]     = re[e];
		z[2 * e + 1] = im[e];
	}
}

unsigned blocks_for(size_t n)
{
	const size_t b = (n + 255) / 256;
	return unsigned(b < 148 * 8 ? (b > 0 ? b : 1) : 148 * 8);
}

} // namespace

cudaError_t complex_split(const double* interleaved, double* split, size_t n, cudaStream_t stream)
{
	if (n == 0)
		return cudaSuccess;
	split_kernel<<<blocks_for(n), 256, 0, stream>>>(interleaved, split, split + n, n);
	return cudaGetLastError();
}

cudaError_t complex_join(const double* split, double* interleaved, size_t n, cudaStream_t stream)
{
	if (n == 0)
		return cudaSuccess;
	join_kernel<<<blocks_for(n), 256, 0, stream>>>(split, split + n, interleaved, n);
	return cudaGetLastError();
}

} // namespace dmrgpp
