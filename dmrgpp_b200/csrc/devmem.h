// Device memory of handles and solver workspaces.
//
// A DMRG sweep creates one sector handle per step and destroys the previous
// one: the same few GB (packed operators, BX, the Lanczos basis) are freed
// and allocated again every step.  cudaMalloc of fresh device memory costs up
// to a few hundred ms per GB-sized buffer, so these buffers come from one
// stream-ordered memory pool per device that keeps freed memory for reuse
// (release threshold: unlimited) until dmrgpp_release_cached_memory trims it.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

namespace dmrgpp {

// bytes on the current device; the memory is ready for use on any stream
// when the call returns
cudaError_t dev_malloc_bytes(void** p, size_t bytes);

// Returns p to the pool after waiting for all work on the device (the same
// implicit synchronisation as cudaFree).  Null is ignored.
void dev_free(void* p);

// A mapped pinned int (zeroed) for a kernel-to-host error word, from slabs
// shared by all handles of the process (a cudaHostAlloc per handle costs
// milliseconds).  *dev is the device view of *host.
cudaError_t error_word_alloc(int** host, int** dev);
void        error_word_free(int* host);

// Copies and clears ordered on the handle's stream st.  A caller's stream
// may be non-blocking (torch's streams are), and such a stream is not
// ordered with the legacy default stream that cudaMemcpy / cudaMemset use:
// a clear there could land after a kernel on st has written the buffer.
// upload_sync / download_sync return once the bytes have arrived.
cudaError_t upload_sync(void* dst, const void* src, size_t bytes, cudaStream_t st);
cudaError_t download_sync(void* dst, const void* src, size_t bytes, cudaStream_t st);
cudaError_t clear_async(void* dst, size_t bytes, cudaStream_t st);

template <class T> cudaError_t dev_malloc(T** p, size_t bytes)
{
	return dev_malloc_bytes(reinterpret_cast<void**>(p), bytes);
}

} // namespace dmrgpp
