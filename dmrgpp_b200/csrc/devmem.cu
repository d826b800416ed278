// Stream-ordered device memory pool of the library (devmem.h).
#include "devmem.h"
#include "dmrgpp_kron.h"

#include <algorithm>
#include <cstdint>
#include <map>
#include <mutex>
#include <unordered_map>
#include <vector>

namespace dmrgpp {

namespace {

// Blocks of 64 MB and more (the packed operators, BX, the solver bases)
// are kept on a free list when released and handed out again to a request
// of their size class or up to a quarter smaller.  Measured on the C3 sweep
// (1 GB and 3 GB Lanczos bases every step, sizes shifting by a few percent):
// the pool's own reuse of such blocks took 0.1-2 s on one call in ten while
// the pool did not grow; a free-list hit is a map lookup.
constexpr size_t kLargeBlock = size_t(64) << 20;

struct DevicePool {
	cudaMemPool_t pool   = nullptr;
	cudaStream_t  stream = nullptr; // allocations and frees are ordered on it
	std::mutex                       mu;     // the two maps below
	std::multimap<size_t, void*>     free_large; // size -> block
	std::unordered_map<void*, size_t> large;     // every live or free large block -> size
	size_t                           free_bytes = 0;
};

std::mutex& pools_mutex()
{
	static std::mutex mu;
	return mu;
}

std::map<int, DevicePool>& pools() // never freed: outlive every handle
{
	static std::map<int, DevicePool>* p = new std::map<int, DevicePool>();
	return *p;
}

cudaError_t pool_of(int device, DevicePool** out)
{
	std::lock_guard<std::mutex> g(pools_mutex());
	DevicePool&                 d = pools()[device];
	if (!d.pool) {
		cudaMemPoolProps props {};
		props.allocType     = cudaMemAllocationTypePinned;
		props.handleTypes   = cudaMemHandleTypeNone;
		props.location.type = cudaMemLocationTypeDevice;
		props.location.id   = device;
		cudaError_t e       = cudaMemPoolCreate(&d.pool, &props);
		if (e != cudaSuccess) {
			d.pool = nullptr;
			return e;
		}
		uint64_t keep = UINT64_MAX;
		int      prev = -1;
		if ((e = cudaMemPoolSetAttribute(d.pool, cudaMemPoolAttrReleaseThreshold, &keep))
		    || (e = cudaGetDevice(&prev)) || (e = cudaSetDevice(device))) {
			cudaMemPoolDestroy(d.pool);
			d.pool = nullptr;
			return e;
		}
		// the pool's stream belongs to its device
		e = cudaStreamCreateWithFlags(&d.stream, cudaStreamNonBlocking);
		cudaSetDevice(prev);
		if (e != cudaSuccess) {
			cudaMemPoolDestroy(d.pool);
			d.pool = nullptr;
			return e;
		}
	}
	*out = &d;
	return cudaSuccess;
}

// error words: one per 64-byte line, 1024 per slab, slabs never freed
constexpr int kWordStride = 16; // ints
constexpr int kSlabWords  = 1024;

struct WordSlabs {
	std::mutex        mu;
	std::vector<int*> free_words;
};

WordSlabs& word_slabs()
{
	static WordSlabs* w = new WordSlabs();
	return *w;
}

} // namespace

cudaError_t error_word_alloc(int** host, int** dev)
{
	WordSlabs&                  w = word_slabs();
	std::lock_guard<std::mutex> g(w.mu);
	if (w.free_words.empty()) {
		int*        slab = nullptr;
		cudaError_t e    = cudaHostAlloc(reinterpret_cast<void**>(&slab),
                                          size_t(kSlabWords) * kWordStride * sizeof(int),
                                          cudaHostAllocMapped | cudaHostAllocPortable);
		if (e != cudaSuccess)
			return e;
		for (int q = kSlabWords - 1; q >= 0; --q)
			w.free_words.push_back(slab + size_t(q) * kWordStride);
	}
	int* word = w.free_words.back();
	int* d    = nullptr;
	if (cudaError_t e = cudaHostGetDevicePointer(reinterpret_cast<void**>(&d), word, 0))
		return e;
	w.free_words.pop_back();
	*word = 0;
	*host = word;
	*dev  = d;
	return cudaSuccess;
}

void error_word_free(int* host)
{
	if (!host)
		return;
	WordSlabs&                  w = word_slabs();
	std::lock_guard<std::mutex> g(w.mu);
	w.free_words.push_back(host);
}

// Requests of 64 MB and more are rounded up to size classes (eight per
// factor of two, at most 12.5% more), so that the buffers of consecutive
// sweep steps, whose sizes differ by a few percent, fit blocks the pool
// already holds instead of making it map new memory.
size_t size_class(size_t bytes)
{
	if (bytes < (size_t(64) << 20))
		return bytes;
	int lg = 63;
	while (!(bytes >> lg))
		--lg;
	const size_t q = size_t(1) << (lg - 3);
	return (bytes + q - 1) / q * q;
}

cudaError_t dev_malloc_bytes(void** p, size_t bytes)
{
	bytes      = size_class(bytes);
	*p         = nullptr;
	int         device;
	cudaError_t e = cudaGetDevice(&device);
	DevicePool* d = nullptr;
	if (e || (e = pool_of(device, &d)))
		return e;
	if (bytes >= kLargeBlock) {
		std::lock_guard<std::mutex> g(d->mu);
		auto it = d->free_large.lower_bound(bytes);
		if (it != d->free_large.end() && it->first <= bytes + bytes / 4) {
			*p = it->second;
			d->free_bytes -= it->first;
			d->free_large.erase(it);
			return cudaSuccess;
		}
	}
	e = cudaMallocFromPoolAsync(p, bytes ? bytes : 1, d->pool, d->stream);
	if (e == cudaErrorMemoryAllocation) {
		// out of memory: the free list's blocks go back to the pool, then once more
		cudaGetLastError();
		{
			std::lock_guard<std::mutex> g(d->mu);
			for (const auto& kv : d->free_large) {
				d->large.erase(kv.second);
				cudaFreeAsync(kv.second, d->stream);
			}
			d->free_large.clear();
			d->free_bytes = 0;
		}
		e = cudaMallocFromPoolAsync(p, bytes ? bytes : 1, d->pool, d->stream);
	}
	if (e)
		return e;
	if ((e = cudaStreamSynchronize(d->stream)))
		return e;
	if (bytes >= kLargeBlock) {
		std::lock_guard<std::mutex> g(d->mu);
		d->large[*p] = bytes;
	}
	return cudaSuccess;
}

cudaError_t upload_sync(void* dst, const void* src, size_t bytes, cudaStream_t st)
{
	if (!bytes)
		return cudaSuccess;
	const cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st);
	return e ? e : cudaStreamSynchronize(st);
}

cudaError_t download_sync(void* dst, const void* src, size_t bytes, cudaStream_t st)
{
	if (!bytes)
		return cudaSuccess;
	const cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st);
	return e ? e : cudaStreamSynchronize(st);
}

cudaError_t clear_async(void* dst, size_t bytes, cudaStream_t st)
{
	return bytes ? cudaMemsetAsync(dst, 0, bytes, st) : cudaSuccess;
}

void dev_free(void* p)
{
	if (!p)
		return;
	int device;
	if (cudaGetDevice(&device) != cudaSuccess)
		return;
	DevicePool* d = nullptr;
	if (pool_of(device, &d) != cudaSuccess)
		return;
	cudaDeviceSynchronize();
	{
		std::lock_guard<std::mutex> g(d->mu);
		auto it = d->large.find(p);
		if (it != d->large.end()) { // kept for the next request of its size
			d->free_large.insert({ it->second, p });
			d->free_bytes += it->second;
			return;
		}
	}
	cudaFreeAsync(p, d->stream);
}

} // namespace dmrgpp

extern "C" {

int dmrgpp_release_cached_memory(int device)
{
	int         prev = -1;
	cudaError_t e    = cudaGetDevice(&prev);
	if (e != cudaSuccess)
		return DMRGPP_CUDA_ERROR;
	const int dev = device >= 0 ? device : prev;
	if (dev != prev && cudaSetDevice(dev) != cudaSuccess)
		return DMRGPP_INVALID_ARG;
	dmrgpp::DevicePool* d = nullptr;
	int                 rc = DMRGPP_OK;
	if (dmrgpp::pool_of(dev, &d) != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) {
		rc = DMRGPP_CUDA_ERROR;
	} else {
		{ // the free list's blocks go back to the pool first
			std::lock_guard<std::mutex> g(d->mu);
			for (const auto& kv : d->free_large) {
				d->large.erase(kv.second);
				cudaFreeAsync(kv.second, d->stream);
			}
			d->free_large.clear();
			d->free_bytes = 0;
		}
		if (cudaStreamSynchronize(d->stream) != cudaSuccess || cudaMemPoolTrimTo(d->pool, 0) != cudaSuccess)
			rc = DMRGPP_CUDA_ERROR;
	}
	if (dev != prev)
		cudaSetDevice(prev);
	return rc;
}

int dmrgpp_cached_memory(int device, size_t* reserved_bytes, size_t* used_bytes)
{
	if (!reserved_bytes || !used_bytes)
		return DMRGPP_INVALID_ARG;
	int prev = -1;
	if (cudaGetDevice(&prev) != cudaSuccess)
		return DMRGPP_CUDA_ERROR;
	const int           dev = device >= 0 ? device : prev;
	dmrgpp::DevicePool* d   = nullptr;
	if (dmrgpp::pool_of(dev, &d) != cudaSuccess)
		return DMRGPP_CUDA_ERROR;
	uint64_t res = 0, used = 0;
	if (cudaMemPoolGetAttribute(d->pool, cudaMemPoolAttrReservedMemCurrent, &res) != cudaSuccess
	    || cudaMemPoolGetAttribute(d->pool, cudaMemPoolAttrUsedMemCurrent, &used) != cudaSuccess)
		return DMRGPP_CUDA_ERROR;
	size_t kept = 0;
	{
		std::lock_guard<std::mutex> g(d->mu);
		kept = d->free_bytes;
	}
	*reserved_bytes = size_t(res);
	*used_bytes     = size_t(used) - std::min(size_t(used), kept); // free-listed blocks are not in use
	return DMRGPP_OK;
}

} // extern "C"
