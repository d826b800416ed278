// Staged upload of the FP64 packed operators at create time (UploadPlan in
// kron_plan.h).  The reference plugin copies the caller's blocks into its own
// slabs in the constructor (setup_sparse_batch.cpp:281-343); here the copy is
// a pipeline: host threads copy the blocks of chunk c into one of two pinned
// buffers while chunk c-1 crosses PCIe, and a kernel places each chunk's parts
// in the packed buffer on the device (the A transposes run there, at HBM
// speed, instead of as strided host loops).
#include "devmem.h"
#include "handle.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <functional>
#include <map>
#include <mutex>
#include <thread>

namespace dmrgpp {

namespace {

constexpr long long kChunkElems = 4ll << 20;  // 32 MB per chunk
constexpr long long kJobElems   = 64ll << 10; // 512 KB per part at most
constexpr int       kSlots      = 2;          // pinned buffers (and device chunks)

// Pinned host buffers of one device, kept for the life of the process (the
// first create pays their allocation; later creates reuse them).  The mutex
// serialises uploads from several host threads.
struct PinnedPool {
	std::mutex  mu;
	double*     buf[kSlots] = {};
	long long   elems       = 0;
	cudaEvent_t copied[kSlots] = {};
};

PinnedPool& pool_of(int device)
{
	static std::mutex                      mu;
	static std::map<int, PinnedPool*>      pools; // never freed: outlive every handle
	std::lock_guard<std::mutex>            g(mu);
	PinnedPool*&                           p = pools[device];
	if (!p)
		p = new PinnedPool();
	return *p;
}

cudaError_t reserve(PinnedPool& p, long long elems)
{
	cudaError_t e = cudaSuccess;
	if (!p.copied[0])
		for (int s = 0; s < kSlots; ++s)
			if ((e = cudaEventCreateWithFlags(&p.copied[s], cudaEventDisableTiming)))
				return e;
	if (p.elems >= elems)
		return cudaSuccess;
	for (int s = 0; s < kSlots; ++s) {
		if (p.buf[s]) {
			cudaFreeHost(p.buf[s]);
			p.buf[s] = nullptr;
		}
	}
	p.elems = 0;
	for (int s = 0; s < kSlots; ++s)
		if ((e = cudaHostAlloc(reinterpret_cast<void**>(&p.buf[s]), size_t(elems) * sizeof(double),
		                       cudaHostAllocPortable)))
			return e;
	p.elems = elems;
	return cudaSuccess;
}

// A fixed team of host threads that runs f(0..n-1) with the caller taking
// part; kept for a whole upload so that each chunk costs a wake-up, not a
// thread start per core.
class Team {
public:
	explicit Team(size_t helpers)
	{
		for (size_t t = 0; t < helpers; ++t)
			threads_.emplace_back([this] { loop(); });
	}
	~Team()
	{
		{
			std::lock_guard<std::mutex> g(mu_);
			quit_ = true;
			++gen_;
		}
		wake_.notify_all();
		for (std::thread& th : threads_)
			th.join();
	}
	void run(size_t n, const std::function<void(size_t)>& f)
	{
		{
			std::lock_guard<std::mutex> g(mu_);
			f_      = &f;
			n_      = n;
			next_.store(0);
			busy_ = threads_.size();
			++gen_;
		}
		wake_.notify_all();
		work();
		std::unique_lock<std::mutex> lk(mu_);
		done_.wait(lk, [this] { return busy_ == 0; });
		f_ = nullptr;
	}

private:
	void work()
	{
		for (;;) {
			const size_t i = next_.fetch_add(1);
			if (i >= n_)
				break;
			(*f_)(i);
		}
	}
	void loop()
	{
		unsigned long long seen = 0;
		for (;;) {
			{
				std::unique_lock<std::mutex> lk(mu_);
				wake_.wait(lk, [&] { return gen_ != seen; });
				seen = gen_;
				if (quit_)
					return;
			}
			work();
			std::lock_guard<std::mutex> g(mu_);
			if (--busy_ == 0)
				done_.notify_one();
		}
	}
	std::vector<std::thread>             threads_;
	std::mutex                           mu_;
	std::condition_variable              wake_, done_;
	const std::function<void(size_t)>*   f_    = nullptr;
	size_t                               n_    = 0;
	std::atomic<size_t>                  next_ { 0 };
	size_t                               busy_ = 0;
	unsigned long long                   gen_  = 0;
	bool                                 quit_ = false;
};

// One CTA per part: a column copy (lanes along the rows) or a 32 x 32 tiled
// transpose through shared memory (reads along the block's rows, writes along
// the transposed rows).
__global__ void __launch_bounds__(256) upload_place_kernel(const UploadJob* __restrict__ jobs,
                                                          const double* __restrict__ chunk,
                                                          double* __restrict__ ops)
{
	__shared__ double tile[32][33];
	const UploadJob j    = jobs[blockIdx.x];
	const double*   src  = chunk + j.src;
	double*         dst  = ops + j.dst;
	const int       lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	if (!j.transpose) {
		for (int c = warp; c < j.cols; c += 8) {
			const double* s = src + (long long)c * j.rows;
			double*       d = dst + (long long)c * j.ld_dst;
			for (int q = lane; q < j.rows; q += 32)
				d[q] = s[q];
		}
		return;
	}
	for (int q0 = 0; q0 < j.rows; q0 += 32)
		for (int c0 = 0; c0 < j.cols; c0 += 32) {
			for (int c = warp; c < 32; c += 8)
				if (q0 + lane < j.rows && c0 + c < j.cols)
					tile[c][lane] = src[(long long)(c0 + c) * j.rows + q0 + lane];
			__syncthreads();
			for (int q = warp; q < 32; q += 8)
				if (q0 + q < j.rows && c0 + lane < j.cols)
					dst[(long long)(q0 + q) * j.ld_dst + c0 + lane] = tile[lane][q];
			__syncthreads();
		}
}

// Diagonal of H, patch by patch, from the packed operators: element
// (iR, iL) of patch i is the sum over its diagonal triples, in triple order,
// of A_k(i,i)(iL,iL) * B_k(i,i)(iR,iR) (unfused multiply and add, as on the
// host).
struct DiagPatch {
	long long y_off; // xy_start[i]
	int       rows;  // r_i
	int       cols;  // l_i
	int       first; // terms [first, first + count)
	int       count;
};
struct DiagTerm {
	long long a_off; // A^T block (l_i x l_i, leading dimension l_i)
	long long b_off; // B block inside Bstack_i (leading dimension M_i)
	int       lda;
	int       ldb;
};

__global__ void __launch_bounds__(256) diagonal_kernel(const DiagPatch* __restrict__ patches,
                                                      const DiagTerm* __restrict__ terms,
                                                      const double* __restrict__ ops,
                                                      double* __restrict__ diag)
{
	const DiagPatch p = patches[blockIdx.x];
	const long long n = (long long)p.rows * p.cols;
	for (long long e = threadIdx.x; e < n; e += blockDim.x) {
		const long long ir = e % p.rows, il = e / p.rows;
		double          d  = 0.0;
		for (int t = p.first; t < p.first + p.count; ++t) {
			const DiagTerm& q = terms[t];
			d                 = __dadd_rn(d, __dmul_rn(ops[q.a_off + il + il * q.lda], ops[q.b_off + ir + ir * q.ldb]));
		}
		diag[p.y_off + e] = d;
	}
}

} // namespace

int upload_diagonal(dmrgpp_kron_handle h)
{
	const KronPlan&        P = h->plan;
	std::vector<DiagPatch> patches;
	std::vector<DiagTerm>  terms;
	// triples are in (i,j,k) order, so each patch's diagonal terms are contiguous
	int last = -1;
	for (size_t t = 0; t < P.triples.size(); ++t) {
		const Triple& tr = P.triples[t];
		if (tr.i != tr.j)
			continue;
		if (tr.i != last) {
			last = tr.i;
			patches.push_back({ P.xy_start[tr.i], int(P.r[tr.i]), int(P.l[tr.i]), int(terms.size()), 0 });
		}
		terms.push_back({ P.at_off[t], P.bstack_off[tr.i] + P.row_off[t], int(P.l[tr.i]), int(P.M[tr.i]) });
		++patches.back().count;
	}
	const size_t D = size_t(std::max<long long>(P.dim(), 1));
	cudaError_t  e;
	if ((e = dev_malloc(&h->d_diag, D * sizeof(double)))
	    || (e = cudaMemsetAsync(h->d_diag, 0, D * sizeof(double), h->stream)))
		return handle_fail(h, DMRGPP_CUDA_ERROR, std::string("diagonal: ") + cudaGetErrorString(e));
	if (patches.empty())
		return cudaStreamSynchronize(h->stream) == cudaSuccess ? DMRGPP_OK
		                                                       : handle_fail(h, DMRGPP_CUDA_ERROR, "diagonal");
	void* buf = nullptr;
	const size_t pb = patches.size() * sizeof(DiagPatch), tb = terms.size() * sizeof(DiagTerm);
	std::vector<unsigned char> host(pb + tb);
	std::memcpy(host.data(), patches.data(), pb);
	std::memcpy(host.data() + pb, terms.data(), tb);
	if ((e = dev_malloc(&buf, host.size()))
	    || (e = cudaMemcpyAsync(buf, host.data(), host.size(), cudaMemcpyHostToDevice, h->stream))) {
		dev_free(buf);
		return handle_fail(h, DMRGPP_CUDA_ERROR, std::string("diagonal: ") + cudaGetErrorString(e));
	}
	diagonal_kernel<<<unsigned(patches.size()), 256, 0, h->stream>>>(
	    static_cast<const DiagPatch*>(buf),
	    reinterpret_cast<const DiagTerm*>(static_cast<unsigned char*>(buf) + pb), h->d_ops, h->d_diag);
	e = cudaGetLastError();
	if (e == cudaSuccess)
		e = cudaStreamSynchronize(h->stream);
	dev_free(buf);
	return e == cudaSuccess ? DMRGPP_OK
	                        : handle_fail(h, DMRGPP_CUDA_ERROR, std::string("diagonal: ") + cudaGetErrorString(e));
}

int upload_operators(dmrgpp_kron_handle h, double* seconds_fill)
{
	const UploadPlan up = build_upload_plan(h->plan, kChunkElems, kJobElems);
	if (up.jobs.empty())
		return DMRGPP_OK;
	PinnedPool&                  p = pool_of(h->device);
	std::lock_guard<std::mutex>  g(p.mu);
	cudaError_t                  e;
	if ((e = reserve(p, up.chunk_elems)))
		return handle_fail(h, DMRGPP_CUDA_ERROR, std::string("pinned staging: ") + cudaGetErrorString(e));

	double*    d_chunk[kSlots] = {};
	UploadJob* d_jobs          = nullptr;
	auto       cleanup = [&](int rc, const std::string& why) {
                cudaStreamSynchronize(h->stream);
                for (int s = 0; s < kSlots; ++s)
                        dmrgpp::dev_free(d_chunk[s]);
                dmrgpp::dev_free(d_jobs);
                return rc == DMRGPP_OK ? rc : handle_fail(h, rc, why);
	};
	const size_t nslots = std::min<size_t>(kSlots, up.chunks());
	for (size_t s = 0; s < nslots; ++s)
		if ((e = dmrgpp::dev_malloc(&d_chunk[s], size_t(up.chunk_elems) * sizeof(double))))
			return cleanup(DMRGPP_CUDA_ERROR, std::string("device allocation (upload chunk): ") + cudaGetErrorString(e));
	if ((e = dmrgpp::dev_malloc(&d_jobs, up.jobs.size() * sizeof(UploadJob)))
	    || (e = cudaMemcpyAsync(d_jobs, up.jobs.data(), up.jobs.size() * sizeof(UploadJob),
	                            cudaMemcpyHostToDevice, h->stream)))
		return cleanup(DMRGPP_CUDA_ERROR, std::string("upload jobs: ") + cudaGetErrorString(e));

	const size_t helpers = size_t(host_threads()) - 1;
	Team         team(helpers);
	double       fill_s = 0.0;
	for (size_t c = 0; c < up.chunks(); ++c) {
		const int    slot  = int(c % kSlots);
		const size_t first = up.chunk_begin[c], n = up.chunk_begin[c + 1] - first;
		if (n == 0)
			continue;
		// the pinned buffer's previous chunk must have left before it is refilled
		if (c >= size_t(kSlots) && (e = cudaEventSynchronize(p.copied[slot])))
			return cleanup(DMRGPP_CUDA_ERROR, std::string("upload wait: ") + cudaGetErrorString(e));
		const auto t0 = std::chrono::steady_clock::now();
		double*    buf = p.buf[slot];
		// parts in groups of ~8 per task keep the per-task overhead small
		const size_t                      per  = 8, tasks = (n + per - 1) / per;
		const std::function<void(size_t)> fill = [&](size_t t) {
			fill_upload_chunk(up, c, t * per, std::min(n, (t + 1) * per), buf);
		};
		team.run(tasks, fill);
		fill_s += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
		// the device chunk was last read by the kernel two chunks back, which
		// precedes this copy on the stream
		if ((e = cudaMemcpyAsync(d_chunk[slot], buf, size_t(up.chunk_fill[c]) * sizeof(double),
		                         cudaMemcpyHostToDevice, h->stream)))
			return cleanup(DMRGPP_CUDA_ERROR, std::string("upload copy: ") + cudaGetErrorString(e));
		upload_place_kernel<<<unsigned(n), 256, 0, h->stream>>>(d_jobs + first, d_chunk[slot], h->d_ops);
		if ((e = cudaGetLastError()) || (e = cudaEventRecord(p.copied[slot], h->stream)))
			return cleanup(DMRGPP_CUDA_ERROR, std::string("upload place: ") + cudaGetErrorString(e));
	}
	if ((e = cudaStreamSynchronize(h->stream)))
		return cleanup(DMRGPP_CUDA_ERROR, std::string("upload: ") + cudaGetErrorString(e));
	if (seconds_fill)
		*seconds_fill = fill_s;
	return cleanup(DMRGPP_OK, "");
}

} // namespace dmrgpp
