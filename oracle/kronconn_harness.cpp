// Oracle harness (test infrastructure, never shipped): the reference's
// default, non-batched CPU H*x -- KronConnections::doTask
// (dmrg/Engine/MatrixVectorKron/KronConnections.h:124-181) over every output
// patch, each (input patch, term) block going to the reference's own
// den_kron_mult (dmrg/KronUtil/den_kron_mult.cpp:355-430, which picks method
// 1, 2 or 3 by its cost model and runs the products through GemmR ->
// kokkos_gemm -> dgemm_), compiled from the reference source where it lies.
//
// The task loop is restated here (the reference parallelises it with
// PsimagLite::Parallelizer over output patches, one GemmR per task with
// gemmRnb = 0 and one second-level thread, ParametersDmrgSolver.h:231-246);
// the blocks come from the GPU-plugin table convention (entry i + j*np +
// k*np*np, all dense, as the batched path densifies them) and the dense/sparse
// discount is the reference default DenseSparseThreshold = 0.2.
#include <PsimagLite/Matrix.h>
#include <PsimagLite/GemmR.h>
#include <PsimagLite/Vector.h>

#include "den_kron_mult.cpp"
#include "den_matmul_post.cpp"
#include "den_matmul_pre.cpp"
#include "estimate_kron_cost.cpp"

#include <dlfcn.h>

#include <atomic>
#include <cstddef>
#include <cstring>
#include <thread>
#include <vector>

namespace {

struct KronConn {
	size_t                                np = 0, nop = 0;
	std::vector<size_t>                   l, r, start;
	std::vector<PsimagLite::Matrix<double>*> A, B; // per table entry, nullptr = absent
	std::vector<double>                   x, y;

	~KronConn()
	{
		for (auto* m : A)
			delete m;
		for (auto* m : B)
			delete m;
	}
};

PsimagLite::Matrix<double>* copy_block(const double* src, size_t ld, size_t rows, size_t cols)
{
	if (!src)
		return nullptr;
	bool nonzero = false;
	auto* m      = new PsimagLite::Matrix<double>(rows, cols);
	for (size_t c = 0; c < cols; ++c)
		for (size_t q = 0; q < rows; ++q) {
			const double v = src[q + c * ld];
			(*m)(q, c)     = v;
			nonzero        = nonzero || v != 0.0;
		}
	if (!nonzero) { // an all-zero block is no connection (setup_nC.cpp:67-121)
		delete m;
		return nullptr;
	}
	return m;
}

} // namespace

extern "C" {

void* ref_kronconn_create(size_t nop, size_t np, const size_t* l, const size_t* r,
                          const double* const* A, const size_t* ldA, const double* const* B,
                          const size_t* ldB)
{
	auto* h = new KronConn;
	h->np   = np;
	h->nop  = nop;
	h->l.assign(l, l + np);
	h->r.assign(r, r + np);
	h->start.assign(np + 1, 0);
	for (size_t p = 0; p < np; ++p)
		h->start[p + 1] = h->start[p] + l[p] * r[p];
	const size_t nt = nop * np * np;
	h->A.assign(nt, nullptr);
	h->B.assign(nt, nullptr);
	for (size_t t = 0; t < nt; ++t) {
		const size_t i = t % np, j = (t / np) % np;
		if (!A[t] || !B[t])
			continue;
		h->A[t] = copy_block(A[t], ldA[t], l[i], l[j]);
		h->B[t] = copy_block(B[t], ldB[t], r[i], r[j]);
		if (!h->A[t] || !h->B[t]) {
			delete h->A[t];
			delete h->B[t];
			h->A[t] = h->B[t] = nullptr;
		}
	}
	h->x.resize(h->start[np]);
	h->y.resize(h->start[np]);
	return h;
}

// y = H x with `threads` workers over the output patches.
void ref_kronconn_apply(void* hv, const double* x, double* y, int threads)
{
	auto*        h  = static_cast<KronConn*>(hv);
	const size_t np = h->np, D = h->start[np];
	std::memcpy(h->x.data(), x, D * sizeof(double));
	std::fill(h->y.begin(), h->y.end(), 0.0);
	std::atomic<size_t> next { 0 };
	auto                work = [&] {
                PsimagLite::GemmR<double> gemmR(false, 0, 1);
                for (;;) {
                        const size_t outPatch = next.fetch_add(1);
                        if (outPatch >= np)
                                break;
                        for (size_t inPatch = 0; inPatch < np; ++inPatch)
                                for (size_t k = 0; k < h->nop; ++k) {
                                        const size_t t = outPatch + inPatch * np + k * np * np;
                                        if (!h->A[t] || !h->B[t])
                                                continue;
                                        den_kron_mult<double>('n', 'n', *h->A[t], *h->B[t], h->x,
                                                              h->start[inPatch], h->y,
                                                              h->start[outPatch], 0.2, gemmR);
                                }
                }
	};
	const int nt = threads > 0 ? threads : 1;
	// the task threads each call the BLAS: one BLAS thread per call, as
	// with the reference's Threads = cores and a single-threaded BLAS
	using SetThreads = void (*)(int);
	using GetThreads = int (*)();
	auto set_blas    = reinterpret_cast<SetThreads>(dlsym(RTLD_DEFAULT, "openblas_set_num_threads"));
	auto get_blas    = reinterpret_cast<GetThreads>(dlsym(RTLD_DEFAULT, "openblas_get_num_threads"));
	const int blas_before = (set_blas && get_blas) ? get_blas() : 0;
	if (set_blas && nt > 1)
		set_blas(1);
	std::vector<std::thread> pool;
	for (int q = 1; q < nt; ++q)
		pool.emplace_back(work);
	work();
	for (auto& th : pool)
		th.join();
	if (set_blas && nt > 1 && blas_before > 0)
		set_blas(blas_before);
	std::memcpy(y, h->y.data(), D * sizeof(double));
}

void ref_kronconn_destroy(void* h) { delete static_cast<KronConn*>(h); }

} // extern "C"
