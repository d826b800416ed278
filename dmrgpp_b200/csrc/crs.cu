// Block tables built on the device from the CRS operators
// (dmrgpp_kron_create_crs in dmrgpp_kron.h): the reference's InitKron set-up,
// InitKronBase::addOneConnection / calculateAhat (InitKronBase.h:249-272,
// 393-413) and ArrayOfMatStruct (ArrayOfMatStruct.h:105-448), whose per-patch
// slices the batched path densifies (BatchedGemmKokkos.h:354-370).
//
// Host: validation and the block-presence scan (which (i, j, k) blocks hold a
// nonzero of Ahat and of B), which fixes the plan exactly as the all-zero scan
// of dense tables does.  Device: each term's CRS arrays are copied as they
// are and one warp per row scatters the row's entries into the packed
// operators (A^T blocks and the B stacks of kron_plan.h), Ahat's entries
// formed as value * sign * a in the reference's order of operations.
#include "devmem.h"
#include "dmrgpp_kron.h"
#include "handle.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstring>
#include <string>
#include <vector>

namespace dmrgpp {

namespace {

// maps every basis state covered by a patch to (patch, index in its group);
// "" or the reason the groups cannot be mapped
std::string map_groups(size_t np, const size_t* off, const size_t* sz, size_t rows, const char* side,
                       std::vector<int>& patch, std::vector<int>& loc)
{
	patch.assign(rows, -1);
	loc.assign(rows, 0);
	for (size_t p = 0; p < np; ++p) {
		if (sz[p] < 1 || sz[p] > size_t(INT_MAX))
			return "patch " + std::to_string(p) + " has an empty or oversized " + side + " group";
		if (off[p] > rows || sz[p] > rows - off[p])
			return "patch " + std::to_string(p) + ": its " + side + " group runs past the basis";
		for (size_t s = off[p]; s < off[p] + sz[p]; ++s) {
			if (patch[s] >= 0)
				return std::string("the patches' ") + side + " groups overlap at state " + std::to_string(s);
			patch[s] = int(p);
			loc[s]   = int(s - off[p]);
		}
	}
	return std::string();
}

// presence of every (i, j) block of one CRS operator (row-major np x np
// bytes); "" or the reason the matrix is malformed
std::string scan_crs(const dmrgpp_crs& m, size_t rows, const std::vector<int>& patch, size_t np,
                     std::vector<unsigned char>& present)
{
	if (m.rows != rows)
		return "operator has " + std::to_string(m.rows) + " rows, the basis " + std::to_string(rows);
	if (!m.rowptr || (!m.colind && rows > 0 && m.rowptr[rows] > 0) || (!m.values && rows > 0 && m.rowptr[rows] > 0))
		return "null CRS array";
	if (m.rowptr[0] != 0)
		return "rowptr[0] must be 0";
	present.assign(np * np, 0);
	std::vector<int> seen(rows, -1); // row that last used each column: repeats
	for (size_t a = 0; a < rows; ++a) {
		const int e0 = m.rowptr[a], e1 = m.rowptr[a + 1];
		if (e1 < e0)
			return "rowptr decreases at row " + std::to_string(a);
		const int pi = patch[a];
		for (int e = e0; e < e1; ++e) {
			const int b = m.colind[e];
			if (b < 0 || size_t(b) >= rows)
				return "column index out of range in row " + std::to_string(a);
			if (seen[size_t(b)] == int(a))
				return "column " + std::to_string(b) + " repeated in row " + std::to_string(a);
			seen[size_t(b)] = int(a);
			const int pj    = patch[size_t(b)];
			if (pi >= 0 && pj >= 0 && m.values[e] != 0.0)
				present[size_t(pi) * np + size_t(pj)] = 1;
		}
	}
	return std::string();
}

struct ScatterArgs {
	const int*           rowptr;
	const int*           colind;
	const double*        values;
	int                  rows;
	const int*           patch;   // basis state -> patch (-1: none)
	const int*           loc;     // basis state -> index in its group
	const int*           tri_ptr; // (k * np + i) -> range of tri_j / tri_t
	const int*           tri_j;
	const int*           tri_t;
	int                  np, k;
	const long long*     dst; // per triple: base of the packed block
	const int*           ld;  // per triple: its leading dimension
	int                  transpose; // 1: (a, b) -> dst + loc[b] + loc[a] ld (A^T); 0: dst + loc[a] + loc[b] ld
	const unsigned char* parity;    // NULL or per state: odd -> sign -1
	double               value;
	double*              ops;
};

// one warp per CRS row: every entry of a contributing block goes to its
// packed position (a binary search over the row's patch's input patches)
__global__ void __launch_bounds__(256) k_scatter_crs(const ScatterArgs s)
{
	const int lane = threadIdx.x & 31;
	for (int a = blockIdx.x * 8 + (threadIdx.x >> 5); a < s.rows; a += gridDim.x * 8) {
		const int pi = s.patch[a];
		if (pi < 0)
			continue;
		const int base = s.tri_ptr[s.k * s.np + pi], end = s.tri_ptr[s.k * s.np + pi + 1];
		if (base == end)
			continue;
		const int    la   = s.loc[a];
		const double sign = (s.parity && s.parity[a]) ? -1.0 : 1.0;
		for (int e = s.rowptr[a] + lane; e < s.rowptr[a + 1]; e += 32) {
			const int b  = s.colind[e];
			const int pj = s.patch[b];
			if (pj < 0)
				continue;
			int lo = base, hi = end;
			while (lo < hi) {
				const int mid = (lo + hi) >> 1;
				if (s.tri_j[mid] < pj)
					lo = mid + 1;
				else
					hi = mid;
			}
			if (lo == end || s.tri_j[lo] != pj)
				continue;
			const int       t   = s.tri_t[lo];
			const int       lb  = s.loc[b];
			const long long off = s.transpose ? s.dst[t] + lb + (long long)la * s.ld[t]
			                                  : s.dst[t] + la + (long long)lb * s.ld[t];
			s.ops[off] = s.values[e] * sign * s.value; // calculateAhat's order
		}
	}
}

// Host arrays to the device through two page-locked buffers of the calling
// thread (kept between creates): the host cores copy one buffer's worth while
// the other crosses PCIe, so the copies run at the page-locked transfer rate
// instead of the pageable one.
struct Stager {
	static constexpr size_t kBytes = size_t(32) << 20;
	unsigned char*          buf[2] = {};
	cudaEvent_t             ev[2]  = {};
	bool                    used[2] = {};
	int                     slot   = 0;
	~Stager()
	{
		for (int s = 0; s < 2; ++s) {
			if (buf[s])
				cudaFreeHost(buf[s]);
			if (ev[s])
				cudaEventDestroy(ev[s]);
		}
	}
	cudaError_t ready()
	{
		cudaError_t e = cudaSuccess;
		for (int s = 0; s < 2 && !e; ++s) {
			if (!buf[s])
				e = cudaHostAlloc(reinterpret_cast<void**>(&buf[s]), kBytes, cudaHostAllocDefault);
			if (!e && !ev[s])
				e = cudaEventCreateWithFlags(&ev[s], cudaEventDisableTiming);
		}
		return e;
	}
	cudaError_t copy(void* dst, const void* src, size_t bytes, cudaStream_t st)
	{
		// small arrays: one pageable copy costs less than a staging round
		if (bytes < (size_t(8) << 20))
			return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st);
		cudaError_t e;
		for (size_t o = 0; o < bytes; o += kBytes) {
			const size_t n = std::min(kBytes, bytes - o);
			if (used[slot] && (e = cudaEventSynchronize(ev[slot])))
				return e;
			const size_t piece = size_t(1) << 20;
			unsigned char* b   = buf[slot];
			const unsigned char* s = static_cast<const unsigned char*>(src) + o;
			parallel_for((n + piece - 1) / piece, [&](size_t q) {
				std::memcpy(b + q * piece, s + q * piece, std::min(piece, n - q * piece));
			});
			if ((e = cudaMemcpyAsync(static_cast<unsigned char*>(dst) + o, b, n, cudaMemcpyHostToDevice, st))
			    || (e = cudaEventRecord(ev[slot], st)))
				return e;
			used[slot] = true;
			slot ^= 1;
		}
		return cudaSuccess;
	}
};

thread_local Stager g_stager;

} // namespace

std::string crs_triples(const dmrgpp_kron_crs_desc* d, CrsSource& src, std::vector<Triple>& triples,
                        std::vector<BlockRef>& blocks, double& f_alg)
{
	const size_t np = d->npatches, K = d->noperator;
	if (np == 0 || K == 0)
		return "noperator and npatches must be >= 1";
	if (!d->left_offset || !d->left_patch_size || !d->right_offset || !d->right_patch_size || !d->A || !d->B)
		return "null table or size array";
	if (np > 46340 || double(np) * double(np) * double(K) > double(1u << 31))
		return "too many patches for the CRS set-up";
	const size_t nL = d->A[0].rows, nR = d->B[0].rows;
	bool         any_fermion = false;
	for (size_t k = 0; k < K; ++k)
		any_fermion = any_fermion || (d->fermion && d->fermion[k]);
	if (any_fermion && !d->left_parity)
		return "a fermionic term needs the left states' parities";
	src.desc        = d;
	std::string msg = map_groups(np, d->left_offset, d->left_patch_size, nL, "left", src.lpatch, src.lloc);
	if (msg.empty())
		msg = map_groups(np, d->right_offset, d->right_patch_size, nR, "right", src.rpatch, src.rloc);
	if (!msg.empty())
		return msg;
	// presence of every block of every operator, all operators at once
	std::vector<std::vector<unsigned char>> pa(K), pb(K);
	std::vector<std::string>                err(2 * K);
	parallel_for(2 * K, [&](size_t q) {
		const size_t k = q / 2;
		if (q % 2 == 0)
			err[q] = scan_crs(d->A[k], nL, src.lpatch, np, pa[k]);
		else
			err[q] = scan_crs(d->B[k], nR, src.rpatch, np, pb[k]);
	});
	for (size_t q = 0; q < 2 * K; ++q)
		if (!err[q].empty())
			return std::string(q % 2 ? "B" : "A") + "[" + std::to_string(q / 2) + "]: " + err[q];
	// contributing triples in (i, j, k) order; a zero factor removes a term
	const size_t* l = d->left_patch_size;
	const size_t* r = d->right_patch_size;
	std::vector<std::vector<std::pair<int, int>>> lists(K * np);
	for (size_t i = 0; i < np; ++i)
		for (size_t j = 0; j < np; ++j)
			for (size_t k = 0; k < K; ++k) {
				if (!pa[k][i * np + j] || !pb[k][i * np + j] || (d->value && d->value[k] == 0.0))
					continue;
				lists[k * np + i].push_back({ int(j), int(triples.size()) });
				triples.push_back({ int(i), int(j), int(k) });
				blocks.push_back({ nullptr, 0, nullptr, 0 });
				f_alg += 2.0 * double(r[i]) * double(l[j]) * (double(r[j]) + double(l[i]));
			}
	src.tri_ptr.assign(K * np + 1, 0);
	src.tri_j.clear();
	src.tri_t.clear();
	for (size_t q = 0; q < K * np; ++q) {
		for (const auto& jt : lists[q]) { // j ascending (triples are in (i, j, k) order)
			src.tri_j.push_back(jt.first);
			src.tri_t.push_back(jt.second);
		}
		src.tri_ptr[q + 1] = int(src.tri_j.size());
	}
	return std::string();
}

int upload_operators_crs(dmrgpp_kron_handle h)
{
	const CrsSource&            src = *h->crs;
	const dmrgpp_kron_crs_desc* d   = src.desc;
	const KronPlan&             P   = h->plan;
	const size_t                nt  = P.triples.size();
	cudaStream_t                st  = h->stream;
	auto fail_cuda = [&](cudaError_t e, const char* where) {
		return handle_fail(h, e == cudaErrorMemoryAllocation ? DMRGPP_OOM : DMRGPP_CUDA_ERROR,
		                   std::string(where) + ": " + cudaGetErrorString(e));
	};
	// per triple: A^T block (ld l_j) and B block in Bstack_j (ld M_j)
	std::vector<long long> dst_a(std::max<size_t>(nt, 1)), dst_b(std::max<size_t>(nt, 1));
	std::vector<int>       ld_a(std::max<size_t>(nt, 1)), ld_b(std::max<size_t>(nt, 1));
	for (size_t t = 0; t < nt; ++t) {
		const Triple& tr = P.triples[t];
		dst_a[t]         = P.at_off[t];
		ld_a[t]          = int(P.l[size_t(tr.j)]);
		dst_b[t]         = P.bstack_off[size_t(tr.j)] + P.row_off[t];
		ld_b[t]          = int(P.M[size_t(tr.j)]);
	}
	const size_t K = d->noperator, nL = src.lpatch.size(), nR = src.rpatch.size();
	// every term's CRS arrays in one device buffer (16-byte aligned pieces)
	auto al = [](size_t b) { return (b + 15) / 16 * 16; };
	std::vector<size_t> crs_off(6 * K + 1, 0);
	for (size_t k = 0; k < K; ++k)
		for (int side = 0; side < 2; ++side) {
			const dmrgpp_crs& m    = side == 0 ? d->A[k] : d->B[k];
			const size_t      rows = side == 0 ? nL : nR;
			const size_t      nnz  = size_t(m.rowptr[rows]);
			const size_t      q    = 6 * k + 3 * size_t(side);
			crs_off[q + 1]         = crs_off[q] + al((rows + 1) * sizeof(int));
			crs_off[q + 2]         = crs_off[q + 1] + al(nnz * sizeof(int));
			crs_off[q + 3]         = crs_off[q + 2] + al(nnz * sizeof(double));
		}
	// one device buffer for the maps and lists
	std::vector<unsigned char> blob;
	std::vector<size_t>        offs;
	auto add = [&](const void* p, size_t bytes) {
		offs.push_back(blob.size());
		blob.resize(blob.size() + al(bytes));
		if (bytes)
			std::memcpy(blob.data() + offs.back(), p, bytes);
	};
	add(src.lpatch.data(), nL * sizeof(int));
	add(src.lloc.data(), nL * sizeof(int));
	add(src.rpatch.data(), nR * sizeof(int));
	add(src.rloc.data(), nR * sizeof(int));
	add(src.tri_ptr.data(), src.tri_ptr.size() * sizeof(int));
	add(src.tri_j.data(), src.tri_j.size() * sizeof(int));
	add(src.tri_t.data(), src.tri_t.size() * sizeof(int));
	add(dst_a.data(), dst_a.size() * sizeof(long long));
	add(ld_a.data(), ld_a.size() * sizeof(int));
	add(dst_b.data(), dst_b.size() * sizeof(long long));
	add(ld_b.data(), ld_b.size() * sizeof(int));
	add(d->left_parity ? d->left_parity : nullptr, d->left_parity ? nL : 0);
	unsigned char* d_blob = nullptr;
	unsigned char* d_crs  = nullptr;
	struct Free {
		unsigned char** a;
		unsigned char** b;
		~Free()
		{
			dev_free(*a);
			dev_free(*b);
		}
	} release { &d_blob, &d_crs };
	cudaError_t e;
	if ((e = dev_malloc(&d_blob, std::max<size_t>(blob.size(), 16)))
	    || (e = dev_malloc(&d_crs, std::max<size_t>(crs_off[6 * K], 16))) || (e = g_stager.ready()))
		return fail_cuda(e, "allocation (CRS set-up)");
	if ((e = cudaMemsetAsync(h->d_ops, 0, size_t(std::max<long long>(P.op_elems, 1)) * sizeof(double), st))
	    || (e = cudaMemcpyAsync(d_blob, blob.data(), blob.size(), cudaMemcpyHostToDevice, st)))
		return fail_cuda(e, "CRS set-up copies");
	if (P.triples.empty())
		return cudaStreamSynchronize(st) == cudaSuccess ? DMRGPP_OK
		                                                : handle_fail(h, DMRGPP_CUDA_ERROR, "CRS set-up");
	auto at = [&](int q) { return d_blob + offs[size_t(q)]; };
	for (size_t k = 0; k < K; ++k)
		for (int side = 0; side < 2; ++side) {
			const dmrgpp_crs& m    = side == 0 ? d->A[k] : d->B[k];
			const size_t      rows = side == 0 ? nL : nR;
			const size_t      nnz  = size_t(m.rowptr[rows]);
			const size_t      q    = 6 * k + 3 * size_t(side);
			int*              d_rowptr = reinterpret_cast<int*>(d_crs + crs_off[q]);
			int*              d_col    = reinterpret_cast<int*>(d_crs + crs_off[q + 1]);
			double*           d_val    = reinterpret_cast<double*>(d_crs + crs_off[q + 2]);
			if ((e = g_stager.copy(d_rowptr, m.rowptr, (rows + 1) * sizeof(int), st))
			    || (nnz && (e = g_stager.copy(d_col, m.colind, nnz * sizeof(int), st)))
			    || (nnz && (e = g_stager.copy(d_val, m.values, nnz * sizeof(double), st))))
				return fail_cuda(e, "CRS copy");
			ScatterArgs s {};
			s.rowptr    = d_rowptr;
			s.colind    = d_col;
			s.values    = d_val;
			s.rows      = int(rows);
			s.patch     = reinterpret_cast<const int*>(at(side == 0 ? 0 : 2));
			s.loc       = reinterpret_cast<const int*>(at(side == 0 ? 1 : 3));
			s.tri_ptr   = reinterpret_cast<const int*>(at(4));
			s.tri_j     = reinterpret_cast<const int*>(at(5));
			s.tri_t     = reinterpret_cast<const int*>(at(6));
			s.np        = int(P.np);
			s.k         = int(k);
			s.dst       = reinterpret_cast<const long long*>(at(side == 0 ? 7 : 9));
			s.ld        = reinterpret_cast<const int*>(at(side == 0 ? 8 : 10));
			s.transpose = side == 0 ? 1 : 0;
			s.parity    = (side == 0 && d->fermion && d->fermion[k]) ? reinterpret_cast<const unsigned char*>(at(11))
			                                                         : nullptr;
			s.value     = (side == 0 && d->value) ? d->value[k] : 1.0;
			s.ops       = h->d_ops;
			const int grid = int(std::min<size_t>((rows + 7) / 8, 148 * 16));
			k_scatter_crs<<<std::max(grid, 1), 256, 0, st>>>(s);
			if ((e = cudaGetLastError()))
				return fail_cuda(e, "CRS scatter launch");
		}
	return cudaStreamSynchronize(st) == cudaSuccess ? DMRGPP_OK
	                                                : handle_fail(h, DMRGPP_CUDA_ERROR, "CRS set-up");
}

} // namespace dmrgpp
