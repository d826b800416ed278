// dmrgpp_kron_gather_index: the sector gather index of the reference's
// copyIn / copyOut, built once per sector solve on the host cores.
//
// InitKronHamiltonian::copyIn (dmrg/Engine/MatrixVectorKron/
// InitKronHamiltonian.h:158-221) and InitKronBase::copyOut (InitKronBase.h:
// 315-360) move a sector vector between the superblock basis order and the
// patch order of the Kronecker product on every matvec:
//     yin[vstart[p] + iR + iL * r_p] = vin[permInverse[(iL + Loff) + (iR + Roff) * nl] - offset]
// for patch p with left group g_L(p) (states Loff .. Loff + l_p - 1 of the
// left block) and right group g_R(p).  Here that map is computed once into an
// index array; dmrgpp_gather / dmrgpp_scatter then apply it on the device
// (idx[q] = position in the superblock sector of patch-order element q).
#include "dmrgpp_kron.h"
#include "handle.h"
#include "kron_plan.h"

#include <cstdint>
#include <map>
#include <string>
#include <vector>

extern "C" int dmrgpp_kron_gather_index(const dmrgpp_gather_index_desc* d, int64_t* idx)
{
	using dmrgpp::handle_fail;
	if (!d || !idx)
		return handle_fail(nullptr, DMRGPP_INVALID_ARG, "null descriptor or index array");
	if ((d->npatches && (!d->patch_left || !d->patch_right)) || !d->left_partition
	    || !d->right_partition || !d->perm_inverse)
		return handle_fail(nullptr, DMRGPP_INVALID_ARG, "null array in the gather-index descriptor");
	const size_t* lp = d->left_partition;
	const size_t* rp = d->right_partition;
	for (size_t g = 0; g < d->left_groups; ++g)
		if (lp[g + 1] < lp[g])
			return handle_fail(nullptr, DMRGPP_INVALID_ARG, "left partition decreases at group " + std::to_string(g));
	for (size_t g = 0; g < d->right_groups; ++g)
		if (rp[g + 1] < rp[g])
			return handle_fail(nullptr, DMRGPP_INVALID_ARG, "right partition decreases at group " + std::to_string(g));
	const size_t nl = lp[d->left_groups];
	// vstart: prefix sums of l_p r_p (InitKronBase::setUpVstart, InitKronBase.h:277-310)
	std::vector<size_t> vstart(d->npatches + 1, 0);
	for (size_t p = 0; p < d->npatches; ++p) {
		if (d->patch_left[p] >= d->left_groups || d->patch_right[p] >= d->right_groups)
			return handle_fail(nullptr, DMRGPP_INVALID_ARG, "patch " + std::to_string(p) + " names a group out of range");
		const size_t gl = d->patch_left[p], gr = d->patch_right[p];
		vstart[p + 1] = vstart[p] + (lp[gl + 1] - lp[gl]) * (rp[gr + 1] - rp[gr]);
	}
	if (vstart[d->npatches] != d->sector_size)
		return handle_fail(nullptr, DMRGPP_INVALID_ARG,
		                   "patches hold " + std::to_string(vstart[d->npatches]) + " states, the sector "
		                       + std::to_string(d->sector_size));
	const size_t nperm = nl * rp[d->right_groups];
	std::vector<char> bad(d->npatches, 0);
	dmrgpp::parallel_for(d->npatches, [&](size_t p) {
		const size_t gl = d->patch_left[p], gr = d->patch_right[p];
		const size_t loff = lp[gl], roff = rp[gr];
		const size_t sl = lp[gl + 1] - loff, sr = rp[gr + 1] - roff;
		int64_t*     out = idx + vstart[p];
		for (size_t il = 0; il < sl; ++il)
			for (size_t ir = 0; ir < sr; ++ir) {
				const size_t g = (il + loff) + (ir + roff) * nl;
				const size_t r = g < nperm ? d->perm_inverse[g] : ~size_t(0);
				// the reference asserts offset <= r < offset + size
				if (g >= nperm || r < d->offset || r - d->offset >= d->sector_size) {
					bad[p] = 1;
					return;
				}
				out[ir + il * sr] = int64_t(r - d->offset);
			}
	});
	for (size_t p = 0; p < d->npatches; ++p)
		if (bad[p])
			return handle_fail(nullptr, DMRGPP_INVALID_ARG,
			                   "patch " + std::to_string(p)
			                       + " maps a state outside the sector (permutationInverse, offset)");
	// a permutation of the sector: the device scatter writes every position once
	std::vector<unsigned char> seen(d->sector_size, 0);
	for (size_t q = 0; q < d->sector_size; ++q) {
		if (seen[size_t(idx[q])])
			return handle_fail(nullptr, DMRGPP_INVALID_ARG,
			                   "two patch-order elements map to sector position " + std::to_string(idx[q]));
		seen[size_t(idx[q])] = 1;
	}
	return DMRGPP_OK;
}

// GenIjPatch::GenIjPatch (dmrg/Engine/MatrixVectorKron/GenIjPatch.h:104-118):
// every (left group i, right group j), i outer and j inner, whose quantum
// numbers combine to the target.  The quantum numbers are additive vectors
// of qn_len integers per group (Sz, particle numbers, ...); the right groups
// are indexed by quantum number, so the search is linear in the groups.
extern "C" int dmrgpp_kron_patch_list(size_t left_groups, const int64_t* left_qn, size_t right_groups,
                                      const int64_t* right_qn, size_t qn_len, const int64_t* target,
                                      size_t capacity, size_t* patch_left, size_t* patch_right,
                                      size_t* npatches)
{
	using dmrgpp::handle_fail;
	if (!npatches || (left_groups && !left_qn) || (right_groups && !right_qn) || (qn_len && !target)
	    || (capacity && (!patch_left || !patch_right)))
		return handle_fail(nullptr, DMRGPP_INVALID_ARG, "null array in the patch-list arguments");
	std::map<std::vector<int64_t>, std::vector<size_t>> by_qn;
	for (size_t j = 0; j < right_groups; ++j)
		by_qn[std::vector<int64_t>(right_qn + j * qn_len, right_qn + (j + 1) * qn_len)].push_back(j);
	size_t              n = 0;
	std::vector<int64_t> need(qn_len);
	for (size_t i = 0; i < left_groups; ++i) {
		for (size_t c = 0; c < qn_len; ++c)
			need[c] = target[c] - left_qn[i * qn_len + c];
		auto f = by_qn.find(need);
		if (f == by_qn.end())
			continue;
		for (size_t j : f->second) {
			if (n < capacity) {
				patch_left[n]  = i;
				patch_right[n] = j;
			}
			++n;
		}
	}
	*npatches = n;
	if (n > capacity)
		return handle_fail(nullptr, DMRGPP_INVALID_ARG,
		                   "the sector has " + std::to_string(n) + " patches, more than the capacity "
		                       + std::to_string(capacity));
	return DMRGPP_OK;
}
