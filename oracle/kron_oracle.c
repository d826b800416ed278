/*
 * ORACLE -- test infrastructure only.  A plain-C, scalar restatement of the
 * reference's superblock H*psi for one symmetry sector, used by tests/ and by
 * the CPU-baseline leg of bench.py to check the CUDA path.  Nothing in the
 * product library links or calls this file.
 *
 * Conventions (GPU-plugin table, dmrg/GPUPlugin/BatchedGemm.h:11-56 and
 * dmrg/Engine/MatrixVectorKron/BatchedGemmPluginSc.h:69-113):
 *   table index t = i + j*np + k*np*np  (i = output patch, j = input patch)
 *   A[t]: column-major l_i x l_j block, leading dimension ldA[t] (or NULL)
 *   B[t]: column-major r_i x r_j block, leading dimension ldB[t] (or NULL)
 *   X, Y: concatenation of column-major r_p x l_p blocks at xy_start[p]
 *         (prefix sums of r_p*l_p, setup_sparse_batch.cpp:98-103)
 * A triple (i,j,k) contributes only if both blocks are present and each has
 * at least one nonzero entry (setup_nC.cpp:67-121).
 *
 * Y_i = sum_{j,k} B_k(i,j) * X_j * A_k(i,j)^T, evaluated per block with
 * "method 1" of the reference: BX = B*X_j, then Y_i += BX * A^T
 * (apply_Htarget_sparse_not_ready.cpp:197-285 pass 1 and :330-449 pass 2;
 * dmrg/KronUtil/den_kron_mult.cpp:75-180).  The plugin computes Y = H*X
 * (overwrite), as does this function.
 */
#include <stddef.h>
#include <stdlib.h>
#include <string.h>

static int block_is_nonzero(const double *m, size_t ld, size_t rows, size_t cols)
{
	if (!m)
		return 0;
	for (size_t c = 0; c < cols; ++c)
		for (size_t r = 0; r < rows; ++r)
			if (m[r + c * ld] != 0.0)
				return 1;
	return 0;
}

/* nC(i,j) and the per-triple "has work" flags (setup_nC.cpp:43-121). */
int oracle_kron_triples(size_t noperator, size_t npatches, const size_t *lsz,
                        const size_t *rsz, const double *const *A, const size_t *ldA,
                        const double *const *B, const size_t *ldB, unsigned char *has_work)
{
	const size_t np2 = npatches * npatches;
	int count = 0;
	for (size_t k = 0; k < noperator; ++k)
		for (size_t j = 0; j < npatches; ++j)
			for (size_t i = 0; i < npatches; ++i) {
				const size_t t = i + j * npatches + k * np2;
				const int w = block_is_nonzero(A[t], ldA[t], lsz[i], lsz[j]) &&
				              block_is_nonzero(B[t], ldB[t], rsz[i], rsz[j]);
				has_work[t] = (unsigned char)w;
				count += w;
			}
	return count;
}

/* F_alg: sum over contributing triples of 2*r_i*l_j*(r_j + l_i)
 * (cal_kron_flops.cpp:27-33 method 1, summed as estimate_work.cpp:114-151). */
double oracle_kron_flops(size_t noperator, size_t npatches, const size_t *lsz,
                         const size_t *rsz, const double *const *A, const size_t *ldA,
                         const double *const *B, const size_t *ldB)
{
	const size_t np2 = npatches * npatches;
	unsigned char *hw = (unsigned char *)malloc(np2 * noperator ? np2 * noperator : 1);
	oracle_kron_triples(noperator, npatches, lsz, rsz, A, ldA, B, ldB, hw);
	double f = 0.0;
	for (size_t k = 0; k < noperator; ++k)
		for (size_t j = 0; j < npatches; ++j)
			for (size_t i = 0; i < npatches; ++i)
				if (hw[i + j * npatches + k * np2])
					f += 2.0 * (double)rsz[i] * (double)lsz[j] *
					     ((double)rsz[j] + (double)lsz[i]);
	free(hw);
	return f;
}

/* y = H*x, both in patch order.  Returns 0 on success. */
int oracle_kron_apply(size_t noperator, size_t npatches, const size_t *lsz, const size_t *rsz,
                      const double *const *A, const size_t *ldA, const double *const *B,
                      const size_t *ldB, const double *x, double *y)
{
	const size_t np2 = npatches * npatches;
	size_t *start = (size_t *)malloc((npatches + 1) * sizeof(size_t));
	unsigned char *hw = (unsigned char *)malloc(np2 * noperator ? np2 * noperator : 1);
	size_t maxr = 1, maxl = 1;
	start[0] = 0;
	for (size_t p = 0; p < npatches; ++p) {
		start[p + 1] = start[p] + lsz[p] * rsz[p];
		if (rsz[p] > maxr)
			maxr = rsz[p];
		if (lsz[p] > maxl)
			maxl = lsz[p];
	}
	oracle_kron_triples(noperator, npatches, lsz, rsz, A, ldA, B, ldB, hw);
	double *bx = (double *)malloc(maxr * maxl * sizeof(double));
	memset(y, 0, start[npatches] * sizeof(double));

	for (size_t i = 0; i < npatches; ++i) {
		const size_t ri = rsz[i], li = lsz[i];
		double *yi = y + start[i];
		/* pass-2 column order of the plugin: j outer, k inner
		 * (setup_sparse_batch.cpp:289-343 packs A/B in that order). */
		for (size_t j = 0; j < npatches; ++j)
			for (size_t k = 0; k < noperator; ++k) {
				const size_t t = i + j * npatches + k * np2;
				if (!hw[t])
					continue;
				const size_t rj = rsz[j], lj = lsz[j];
				const double *xj = x + start[j];
				const double *b = B[t];
				const double *a = A[t];
				const size_t lb = ldB[t], la = ldA[t];
				/* BX (ri x lj) = B (ri x rj) * X_j (rj x lj) */
				for (size_t c = 0; c < lj; ++c)
					for (size_t r = 0; r < ri; ++r) {
						double s = 0.0;
						for (size_t q = 0; q < rj; ++q)
							s += b[r + q * lb] * xj[q + c * rj];
						bx[r + c * ri] = s;
					}
				/* Y_i (ri x li) += BX (ri x lj) * A^T (lj x li) */
				for (size_t c = 0; c < li; ++c)
					for (size_t r = 0; r < ri; ++r) {
						double s = 0.0;
						for (size_t q = 0; q < lj; ++q)
							s += bx[r + q * ri] * a[c + q * la];
						yi[r + c * ri] += s;
					}
			}
	}
	free(bx);
	free(hw);
	free(start);
	return 0;
}

/* Sector gather (InitKronHamiltonian.h:158-221, copyIn): for patch p with left
 * group g_L(p) and right group g_R(p),
 *   idx[vstart[p] + iR + iL*r_p] = permInverse[(iL+Loff) + (iR+Roff)*nL] - offset
 * so that yin[q] = vin[idx[q]] and the scatter (InitKronBase.h:315-360,
 * copyOut) is vout[idx[q]] = xout[q].  Returns the sector dimension. */
size_t oracle_gather_index(size_t npatches, const size_t *left_part, const size_t *right_part,
                           const size_t *patch_left, const size_t *patch_right, size_t nl,
                           const size_t *perm_inverse, size_t offset, long long *idx)
{
	size_t ip = 0;
	for (size_t p = 0; p < npatches; ++p) {
		const size_t gl = patch_left[p], gr = patch_right[p];
		const size_t loff = left_part[gl], roff = right_part[gr];
		const size_t sl = left_part[gl + 1] - loff, sr = right_part[gr + 1] - roff;
		for (size_t il = 0; il < sl; ++il)
			for (size_t ir = 0; ir < sr; ++ir)
				idx[ip + ir + il * sr] =
				    (long long)perm_inverse[(il + loff) + (ir + roff) * nl] - (long long)offset;
		ip += sl * sr;
	}
	return ip;
}
