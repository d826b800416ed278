// Oracle harness (test infrastructure, never shipped): compiles the
// reference's own CPU hot-path code from its source tree and exposes it
// through a small C ABI so that tests and the CPU baseline can call it.
//
//   * Dmrg::BatchedGemmCpu<...>::matrixVector  -- the "BLAS batched path"
//     (dmrg/Engine/MatrixVectorKron/BatchedGemmCpu.h:33-301)
//   * PsimagLite::LanczosSolver<...>::computeAllStatesBelow
//     (PsimagLite/src/PsimagLite/LanczosSolver.h:68-88, LanczosCore.h:147-272)
//
// The InitKron object that BatchedGemmCpu expects is replaced by a small
// table-backed stand-in (the same technique as the reference's own unit test,
// dmrg/Engine/tests/test_BatchedGemm.cpp:18-169): left group p and right group
// p are patch p, partitions are prefix sums of the patch sizes, and
// xc(k)(i,j) / yc(k)(i,j) return the dense blocks A_k(i,j) / B_k(i,j) of the
// plugin table (Amatrix[i + j*np + k*np*np], BatchedGemmPluginSc.h:95-101).
#include <PsimagLite/CrsMatrix.h>

#include "BatchedGemmCpu.h"
#include <PsimagLite/LanczosSolver.h>

#include <cstddef>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

namespace {

using SizeT = unsigned long;

struct HarnessParams {
	struct Opt {
		bool isSet(const std::string& s) const { return s == "BatchedGemm"; }
	} options;
};

struct HarnessBasis {
	std::vector<int> parts; // group partition points, size groups+1
	int              partition(SizeT g) const { return parts[g]; }
	int              size() const { return parts.back(); }
};

struct HarnessLrs {
	HarnessBasis        l, r;
	const HarnessBasis& left() const { return l; }
	const HarnessBasis& right() const { return r; }
};

struct HarnessBlock {
	using value_type = double;
	using VectorType = PsimagLite::Vector<double>::Type;
	using MatrixType = PsimagLite::Matrix<double>;
	MatrixType        mat;
	bool              isDense() const { return true; }
	const MatrixType& dense() const { return mat; }
	int               rows() const { return mat.rows(); }
	int               cols() const { return mat.cols(); }
};

struct HarnessArrayOfMat {
	using MatrixDenseOrSparseType = HarnessBlock;
	SizeT                                      np = 0;
	std::vector<std::unique_ptr<HarnessBlock>> blocks; // [i + j*np]
	const HarnessBlock* operator()(SizeT i, SizeT j) const { return blocks[i + j * np].get(); }
};

struct HarnessGenIjPatch {
	enum LeftOrRightEnumType
	{
		LEFT  = 0,
		RIGHT = 1
	};
	using BasisType = int;
};

struct HarnessInitKron {
	enum WhatBasisEnum
	{
		OLD = 0,
		NEW = 1
	};
	using ArrayOfMatStructType = HarnessArrayOfMat;
	using GenIjPatchType       = HarnessGenIjPatch;

	HarnessParams                  p;
	HarnessLrs                     lrs_;
	std::vector<SizeT>             patchIdx;
	std::vector<SizeT>             offsets; // np+1
	std::vector<HarnessArrayOfMat> xc_, yc_;
	SizeT                          np_ = 0, nop_ = 0;

	const HarnessParams&      params() const { return p; }
	SizeT                     numberOfPatches(int) const { return np_; }
	SizeT                     connections() const { return nop_; }
	const std::vector<SizeT>& patch(WhatBasisEnum, HarnessGenIjPatch::LeftOrRightEnumType) const
	{
		return patchIdx;
	}
	const HarnessLrs&        lrs(WhatBasisEnum) const { return lrs_; }
	SizeT                    offsetForPatches(WhatBasisEnum, SizeT p) const { return offsets[p]; }
	const HarnessArrayOfMat& xc(SizeT k) const { return xc_[k]; }
	const HarnessArrayOfMat& yc(SizeT k) const { return yc_[k]; }
};

struct RefKron {
	HarnessInitKron                                    ik;
	std::unique_ptr<Dmrg::BatchedGemmCpu<HarnessInitKron>> bg;
	SizeT                                              dim = 0;
};

// Dense copy of one column-major block; nullptr source means "absent".
std::unique_ptr<HarnessBlock>
copyBlock(const double* src, SizeT ld, SizeT rows, SizeT cols)
{
	if (!src)
		return nullptr;
	auto b = std::make_unique<HarnessBlock>();
	b->mat.resize(rows, cols);
	for (SizeT c = 0; c < cols; ++c)
		for (SizeT r = 0; r < rows; ++r)
			b->mat(r, c) = src[r + c * ld];
	return b;
}

// Lanczos matrix adaptor: PsimagLite wants x += H*y (LanczosCore.h:93-98).
typedef void (*ref_matvec_fn)(void* ctx, const double* y, double* hy);

struct CallbackMatrix {
	using value_type = double;
	SizeT               n;
	ref_matvec_fn       fn;
	void*               ctx;
	mutable std::vector<double> tmp;
	SizeT               rows() const { return n; }
	void matrixVectorProduct(std::vector<double>& x, const std::vector<double>& y) const
	{
		tmp.assign(n, 0.0);
		fn(ctx, y.data(), tmp.data());
		for (SizeT i = 0; i < n; ++i)
			x[i] += tmp[i];
	}
};

} // namespace

extern "C" {

// Builds the reference BatchedGemmCpu for one sector.  Tables follow the
// GPU-plugin convention: entry i + j*np + k*np*np is the column-major block
// A_k(i,j) (l_i x l_j, leading dimension ldA[...]) or nullptr.
void* ref_kron_create(SizeT               noperator,
                      SizeT               npatches,
                      const SizeT*        left_size,
                      const SizeT*        right_size,
                      const double* const* Amatrix,
                      const SizeT*        ldA,
                      const double* const* Bmatrix,
                      const SizeT*        ldB)
{
	auto* rk      = new RefKron();
	auto& ik      = rk->ik;
	ik.np_        = npatches;
	ik.nop_       = noperator;
	ik.lrs_.l.parts = { 0 };
	ik.lrs_.r.parts = { 0 };
	ik.patchIdx.resize(npatches);
	ik.offsets.assign(npatches + 1, 0);
	for (SizeT p = 0; p < npatches; ++p) {
		ik.lrs_.l.parts.push_back(ik.lrs_.l.parts.back() + int(left_size[p]));
		ik.lrs_.r.parts.push_back(ik.lrs_.r.parts.back() + int(right_size[p]));
		ik.patchIdx[p]     = p;
		ik.offsets[p + 1] = ik.offsets[p] + left_size[p] * right_size[p];
	}
	rk->dim = ik.offsets[npatches];
	ik.xc_.resize(noperator);
	ik.yc_.resize(noperator);
	const SizeT np2 = npatches * npatches;
	for (SizeT k = 0; k < noperator; ++k) {
		ik.xc_[k].np = npatches;
		ik.yc_[k].np = npatches;
		ik.xc_[k].blocks.resize(np2);
		ik.yc_[k].blocks.resize(np2);
		for (SizeT j = 0; j < npatches; ++j)
			for (SizeT i = 0; i < npatches; ++i) {
				const SizeT t = i + j * npatches + k * np2;
				if (!Amatrix[t] || !Bmatrix[t])
					continue;
				ik.xc_[k].blocks[i + j * npatches]
				    = copyBlock(Amatrix[t], ldA[t], left_size[i], left_size[j]);
				ik.yc_[k].blocks[i + j * npatches]
				    = copyBlock(Bmatrix[t], ldB[t], right_size[i], right_size[j]);
			}
	}
	rk->bg = std::make_unique<Dmrg::BatchedGemmCpu<HarnessInitKron>>(ik);
	return rk;
}

// y = H*x in patch order (BatchedGemmCpu overwrites vout, BatchedGemmCpu.h:253-300).
void ref_kron_apply(void* h, const double* x, double* y)
{
	auto*               rk = static_cast<RefKron*>(h);
	std::vector<double> vin(x, x + rk->dim), vout(rk->dim, 0.0);
	rk->bg->matrixVector(vout, vin);
	std::memcpy(y, vout.data(), rk->dim * sizeof(double));
}

SizeT ref_kron_dim(void* h) { return static_cast<RefKron*>(h)->dim; }

void ref_kron_destroy(void* h) { delete static_cast<RefKron*>(h); }

// Adapter so a RefKron handle can drive the reference Lanczos solver.
void ref_kron_matvec_cb(void* h, const double* y, double* hy) { ref_kron_apply(h, y, hy); }

// Lowest eigenpair through PsimagLite::LanczosSolver::computeAllStatesBelow
// with lotaMemory and optional full reorthogonalisation ("reortho").
// Returns the number of Lanczos steps taken.
SizeT ref_lanczos(SizeT         n,
                  ref_matvec_fn fn,
                  void*         ctx,
                  const double* init,
                  SizeT         steps,
                  SizeT         min_steps,
                  double        tolerance,
                  int           reortho,
                  double*       energy,
                  double*       z)
{
	CallbackMatrix                          H { n, fn, ctx, {} };
	PsimagLite::ParametersForSolver<double> p;
	p.lotaMemory = true;
	p.tolerance  = tolerance;
	p.steps      = steps;
	p.minSteps   = min_steps;
	p.options    = reortho ? "reortho" : "";
	PsimagLite::LanczosSolver<CallbackMatrix> ls(H, p);
	std::vector<double>              iv(init, init + n);
	std::vector<double>              eigs;
	std::vector<std::vector<double>> zz(1, std::vector<double>(n, 0.0));
	// excited=1: the stop test then watches the lowest Ritz value
	// (LanczosCore.h:222-240 uses min(excited, size) eigenvalues); with 0
	// it would stop unconditionally after MinSteps.
	ls.computeAllStatesBelow(eigs, zz, iv, 1);
	*energy = eigs[0];
	std::memcpy(z, zz[0].data(), n * sizeof(double));
	return ls.steps();
}

} // extern "C"
