// BatchedGemm.h -- C++ drop-in for dmrg/GPUPlugin/BatchedGemm.h:11-56.
//
// Same class template name, same constructor arguments
// (noperator, npatches, left_patch_size, right_patch_size, Amatrix,
// ld_Amatrix, Bmatrix, ld_Bmatrix) and the same operation y = H x, backed by
// the B200 library through the C ABI of dmrgpp_kron.h.  Differences, all
// deliberate:
//   * apply_Htarget takes raw pointers (const T* vin, T* vout) instead of
//     Kokkos::View<..., SharedSpace>; the only caller,
//     BatchedGemmPluginSc::matrixVector (BatchedGemmPluginSc.h:139-161),
//     passes vin.data() / vout.data() (host memory) instead of building
//     SharedSpace mirrors.  A device-pointer overload is provided for callers
//     that keep vectors resident on the GPU.
//   * errors throw std::runtime_error carrying the library's message instead
//     of assert/printf (dmrg_malloc_cuda.cpp:24-29).
//   * T = double and T = std::complex<double>, the two instantiations of the
//     reference (BatchedGemm.cpp:117-119); complex handles come from
//     dmrgpp_kron_create_complex (the real embedding of the complex sector).
#ifndef DMRGPP_B200_BATCHEDGEMM_H
#define DMRGPP_B200_BATCHEDGEMM_H

#include "dmrgpp_kron.h"

#include <complex>
#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

template <typename T> class BatchedGemm {

	static_assert(std::is_same<T, double>::value || std::is_same<T, std::complex<double>>::value,
	              "the B200 library implements BatchedGemm<double> and BatchedGemm<std::complex<double>>");
	static constexpr bool kComplex = std::is_same<T, std::complex<double>>::value;

public:

	// PsimagLite's SizeType (AllocatorCpu.h:43-47): 32-bit with USE_SHORT, so
	// that the caller's VectorSizeType& arguments bind either way
#ifdef USE_SHORT
	using SizeType = std::uint32_t;
#else
	using SizeType = long unsigned int;
#endif
	using VectorSizeType = std::vector<SizeType>;

	BatchedGemm(SizeType         noperator,
	            SizeType         npatches,
	            VectorSizeType&  left_patch_size,
	            VectorSizeType&  right_patch_size,
	            std::vector<T*>& Amatrix,
	            VectorSizeType&  ld_Amatrix,
	            std::vector<T*>& Bmatrix,
	            VectorSizeType&  ld_Bmatrix,
	            int              precision = DMRGPP_FP64,
	            void*            stream    = nullptr)
	    : handle_(nullptr)
	    , dim_(0)
	{
		// the C ABI takes size_t arrays
		const std::vector<std::size_t> l(left_patch_size.begin(), left_patch_size.end());
		const std::vector<std::size_t> r(right_patch_size.begin(), right_patch_size.end());
		const std::vector<std::size_t> lda(ld_Amatrix.begin(), ld_Amatrix.end());
		const std::vector<std::size_t> ldb(ld_Bmatrix.begin(), ld_Bmatrix.end());
		dmrgpp_kron_desc               d {};
		d.noperator        = noperator;
		d.npatches         = npatches;
		d.left_patch_size  = l.data();
		d.right_patch_size = r.data();
		// std::complex<double> is two doubles (real, imaginary)
		d.Amatrix          = reinterpret_cast<const double* const*>(Amatrix.data());
		d.ld_Amatrix       = lda.data();
		d.Bmatrix          = reinterpret_cast<const double* const*>(Bmatrix.data());
		d.ld_Bmatrix       = ldb.data();
		d.precision        = precision;
		d.stream           = stream;
		d.device           = -1;
		check(kComplex ? dmrgpp_kron_create_complex(&d, &handle_) : dmrgpp_kron_create(&d, &handle_),
		      nullptr);
		std::size_t dim = 0;
		check(dmrgpp_kron_dim(handle_, &dim), handle_);
		dim_ = SizeType(dim);
	}

	// vout = H vin, both host vectors in patch order (BatchedGemm.cpp:81-115).
	void apply_Htarget(const T* vin, T* vout) const
	{
		check(dmrgpp_kron_apply(handle_, reinterpret_cast<const double*>(vin),
		                        reinterpret_cast<double*>(vout), 0),
		      handle_);
	}

	// vout = H vin with device-resident vectors; enqueued on the handle's stream.
	void apply_Htarget_device(const T* vin_dev, T* vout_dev) const
	{
		check(dmrgpp_kron_apply(handle_, reinterpret_cast<const double*>(vin_dev),
		                        reinterpret_cast<double*>(vout_dev), 1),
		      handle_);
	}

	SizeType size() const { return dim_; }

	double flops() const
	{
		double f = 0;
		check(dmrgpp_kron_flops(handle_, &f), handle_);
		return f;
	}

	~BatchedGemm() { dmrgpp_kron_destroy(handle_); }

	BatchedGemm(const BatchedGemm&)            = delete;
	BatchedGemm& operator=(const BatchedGemm&) = delete;

private:

	static void check(int status, dmrgpp_kron_handle h)
	{
		if (status != DMRGPP_OK)
			throw std::runtime_error(std::string("dmrgpp-b200: ")
			                         + dmrgpp_kron_last_error(h));
	}

	dmrgpp_kron_handle handle_;
	SizeType           dim_;
};

#endif // DMRGPP_B200_BATCHEDGEMM_H
