// Oracle build only: the reference routes every dense GEMM through
// PsimagLite::kokkos_gemm (PsimagLite/src/PsimagLite/KokkosGemm.cpp:11-96,
// which needs KokkosKernels).  Without Kokkos, forward the double
// specialisation to the Fortran BLAS dgemm_ of the OpenBLAS shipped in the
// Python environment.  Kept in its own translation unit so the explicit
// specialisation is seen before any implicit instantiation.
#include <PsimagLite/KokkosGemm.h>

extern "C" void dgemm_(const char*, const char*, const int*, const int*, const int*,
                       const double*, const double*, const int*, const double*, const int*,
                       const double*, double*, const int*);

namespace PsimagLite {
template <>
void kokkos_gemm<double, int>(const Kokkos::DefaultExecutionSpace&,
                              char          ta,
                              char          tb,
                              int           m,
                              int           n,
                              int           k,
                              const double& alpha,
                              const double* A,
                              int           lda,
                              const double* B,
                              int           ldb,
                              const double& beta,
                              double*       C,
                              int           ldc)
{
	dgemm_(&ta, &tb, &m, &n, &k, &alpha, A, &lda, B, &ldb, &beta, C, &ldc);
}
} // namespace PsimagLite
