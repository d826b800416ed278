/*
 * dmrgpp_kron.h -- C ABI of the B200 superblock Hamiltonian-times-vector
 * engine for DMRG++.
 *
 * It replaces the GPU plugin behind DMRG_BATCHED_GEMM_TYPE=Plugin
 * (dmrg/GPUPlugin/BatchedGemm.h:11-56, selected by
 * dmrg/Engine/MatrixVectorKron/BatchedGemmInclude.hh:7-9 and driven by
 * dmrg/Engine/MatrixVectorKron/BatchedGemmPluginSc.h:40-189).
 *
 * One handle holds one symmetry sector of the superblock:
 *   npatches patches; patch p pairs a left group of l_p states with a right
 *   group of r_p states.  The sector vector is the concatenation, in patch
 *   order, of column-major r_p x l_p blocks X_p.
 *   noperator Kronecker terms; term k has blocks A_k(i,j) (l_i x l_j) and
 *   B_k(i,j) (r_i x r_j), column-major.
 *   y = H x  means  Y_i = sum_{j,k} B_k(i,j) X_j A_k(i,j)^T.
 *
 * Table convention (identical to the plugin's, BatchedGemmPluginSc.h:95-113):
 *   Amatrix[i + j*npatches + k*npatches*npatches] points to A_k(i,j) with
 *   leading dimension ld_Amatrix[same index]; NULL (or an all-zero block)
 *   means the term does not couple patch j to patch i (setup_nC.cpp:67-121).
 *   Bmatrix / ld_Bmatrix likewise.  The caller's blocks are read during
 *   dmrgpp_kron_create only; the handle keeps its own packed device copy.
 *
 * Errors: every entry point returns a dmrgpp_status.  The reference reports
 * errors with assert/printf and C++ exceptions; a C++ caller converts a
 * non-OK status into its own exception (include/BatchedGemm.h does).
 * dmrgpp_kron_last_error() gives a human-readable reason.
 *
 * Threading: a handle is used by one host thread at a time; distinct handles
 * may run concurrently on distinct streams.
 */
#ifndef DMRGPP_KRON_H
#define DMRGPP_KRON_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
	DMRGPP_OK            = 0,
	DMRGPP_INVALID_ARG   = 1,
	DMRGPP_OOM           = 2,
	DMRGPP_CUDA_ERROR    = 3,
	DMRGPP_TIMEOUT       = 4,
	DMRGPP_NOT_SUPPORTED = 5,
	DMRGPP_NOT_CONVERGED = 6
} dmrgpp_status;

/* Arithmetic of the Kronecker GEMMs.  FP64 is the plain method. */
typedef enum {
	DMRGPP_FP64       = 0,
	DMRGPP_SPLIT_BF16 = 1,
	DMRGPP_TF32X3     = 2
} dmrgpp_precision;

typedef struct dmrgpp_kron_s* dmrgpp_kron_handle;

/* Mirrors the constructor arguments of BatchedGemm<T>
 * (dmrg/GPUPlugin/BatchedGemm.h:22-29): noperator, npatches,
 * left_patch_size, right_patch_size, Amatrix, ld_Amatrix, Bmatrix,
 * ld_Bmatrix; plus the arithmetic mode, the CUDA stream on which every
 * operation of the handle is enqueued (cudaStream_t; NULL is the default
 * stream) and the device (-1: current). */
typedef struct {
	size_t               noperator;
	size_t               npatches;
	const size_t*        left_patch_size;
	const size_t*        right_patch_size;
	const double* const* Amatrix;
	const size_t*        ld_Amatrix;
	const double* const* Bmatrix;
	const size_t*        ld_Bmatrix;
	int                  precision;
	void*                stream;
	int                  device;
} dmrgpp_kron_desc;

/* Replaces BatchedGemm<T>::BatchedGemm (dmrg/GPUPlugin/BatchedGemm.cpp:8-69,
 * which calls setup_sparse_batch, setup_sparse_batch.cpp:14-379): validates
 * the tables, finds the contributing (i,j,k) triples, packs the operators on
 * the device and builds the launch schedule. */
int dmrgpp_kron_create(const dmrgpp_kron_desc* desc, dmrgpp_kron_handle* out);

/* ---- Building the block tables on the device from the CRS operators ----
 * The reference's InitKron set-up: each connection's left operator A and
 * right operator B are CRS matrices over the left and right block bases
 * (PsimagLite::CrsMatrix, 0-based rowptr / colind / values);
 * InitKronBase::calculateAhat (InitKronBase.h:393-413) forms
 * Ahat(a,:) = A(a,:) * sign * value with sign = -1 for a fermionic term on a
 * left state of odd parity, and ArrayOfMatStruct (ArrayOfMatStruct.h:105-448)
 * slices Ahat and B into the per-patch blocks A_k(i,j) (rows of patch i's
 * left group, columns of patch j's) and B_k(i,j) (right groups), which the
 * batched path densifies (BatchedGemmKokkos.h:354-370).  Here the CRS arrays
 * go to the device as they are and a scatter kernel writes every entry into
 * the handle's packed blocks; only the block-presence scan (which blocks hold
 * a nonzero) runs on the host.  The handle is the one dmrgpp_kron_create
 * builds from the same blocks as dense tables, bit for bit. */
typedef struct {
	size_t        rows;   /* square operator: rows x rows */
	const int*    rowptr; /* rows + 1, rowptr[0] = 0 */
	const int*    colind; /* rowptr[rows] entries, each in [0, rows), no repeats within a row */
	const double* values;
} dmrgpp_crs;

typedef struct {
	size_t               noperator;        /* Kronecker terms k */
	size_t               npatches;
	const size_t*        left_offset;      /* per patch: first state of its left group in the left basis */
	const size_t*        left_patch_size;
	const size_t*        right_offset;     /* per patch: first state of its right group */
	const size_t*        right_patch_size;
	const dmrgpp_crs*    A;                /* noperator left-basis operators (all the same rows) */
	const dmrgpp_crs*    B;                /* noperator right-basis operators */
	const double*        value;            /* per term: the factor on A (NULL: 1) */
	const int*           fermion;          /* per term: 1 = sign by the left state's parity (NULL: none) */
	const unsigned char* left_parity;      /* per left state: 1 = odd (needed when a term is fermionic) */
	int                  precision;
	void*                stream;
	int                  device;
} dmrgpp_kron_crs_desc;

/* The patches' left groups (and right groups) must not overlap. */
int dmrgpp_kron_create_crs(const dmrgpp_kron_crs_desc* desc, dmrgpp_kron_handle* out);

/* Many independent sectors in one handle (no counterpart in the reference,
 * whose plugin holds one sector): sector s keeps its own tables (descs[s],
 * all with the same precision, device and stream), its patches follow those
 * of sectors 0..s-1, and no block connects two sectors, so the group's H is
 * block-diagonal.  One dmrgpp_kron_apply then applies every sector in one
 * persistent launch to the concatenated vector x = [x_0; x_1; ...]; the
 * eigensolvers treat the group as one sector, dmrgpp_lanczos_lowest_group
 * solves every sector separately. */
int dmrgpp_kron_create_group(const dmrgpp_kron_desc* descs, size_t nsectors,
                             dmrgpp_kron_handle* out);

/* Number of sectors of a handle (1 unless made by dmrgpp_kron_create_group)
 * and, if offsets is not NULL, their nsectors + 1 start offsets in x. */
int dmrgpp_kron_group_sectors(dmrgpp_kron_handle h, size_t* nsectors, long long* offsets);

/* Replaces BatchedGemm<T>::~BatchedGemm (dmrg/GPUPlugin/BatchedGemm.cpp:72-79). */
int dmrgpp_kron_destroy(dmrgpp_kron_handle h);

/* Replaces BatchedGemm<T>::apply_Htarget (dmrg/GPUPlugin/BatchedGemm.cpp:81-115,
 * apply_Htarget_sparse_not_ready.cpp:14-478): y = H x (overwrite) in patch
 * order.  on_device = 0: x and y are host pointers (copied in and out on the
 * handle's stream; the call returns when y is written).  on_device = 1: x
 * and y are device pointers; the call only enqueues work on the stream. */
int dmrgpp_kron_apply(dmrgpp_kron_handle h, const double* x, double* y, int on_device);

/* Switches the arithmetic of later applies (and of the eigensolvers) between
 * DMRGPP_FP64 and the mixed mode the handle was created with; FP64 is always
 * available.  No counterpart in the reference. */
int dmrgpp_kron_set_precision(dmrgpp_kron_handle h, int precision);

/* The precision that H*x launches of the handle currently use (DMRGPP_FP64
 * or the mixed mode it was created with). */
int dmrgpp_kron_get_precision(dmrgpp_kron_handle h, int* precision);

/* Waits for the handle's stream and reports errors of work enqueued by
 * device-pointer applies (DMRGPP_TIMEOUT if a dependency wait inside the
 * kernel gave up, DMRGPP_CUDA_ERROR for a CUDA failure).  No counterpart in
 * the reference, whose apply is synchronous. */
int dmrgpp_kron_synchronize(dmrgpp_kron_handle h);

/* Test hook (no counterpart in the reference): with on != 0 every following
 * apply makes a bounded wait inside the kernels unsatisfiable -- FP64: the
 * dependency waits on input patch 0 (time limit about 0.2 s); TF32x3: the
 * first pipeline stage of one CTA of pass 1 is never filled, so the MMA
 * thread's mbarrier wait runs out (about 0.5 s), the CTA drains its copies,
 * frees its tensor memory and exits.  The apply then reports DMRGPP_TIMEOUT
 * and the handle stays usable.  Used to test failure detection without
 * faulting the GPU. */
int dmrgpp_kron_test_stall_dependency(dmrgpp_kron_handle h, int on);

/* The diagonal of the sector's H (patch order) into diag (device pointer). */
int dmrgpp_kron_diagonal(dmrgpp_kron_handle h, double* diag);

/* Sector dimension D = sum_p l_p r_p (xy_patch_start, setup_sparse_batch.cpp:98-103). */
int dmrgpp_kron_dim(dmrgpp_kron_handle h, size_t* dim);

/* Complex sectors (the reference's BatchedGemm<std::complex<double>>,
 * BatchedGemm.cpp:117-119): the descriptor's blocks are std::complex<double>
 * (interleaved real and imaginary parts, passed as const double*), column-
 * major with leading dimensions in complex elements.  dmrgpp_kron_apply then
 * takes interleaved complex x and y of dmrgpp_kron_dim(h) complex entries
 * (y = H x, H = sum_k A_k (x) B_k without conjugation).  The handle runs the
 * real embedding: patches of Re x and of Im x, and for every complex term the
 * real terms Ar(x)Br, -Ai(x)Bi (diagonal quadrants), Ar(x)Bi, Ai(x)Br
 * (Im from Re) and -Ar(x)Bi, -Ai(x)Br (Re from Im), so dmrgpp_kron_flops
 * reports the real flops executed.  The device eigensolvers return
 * DMRGPP_NOT_SUPPORTED on complex handles. */
int dmrgpp_kron_create_complex(const dmrgpp_kron_desc* desc, dmrgpp_kron_handle* out);
int dmrgpp_kron_is_complex(dmrgpp_kron_handle h, int* is_complex);

/* Algorithmic flops of one apply: sum over contributing triples of
 * 2 r_i l_j (r_j + l_i) (dmrg/GPUPlugin/cal_kron_flops.cpp:27-33 method 1,
 * summed as estimate_work.cpp:114-151). */
int dmrgpp_kron_flops(dmrgpp_kron_handle h, double* f_alg);

/* Wall-clock seconds of the phases of this handle's create (host clock,
 * each phase waits for its device work): the plugin constructor's work
 * (BatchedGemm.cpp:8-79, setup_sparse_batch.cpp:14-379) split into
 *   PLAN         all-zero block scan, triple list, offsets, tile lists
 *   ALLOC        device allocations and the persistent schedule
 *   UPLOAD       the staged copy of the blocks into the packed operators
 *   UPLOAD_FILL  of which host time copying blocks into pinned staging
 *   DIAGONAL     the diagonal of H (preconditioners)
 *   MIXED        the TF32x3 form (0 for FP64 handles)
 *   TOTAL        the whole create
 * n (<= DMRGPP_SETUP_NPHASES) values are written to t. */
enum {
	DMRGPP_SETUP_PLAN        = 0,
	DMRGPP_SETUP_ALLOC       = 1,
	DMRGPP_SETUP_UPLOAD      = 2,
	DMRGPP_SETUP_UPLOAD_FILL = 3,
	DMRGPP_SETUP_DIAGONAL    = 4,
	DMRGPP_SETUP_MIXED       = 5,
	DMRGPP_SETUP_TOTAL       = 6,
	DMRGPP_SETUP_NPHASES     = 7
};
int dmrgpp_kron_setup_profile(dmrgpp_kron_handle h, double* t, size_t n);

/* Device memory of handles and solver workspaces comes from one
 * stream-ordered pool per device that keeps freed memory for the next handle
 * (a sweep destroys and creates a handle of similar size every step); freed
 * blocks of 64 MB and more also stay on a free list by size for the next
 * request of about their size.  dmrgpp_release_cached_memory returns the
 * unused part to the device (device < 0: the current device);
 * dmrgpp_cached_memory reports the pool's reserved bytes and the bytes in
 * use (free-listed blocks not counted). */
int dmrgpp_release_cached_memory(int device);
int dmrgpp_cached_memory(int device, size_t* reserved_bytes, size_t* used_bytes);

/* Host-only planning statistics (no device work; usable without a GPU):
 * number of contributing triples, F_alg, packed operator bytes and the
 * bytes of the intermediate BX buffer. */
typedef struct {
	size_t ntriples;
	size_t dim;
	double f_alg;
	size_t operator_bytes;
	size_t bx_bytes;
	size_t pass1_tiles;
	size_t pass2_tiles;
} dmrgpp_kron_plan_info;

int dmrgpp_kron_plan_info_get(const dmrgpp_kron_desc* desc, dmrgpp_kron_plan_info* info);

/* No counterpart in the reference.  One-shot y = H x that performs no device
 * memory allocation, for callers that cannot call cudaMalloc (for example
 * code running while another component owns all device memory through its
 * own allocator, or a runtime that forbids allocation after start-up).
 * desc is read as by dmrgpp_kron_create (host tables, FP64 only); x and y
 * are device pointers of the sector dimension; the work is enqueued on
 * desc->stream and the call returns without waiting for it.
 * All scratch (packed operators, the pass-1 buffer, launch lists) lives in
 * one file-scope device array of DMRGPP_NOALLOC_SCRATCH_BYTES that every GPU
 * which loads the library holds until the process exits; a sector needing
 * more is rejected with DMRGPP_INVALID_ARG.  The first call on a device looks
 * up the array's device address (cudaGetSymbolAddress) and sets kernel
 * attributes, so make that first call before any stream capture.  A call
 * made on a stream that is being captured returns DMRGPP_NOT_SUPPORTED: its
 * uploads read host memory that the call frees before returning.  Every call
 * shares the one array: calls that may overlap on the GPU (other streams,
 * other host threads) race and must be serialised by the caller.  Each call
 * rewrites every scratch byte it reads, so no clearing is needed between
 * calls.  Errors: dmrgpp_kron_noalloc_last_error(). */
#define DMRGPP_NOALLOC_SCRATCH_BYTES ((size_t)16 << 20)
int dmrgpp_kron_apply_noalloc(const dmrgpp_kron_desc* desc, const double* x, double* y);
const char* dmrgpp_kron_noalloc_last_error(void);

/* ---- Launch tuning (no counterpart in the reference, whose GPU tiling is a
 * set of fixed constants, BatchedGemmKokkos.h:110-130) ----
 * Tile configurations of the H*x kernel.  Two-pass persistent form:
 * 0: 32x32 tiles, k-chunk 16; 1: 32x32, k32; 2: 64x64, k16; 3: 64x64, k32;
 * 4: 32x32, k32, deeper pipeline; 5: 32x32, k64; items_per_cta: pass-2
 * work items per resident CTA below which output tiles are split along K.
 * Fused form (both passes of an output tile in one CTA, parts of a tile
 * summed inside a thread-block cluster; for sectors of small patches):
 * 6: 32x128 output tiles, 64-column units, clusters of 8; 7: the same with
 * clusters of 16;
 * items_per_cta: rounds of parts per resident CTA the tiles' work is cut
 * into. */
int dmrgpp_kron_get_config(dmrgpp_kron_handle h, int* cfg, int* items_per_cta);
int dmrgpp_kron_set_config(dmrgpp_kron_handle h, int cfg, int items_per_cta);

/* Times every configuration on this sector (reps applies each, minimum
 * kept), keeps the fastest and returns it with its time in microseconds.
 * cache_path (may be NULL): text file of earlier choices keyed by a
 * signature of the sector-size histogram (work quartiles and maximum of the
 * patch dimensions by octave, total work, terms) and the GPU name; a hit
 * skips the timing, a miss appends the new choice. */
int dmrgpp_kron_autotune(dmrgpp_kron_handle h, const char* cache_path, int reps, int* cfg,
                         double* us);

/* The last autotune's best FP64 apply time and, for a handle created with
 * DMRGPP_TF32X3, its TF32x3 apply time on the same sector (microseconds; -1
 * when not measured), so that a mixed-precision solve can pick the faster
 * arithmetic per sector (the TF32x3 form pays on large patches, not on
 * sectors of small ones).  Both times are kept in the tuning cache beside
 * the configuration. */
int dmrgpp_kron_tuned_times(dmrgpp_kron_handle h, double* fp64_us, double* tf32x3_us);

/* ---- Eigensolver on the device (replaces PsimagLite::LanczosSolver for one
 * sector, PsimagLite/src/PsimagLite/LanczosSolver.h:68-88 with
 * LanczosCore.h:147-272 and LanczosVectors.h:192-271) ---- */
typedef struct {
	size_t steps;         /* LanczosSteps, maximum steps (default 200) */
	size_t min_steps;     /* MinSteps (default 4) */
	size_t eigs_for_stop; /* EigsForStop: lowest Ritz values watched (default 1) */
	double tolerance;     /* LanczosEps: stop when they change by less (default 1e-12) */
	int    reortho;       /* full reorthogonalisation, Options=reortho (default 1) */
	int    check_every;   /* steps enqueued between stopping tests on the host (default 8) */
	int    use_graph;     /* 1 (default): the steps between two tests run as one CUDA graph,
	                         captured once per solve and replayed (the kernels choose their
	                         Lanczos columns on the device); 0: launched one by one.  Results
	                         are bitwise identical. */
	double residual_gap_ratio; /* 0 (default): off.  > 0: also stop (after min_steps) once the
	                         lowest Ritz pair's residual estimate beta_{j+1} |s_j| is below
	                         this fraction of the gap to the second Ritz value -- the start
	                         of a refinement that must converge to the lowest state.  No
	                         counterpart in the reference. */
} dmrgpp_lanczos_params;

/* Fills the reference's defaults (ParametersForSolver.h:93-120). */
void dmrgpp_lanczos_params_init(dmrgpp_lanczos_params* p);

/* Lowest eigenpair of the sector's H by Lanczos from init (patch order).
 * The Lanczos vectors stay on the device.  on_device: init and z are device
 * pointers (else host).  energy = lowest Ritz value of the final tridiagonal,
 * z = its Ritz vector (unit norm), steps_taken = the step at which the
 * stopping test passed.  Synchronous. */
int dmrgpp_lanczos_lowest(dmrgpp_kron_handle h, const dmrgpp_lanczos_params* p,
                          const double* init, int on_device, double* energy, double* z,
                          size_t* steps_taken);

/* Lowest eigenpair of every sector of a group handle (dmrgpp_kron_create_group)
 * by Lanczos, all sectors in lockstep: each step applies H to all sectors in
 * one persistent launch, and every vector operation is segmented by sector.
 * init and z are the concatenated sector vectors (device pointers when
 * on_device, else host); energies[s] and steps_taken[s] (may be NULL) per
 * sector.  Same recurrence and parameters as dmrgpp_lanczos_lowest; the
 * stopping test runs every check_every steps (a sector stops at the first
 * test point where its lowest eigs_for_stop Ritz values changed by less than
 * the tolerance over the last step, after min_steps, or when its Krylov space
 * is exhausted) and stopped sectors drop out of the vector work.  No
 * counterpart in the reference.  Synchronous. */
int dmrgpp_lanczos_lowest_group(dmrgpp_kron_handle h, const dmrgpp_lanczos_params* p,
                                const double* init, int on_device, double* energies, double* z,
                                size_t* steps_taken);

/* dmrgpp_lanczos_lowest_group restricted to the sectors with mask[s] != 0
 * (mask: host array, one int per sector; NULL = every sector).  The others
 * take no part (their H*x items and vector work are skipped): their
 * energies are NaN, their part of z is zero and their steps_taken 0.  For
 * finishing a few sectors of a group (e.g. those whose refinement did not
 * converge) at the cost of those sectors only.  No counterpart in the
 * reference.  Synchronous. */
int dmrgpp_lanczos_lowest_group_masked(dmrgpp_kron_handle h, const dmrgpp_lanczos_params* p,
                                       const double* init, int on_device, const int* mask,
                                       double* energies, double* z, size_t* steps_taken);

/* ---- Davidson with a preconditioned correction (no counterpart in the
 * reference, whose only eigensolver for this path is Lanczos) ---- */
typedef struct dmrgpp_mlp_s* dmrgpp_mlp_handle;

typedef enum {
	DMRGPP_PRECOND_NONE   = 0, /* correction = residual */
	DMRGPP_PRECOND_JACOBI = 1, /* correction = r / (theta - diag(H)) */
	DMRGPP_PRECOND_MLP    = 2  /* learned: dmrgpp_mlp_* network */
} dmrgpp_preconditioner;

typedef struct {
	size_t            max_iterations;    /* default 500 */
	size_t            max_subspace;      /* restart size, default 32 */
	double            tolerance;         /* stop when |r| <= tolerance * max(1, |theta|), default 1e-8 */
	int               preconditioner;    /* dmrgpp_preconditioner, default Jacobi */
	dmrgpp_mlp_handle mlp;               /* network for DMRGPP_PRECOND_MLP */
	double            mixed_tolerance;   /* mixed handles: leave the mixed phase below this, default 1e-4 */
	double            denominator_floor; /* Jacobi: |theta - d| >= floor * max(1,|theta|), default 1e-3 */
} dmrgpp_davidson_params;

typedef struct {
	size_t iterations;    /* Rayleigh-Ritz steps */
	size_t mixed_matvecs; /* H*x in the handle's mixed mode */
	size_t fp64_matvecs;  /* H*x in FP64 */
	size_t restarts;
	double residual_norm; /* final FP64 |H u - theta u| */
	int    converged;
} dmrgpp_davidson_stats;

void dmrgpp_davidson_params_init(dmrgpp_davidson_params* p);

/* Lowest eigenpair by Davidson from init (patch order).  On a handle created
 * with a mixed precision, the matvecs run in that mode until the residual
 * falls below mixed_tolerance (or stalls), then the solver restarts from its
 * Ritz vector in FP64 (FP64 refinement): the returned energy is the FP64
 * Rayleigh quotient and the convergence test is on the FP64 residual.
 * Returns DMRGPP_NOT_CONVERGED (with the best pair) after max_iterations. */
int dmrgpp_davidson_lowest(dmrgpp_kron_handle h, const dmrgpp_davidson_params* p,
                           const double* init, int on_device, double* energy, double* z,
                           dmrgpp_davidson_stats* stats);

/* Exact correction for training the learned preconditioner: solves
 * (I - u u^T)(H - theta)(I - u u^T) t = -r, t orthogonal to u, by conjugate
 * gradients in FP64 on the device (u unit norm, r orthogonal to u, theta
 * below the second eigenvalue).  All vectors are device pointers. */
int dmrgpp_correction_solve(dmrgpp_kron_handle h, const double* u, double theta, const double* r,
                            double* t, int max_iterations, double rel_tolerance, int* iterations,
                            double* rel_residual);

/* The preconditioner of the correction solves of this handle
 * (dmrgpp_correction_solve and the FP64 refinement): DMRGPP_PRECOND_NONE
 * (conjugate gradients on the projected operator, the default) or
 * DMRGPP_PRECOND_JACOBI (preconditioned by K = diag(H) - theta, kept at
 * least 1e-3 max(1, |theta|), projected as in Jacobi-Davidson:
 * z = K^-1 r - (<u, K^-1 r> / <u, K^-1 u>) K^-1 u).  Either solves the same
 * equation; the refinement's convergence test stays the FP64 residual.  No
 * counterpart in the reference. */
int dmrgpp_set_correction_preconditioner(dmrgpp_kron_handle h, int preconditioner);

/* FP64 residual refinement of an approximate lowest eigenvector psi (device,
 * patch order, updated in place), typically the Ritz vector of a solve with
 * mixed-precision matvecs.  Each outer step computes in FP64 the Rayleigh
 * quotient theta and residual r = H psi - theta psi; while |r| > tolerance *
 * max(1, |theta|) it solves the projected correction equation
 * (I - psi psi^T)(H - theta)(I - psi psi^T) t = -r by conjugate gradients
 * with the handle's current (mixed) matvecs (inner_iterations,
 * inner_tolerance) and sets psi <- (psi + t) / |psi + t|.  energy = final
 * FP64 Rayleigh quotient.  No counterpart in the reference. */
typedef struct {
	size_t outer_iterations;
	size_t inner_matvecs; /* matvecs of the correction solves (handle precision) */
	size_t fp64_matvecs;
	double residual_norm; /* final FP64 |H psi - theta psi| */
	int    converged;
} dmrgpp_refine_stats;

int dmrgpp_refine_lowest(dmrgpp_kron_handle h, double* psi, int max_outer, double tolerance,
                         int inner_iterations, double inner_tolerance, double* energy,
                         dmrgpp_refine_stats* stats);

/* The same refinement for every sector of a group handle
 * (dmrgpp_kron_create_group) at once: each sector runs the iteration of
 * dmrgpp_refine_lowest with its own Rayleigh quotient, residual and
 * conjugate-gradient scalars, and one launch per step applies H to all
 * sectors (FP64 for the Rayleigh quotients, the handle's precision in the
 * correction solves).  A sector leaves the outer iteration once
 * |r| <= tolerance * max(1, |theta|), and the conjugate gradients once its
 * residual is below inner_tolerance times its initial one or its projected
 * operator is not positive definite.  psi: the concatenated sector vectors
 * (device, updated in place); energies[s]: sector s's final FP64 Rayleigh
 * quotient; converged (may be NULL): per sector 1 when it met the tolerance.
 * stats (may be NULL): outer_iterations = most outer steps of any sector,
 * inner_matvecs and fp64_matvecs = group launches, residual_norm = largest
 * final sector residual, converged = every sector converged.  Returns
 * DMRGPP_NOT_CONVERGED when a sector did not converge (energies are still
 * written).  No counterpart in the reference.  Synchronous. */
int dmrgpp_refine_lowest_group(dmrgpp_kron_handle h, double* psi, int max_outer, double tolerance,
                               int inner_iterations, double inner_tolerance, double* energies,
                               int* converged, dmrgpp_refine_stats* stats);

/* Lowest eigenpair of every sector of a group handle (dmrgpp_kron_create_group)
 * by Davidson, all sectors in lockstep: per sector the iteration of
 * dmrgpp_davidson_lowest, with one group launch per iteration applying H to
 * every sector's new basis vector in the handle's precision (no FP64 phase:
 * on a mixed handle follow with dmrgpp_refine_lowest_group), each sector's
 * own projected matrix and lowest Ritz pair, and its own correction (none,
 * Jacobi, or the learned one with the sector's Ritz value and residual norm,
 * dmrgpp_mlp_precondition_group).  A sector stops once its residual
 * |r| <= tolerance * max(1, |theta|) (or its basis spans the sector) and then
 * drops out of the vector work and of the group H*x; all sectors restart
 * together when the basis reaches max_subspace (at most 128 here).
 * energies[s], z (the concatenated Ritz vectors: device when on_device),
 * converged (may be NULL: per sector 1 when its residual met the tolerance
 * or its basis spans the sector);
 * stats (may be NULL): iterations (lockstep), mixed_matvecs / fp64_matvecs
 * (group launches), restarts, residual_norm (largest sector residual),
 * converged (every sector).  Returns DMRGPP_NOT_CONVERGED with the last
 * pairs after max_iterations.  No counterpart in the reference. */
int dmrgpp_davidson_lowest_group(dmrgpp_kron_handle h, const dmrgpp_davidson_params* p,
                                 const double* init, int on_device, double* energies, double* z,
                                 int* converged, dmrgpp_davidson_stats* stats);

/* ---- Learned preconditioner: per-element MLP 4 -> 256 -> 256 -> 1 ----
 * Trained on the GPU by these kernels (FP32 master weights, Adam); inference
 * uses BF16 weights with FP32 accumulation.  All arrays are device pointers
 * unless named host. */
size_t      dmrgpp_mlp_num_params(void);
int         dmrgpp_mlp_create(unsigned long long seed, dmrgpp_mlp_handle* out);
int         dmrgpp_mlp_destroy(dmrgpp_mlp_handle m);
int         dmrgpp_mlp_get_params(dmrgpp_mlp_handle m, float* host, size_t n);
int         dmrgpp_mlp_set_params(dmrgpp_mlp_handle m, const float* host, size_t n);
int         dmrgpp_mlp_get_grads(dmrgpp_mlp_handle m, float* host, size_t n);
/* features x (n x 4, float) of residual r at Ritz value theta with |r| = rnorm */
int         dmrgpp_mlp_features(const double* diag, const double* r, double theta, double rnorm,
                                size_t n, float* x, void* stream);
/* FP32 forward of rows feature rows (activations kept for backward); out may be NULL */
int         dmrgpp_mlp_forward(dmrgpp_mlp_handle m, const float* x, int rows, float* out, void* stream);
/* gradients of the weighted mean squared error against targets y for the last
 * forward (weight may be NULL); *loss (host) receives the loss; synchronous */
int         dmrgpp_mlp_backward(dmrgpp_mlp_handle m, const float* x, const float* y,
                                const float* weight, double* loss, void* stream);
int         dmrgpp_mlp_adam_step(dmrgpp_mlp_handle m, float lr, void* stream);
/* t = learned correction of residual r (what the Davidson solver applies).
 * Inference uses the BF16 copy of the weights with FP32 accumulation:
 * DMRGPP_MLP_TENSOR_CORES (default) runs one fused tcgen05 kernel (layer 1
 * and both tanh on the CUDA cores, h1 rounded to BF16, layer 2 as BF16 MMAs
 * into FP32 tensor memory); DMRGPP_MLP_CUDA_CORES runs the FP32 GEMM kernels
 * of training with the BF16 weights widened to FP32 (h1 kept in FP32).  A
 * tensor-core launch whose bounded wait gave up is reported as
 * DMRGPP_TIMEOUT by the next precondition call. */
enum { DMRGPP_MLP_TENSOR_CORES = 0, DMRGPP_MLP_CUDA_CORES = 1 };
int         dmrgpp_mlp_set_inference(dmrgpp_mlp_handle m, int mode);
int         dmrgpp_mlp_precondition(dmrgpp_mlp_handle m, const double* diag, const double* r,
                                    double theta, double rnorm, double* t, size_t n, void* stream);
/* The learned correction of the concatenated residuals of nsectors sectors
 * (a group handle's layout): element e of sector s is corrected with that
 * sector's Ritz value theta[s] and residual norm rnorm[s], bitwise as
 * dmrgpp_mlp_precondition on the sector alone.  sector_start (nsectors + 1
 * offsets), theta and rnorm are device arrays. */
int         dmrgpp_mlp_precondition_group(dmrgpp_mlp_handle m, const double* diag, const double* r,
                                          const long long* sector_start, const double* theta,
                                          const double* rnorm, int nsectors, double* t, size_t n,
                                          void* stream);
const char* dmrgpp_mlp_last_error(dmrgpp_mlp_handle m);

/* Host helper: eigenvalues (ascending) and, when vectors != NULL, eigenvectors
 * (n x n column-major) of the symmetric tridiagonal matrix diag/offdiag; the
 * role of dstedc in TridiagonalMatrix.cpp:21. */
int dmrgpp_tridiag_eigen(size_t n, const double* diag, const double* offdiag, double* eigs,
                         double* vectors);

/* Sector gather / scatter on the device (InitKronHamiltonian.h:158-221 copyIn,
 * InitKronBase.h:315-360 copyOut): dst[q] = src[idx[q]] and dst[idx[q]] =
 * src[q] for q < n, with idx the map from patch order to the sector's
 * positions in super-basis order; enqueued on stream (cudaStream_t). */
int dmrgpp_gather(const double* src, const int64_t* idx, double* dst, size_t n, void* stream);
int dmrgpp_scatter(const double* src, const int64_t* idx, double* dst, size_t n, void* stream);

/* The index those two apply, built on the host cores from the superblock
 * basis as the reference's copyIn / copyOut read it
 * (InitKronHamiltonian.h:158-221, InitKronBase.h:315-360):
 *   idx[vstart[p] + iR + iL * r_p] = perm_inverse[(iL + Loff) + (iR + Roff) * nl] - offset
 * for patch p = (left group patch_left[p], right group patch_right[p]), its
 * l_p and r_p states starting at Loff = left_partition[patch_left[p]] and
 * Roff = right_partition[patch_right[p]], nl = left_partition[left_groups],
 * vstart the prefix sums of l_p r_p (InitKronBase.h:277-310).  The arrays are
 * the reference's GenIjPatch patches (GenIjPatch.h:104-118), Basis::partition
 * of the left and right blocks (left_groups + 1 and right_groups + 1
 * offsets), super().permutationInverse() (nl x nr entries) and the sector's
 * offset and size.  Every entry is checked as the reference asserts
 * (offset <= perm_inverse[.] < offset + sector_size) and the map must be a
 * permutation of the sector; otherwise DMRGPP_INVALID_ARG with the reason in
 * dmrgpp_kron_last_error(NULL).  idx: sector_size host entries. */
typedef struct {
	size_t        npatches;
	const size_t* patch_left;      /* per patch: its left group */
	const size_t* patch_right;     /* per patch: its right group */
	size_t        left_groups;
	const size_t* left_partition;  /* left_groups + 1 state offsets */
	size_t        right_groups;
	const size_t* right_partition; /* right_groups + 1 state offsets */
	const size_t* perm_inverse;    /* nl x nr super-basis positions */
	size_t        offset;          /* first super-basis position of the sector */
	size_t        sector_size;
} dmrgpp_gather_index_desc;

int dmrgpp_kron_gather_index(const dmrgpp_gather_index_desc* desc, int64_t* idx);

/* The sector's patches (GenIjPatch::GenIjPatch, GenIjPatch.h:104-118): every
 * (left group i, right group j), i outer and j inner, whose quantum numbers
 * add up to the target.  left_qn / right_qn: qn_len integers per group
 * (additive components: 2 Sz, N_up, N_down, ...), target: qn_len integers.
 * Writes up to capacity pairs, the count to *npatches; DMRGPP_INVALID_ARG if
 * there are more.  Host only. */
int dmrgpp_kron_patch_list(size_t left_groups, const int64_t* left_qn, size_t right_groups,
                           const int64_t* right_qn, size_t qn_len, const int64_t* target,
                           size_t capacity, size_t* patch_left, size_t* patch_right,
                           size_t* npatches);

/* ---- Wave-function transformation between two patch layouts ----
 * The GEMM core of the reference's patch-wise WFT (Wft/WftAccelPatches.h:
 * 43-66, BlockDiagWf.h:131-260 ParallelBlockTransform::doTask): per patch,
 * Ynew = opL(W_L) * Yold * opR(W_R) with the block-diagonal transformations
 * of the system and environment.  In the sector layout of this library a
 * patch block is r x l column-major (right index fastest), so for every
 * output patch q with source patch p = src[q] >= 0:
 *     Y_q = WR_q * X_p * WL_q^T,
 * WR_q applied to the right index (r_out[q] x r_in[p]) and WL_q to the left
 * index (l_out[q] x l_in[p]); in the reference's terms WL = opL(W_L) and
 * WR = opR(W_R)^T.  trans_WL / trans_WR = 1: the given block is stored
 * transposed (l_in[p] x l_out[q] / r_in[p] x r_out[q]), which covers the
 * reference's 'C' / 'T' / 'N' choices for real blocks.  Output patches
 * without a source (src[q] < 0) are zero.  The re-indexing of the
 * transformed patches into the new superblock's order
 * (BlockDiagWf::toVectorWithOffsets) is a permutation: dmrgpp_gather.
 * Both contractions run as FP64 grouped GEMMs on the FP64 tensor pipe. */
typedef struct {
	size_t               np_in;
	const size_t*        l_in;
	const size_t*        r_in;
	size_t               np_out;
	const size_t*        l_out;
	const size_t*        r_out;
	const long long*     src;   /* np_out entries: source input patch or -1 */
	const double* const* WL;    /* np_out blocks (NULL where src < 0) */
	const size_t*        ld_WL;
	const double* const* WR;
	const size_t*        ld_WR;
	int                  trans_WL;
	int                  trans_WR;
	void*                stream; /* cudaStream_t, NULL = default stream */
	int                  device; /* -1 = current device */
} dmrgpp_wft_desc;

typedef struct dmrgpp_wft_s* dmrgpp_wft_handle;

int dmrgpp_wft_create(const dmrgpp_wft_desc* desc, dmrgpp_wft_handle* out);
/* y (output layout) = transform of x (input layout); host pointers are copied
 * through device staging, device pointers (on_device = 1) are used in place
 * and the call only enqueues. */
int dmrgpp_wft_apply(dmrgpp_wft_handle h, const double* x, double* y, int on_device);
int dmrgpp_wft_dims(dmrgpp_wft_handle h, size_t* dim_in, size_t* dim_out);
/* sum over transformed patches of 2 r_out r_in l_in + 2 r_out l_in l_out */
int dmrgpp_wft_flops(dmrgpp_wft_handle h, double* flops);
int dmrgpp_wft_destroy(dmrgpp_wft_handle h);
const char* dmrgpp_wft_last_error(dmrgpp_wft_handle h);

/* ---- Density-matrix truncation after a sector solve ----
 * The reference's per-patch SVD route (DensityMatrixSvd.h:285-410,
 * Truncation.h:218-285 changeBasis, 373-519 updateKeptStates /
 * computeKeptStates).  The block being truncated (the system block when
 * side = 0, the environment when side = 1) has ngroups quantum-number groups
 * of group_size[g] states; patch p of the sector (left group of l_p, right
 * group of r_p states; block X_p is r_p x l_p column-major) belongs to group
 * patch_group[p] of that block.  For ntargets sector vectors (psi: device,
 * ntargets x D, target-major, patch order) with weights w_t:
 *     side 0:  rho_g = sum_t w_t sum_{p in g} X_{t,p}^T X_{t,p}   (l_p x l_p)
 *     side 1:  rho_g = sum_t w_t sum_{p in g} X_{t,p} X_{t,p}^T   (r_p x r_p)
 * which is M_g M_g^T of the reference's stacked per-group matrix M_g, so its
 * eigenvalues are the squared singular values the reference takes from
 * svd('A', M_g).  The rho_g are formed by grouped DGEMMs on the FP64 tensor
 * pipe; their tridiagonal reductions (Householder) and eigenvalues (implicit
 * QL) are computed on the host cores, the kept eigenvectors by inverse
 * iteration there and transformed back on the device; groups without
 * patches have rho_g = 0.  All states are ranked by eigenvalue
 * (ascending; ties by group, then by index), the kept number K follows
 * computeKeptStates (tolerance < 0: K = m; else the fewest states, not below
 * m_min, whose removal keeps the discarded weight within the tolerance, never
 * more than m), and the N - K lowest are removed. */
typedef struct {
	size_t        npatches;
	const size_t* left_patch_size;
	const size_t* right_patch_size;
	const size_t* patch_group; /* per patch: its group in the block being truncated */
	size_t        ngroups;
	const size_t* group_size;  /* states per group; l_p (side 0) or r_p (side 1) of its patches */
	int           side;        /* 0: system (left) block, 1: environment (right) block */
	size_t        ntargets;
	const double* psi;         /* device, ntargets x D */
	const double* weights;     /* host, ntargets; NULL: every weight 1 */
	void*         stream;
	int           device;      /* -1: current */
} dmrgpp_density_desc;

/* Host outputs: eigenvalues (sum_g group_size[g] entries): each group's
 * eigenvalues ascending, group after group; kept[g]: states kept in group g
 * (its kept[g] largest eigenvalues); vectors (may be NULL; room for
 * sum_g group_size[g]^2 doubles): the kept eigenvectors, group after group,
 * group g's as a group_size[g] x kept[g] column-major block whose columns
 * follow its last kept[g] eigenvalues (ascending) -- the truncated
 * transformation of the reference's changeBasis; *kept_total = K;
 * *discarded = the sum of the removed eigenvalues' magnitudes (the
 * reference's "Discarded weight").  Synchronous.  Errors: the calling
 * thread's message, dmrgpp_kron_last_error(NULL). */
int dmrgpp_density_truncate(const dmrgpp_density_desc* d, size_t m, double tolerance, size_t m_min,
                            double* eigenvalues, double* vectors, size_t* kept, size_t* kept_total,
                            double* discarded);

/* Wall-clock seconds of the phases of the calling thread's last
 * dmrgpp_density_truncate (host clock, each phase waiting for its device
 * work): RHO the density matrices (device, to the host), EIGENVALUES the
 * tridiagonal reductions and eigenvalues (host cores), SELECT the ranking,
 * VECTORS_HOST the inverse iterations and packing, VECTORS_DEVICE the
 * back-transformation and copy out, TOTAL the whole call.  n (<=
 * DMRGPP_TRUNC_NPHASES) values are written to t. */
enum {
	DMRGPP_TRUNC_RHO            = 0,
	DMRGPP_TRUNC_EIGENVALUES    = 1,
	DMRGPP_TRUNC_SELECT         = 2,
	DMRGPP_TRUNC_VECTORS_HOST   = 3,
	DMRGPP_TRUNC_VECTORS_DEVICE = 4,
	DMRGPP_TRUNC_TOTAL          = 5,
	DMRGPP_TRUNC_NPHASES        = 6
};
int dmrgpp_density_profile(double* t, int n);

/* Last error message of a handle, or of the calling thread's last failed
 * create when h is NULL.  Never returns NULL. */
const char* dmrgpp_kron_last_error(dmrgpp_kron_handle h);

/* Library version string. */
const char* dmrgpp_version(void);

#ifdef __cplusplus
}
#endif

#endif /* DMRGPP_KRON_H */
