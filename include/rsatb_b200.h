/*
 * rsatb_b200.h -- C ABI of the B200 (sm_100a) implementation of RSATB's
 * KPM / S^-1/2 / FFT-Chebyshev hot path.
 *
 * Plain C: opaque handles, raw pointers and sizes, integer status codes.
 * No exception crosses this boundary; on failure a function returns a
 * non-zero rsatb_status and rsatb_last_error() holds a message for the
 * calling thread.
 *
 * Every call is asynchronous with respect to the host unless its comment
 * says it copies results to host memory (those synchronise the context's
 * stream before returning).  A context owns one CUDA stream and is not
 * re-entrant: one host thread at a time per context.
 *
 * Data layouts (all row-major, matching vbcsr's DistMultiVector):
 *   multivector   N x R, element (row, col) at [row * R + col]; a complex
 *                 multivector stores (re, im) pairs, so it is N x 2R reals.
 *   BSR matrix    uniform b x b blocks; block k of block row i holds
 *                 A[i*b + r, col_ind[k]*b + c] at values[k*b*b + r*b + c]
 *                 (vbcsr MatrixLayout::RowMajor); complex values interleaved.
 */
#ifndef RSATB_B200_H
#define RSATB_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define RSATB_API __attribute__((visibility("default")))
#else
#define RSATB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  0..6 mirror rsatb::calc::isqrt::Status
 * (rsatb/calc/isqrt_action.hpp:84-92, in that order); the rest are device
 * conditions the CPU reference does not have. */
typedef enum {
    RSATB_SUCCESS = 0,
    RSATB_INVALID_ARGUMENT = 1,
    RSATB_FAST_PATH_REJECTED = 2,
    RSATB_RANK_BREAKDOWN = 3,
    RSATB_NOT_POSITIVE_DEFINITE = 4,
    RSATB_NEAR_SINGULAR = 5,
    RSATB_NUMERICAL_FAILURE = 6,   /* isqrt::Status::LapackFailure */
    RSATB_CUDA_ERROR = 16,
    RSATB_OUT_OF_MEMORY = 17,
    RSATB_NOT_SUPPORTED = 18,
    RSATB_DIVERGED = 19,
    RSATB_INTERRUPTED = 20
} rsatb_status;

/* Element types of matrices and multivectors. */
typedef enum {
    RSATB_F64 = 0,
    RSATB_F32 = 1,
    RSATB_C128 = 2,   /* complex<double>, interleaved */
    RSATB_C64 = 3     /* complex<float>, interleaved */
} rsatb_dtype;

/* Operator forms, rsatb::calc::ChebyOpForm (rsatb/calc/cheby.hpp:78-82).
 * The Solve form runs one batched CG with S per application; it is served
 * by rsatb_cheb_apply_op and (plain recurrence) rsatb_kpm_dos_moments. */
typedef enum {
    RSATB_FORM_ORTHOGONAL = 0,
    RSATB_FORM_SANDWICH = 1,
    RSATB_FORM_SOLVE = 2
} rsatb_form;

/* Summation kernels, rsatb::calc::KpmKernel (rsatb/calc/kpm.hpp:49). */
typedef enum {
    RSATB_KPM_NONE = 0,
    RSATB_KPM_JACKSON = 1,
    RSATB_KPM_COSTAPER = 2,
    RSATB_KPM_VPTAPER = 3
} rsatb_kpm_kernel;

/* Sample-vector distributions for rsatb_set_random. */
typedef enum {
    RSATB_RANDOM_PHASE = 0,       /* e^{i theta}, theta uniform; complex only */
    RSATB_RANDOM_RADEMACHER = 1,  /* +-1 */
    RSATB_RANDOM_UNIFORM = 2      /* uniform in [-1, 1) (real and imaginary) */
} rsatb_random_kind;

/* rsatb_bsr_create flags. */
#define RSATB_BSR_DEVICE_POINTERS 1u  /* row_ptr/col_ind/values are device pointers */
#define RSATB_BSR_IMAGINARY_UNIT  2u  /* real values W; the matrix is i*W */

typedef struct rsatb_context* rsatb_ctx_t;
typedef struct rsatb_bsr_matrix* rsatb_bsr_t;

/* ------------------------------------------------------------------ errors */

/* Message of the last failure on the calling thread ("" if none). */
RSATB_API const char* rsatb_last_error(void);
/* Library version, major*10000 + minor*100 + patch. */
RSATB_API int rsatb_version(void);

/* ----------------------------------------------------------- context, memory */

/* Creates a context on `device` with its own non-blocking stream. */
RSATB_API int rsatb_ctx_create(int device, rsatb_ctx_t* out);
RSATB_API int rsatb_ctx_destroy(rsatb_ctx_t ctx);
/* Launches on the caller's cudaStream_t (passed as void*) from now on; NULL
 * is the legacy default stream.  Work already queued on the previous stream
 * is waited for first. */
RSATB_API int rsatb_ctx_set_stream(rsatb_ctx_t ctx, void* stream);
/* The stream the context launches on (a cudaStream_t). */
RSATB_API void* rsatb_ctx_stream(rsatb_ctx_t ctx);
/* Waits for the work queued on the context's stream.  Returns
 * RSATB_CUDA_ERROR ("... bounded wait ...") when a step kernel of an
 * asynchronous call queued since the last check gave up on a bounded wait
 * (rsatb_bsr_mult_dense, rsatb_cheb_apply_op, rsatb_cheb_apply_dual and
 * rsatb_cheb_propagate return before their kernels run, so they cannot
 * report it themselves); the report clears the context's fault word.  Every
 * entry point that synchronises (moments, transport, CG, the adjoint)
 * reports such a give-up the same way, its own or an earlier call's. */
RSATB_API int rsatb_ctx_synchronize(rsatb_ctx_t ctx);
/* Number of kernels the context has launched so far (all entry points). */
RSATB_API int64_t rsatb_ctx_launch_count(rsatb_ctx_t ctx);

RSATB_API int rsatb_device_alloc(rsatb_ctx_t ctx, size_t bytes, void** out);
RSATB_API int rsatb_device_free(rsatb_ctx_t ctx, void* ptr);
/* Stream-ordered copies; the *_sync forms return after the copy landed. */
RSATB_API int rsatb_copy_to_device(rsatb_ctx_t ctx, void* dst, const void* src, size_t bytes);
RSATB_API int rsatb_copy_to_host_sync(rsatb_ctx_t ctx, void* dst, const void* src, size_t bytes);

/* ------------------------------------------------------------- BSR matrices */

/* vbcsr BlockSpMat<T> with a uniform block size (construct + add_block +
 * assemble in one call).  row_ptr has n_block_rows+1 entries, col_ind
 * nnz_blocks entries (sorted within a row), values nnz_blocks*b*b
 * elements of `dtype`.  Host pointers are copied; with
 * RSATB_BSR_DEVICE_POINTERS they are copied device-to-device. */
RSATB_API int rsatb_bsr_create(rsatb_ctx_t ctx, int n_block_rows, int n_block_cols,
                     int block_size, int64_t nnz_blocks, const int32_t* row_ptr,
                     const int32_t* col_ind, const void* values, rsatb_dtype dtype,
                     unsigned flags, rsatb_bsr_t* out);
RSATB_API int rsatb_bsr_destroy(rsatb_bsr_t A);
/* A^H as a new matrix (BlockSpMat::mult_dense_adjoint's operator, built once
 * so that every later apply uses the forward row-gather kernel). */
RSATB_API int rsatb_bsr_adjoint(rsatb_ctx_t ctx, rsatb_bsr_t A, rsatb_bsr_t* out);
/* Copy of A with values converted to `dtype` (F64 <-> F32, C128 <-> C64). */
RSATB_API int rsatb_bsr_convert(rsatb_ctx_t ctx, rsatb_bsr_t A, rsatb_dtype dtype, rsatb_bsr_t* out);
RSATB_API int rsatb_bsr_info(rsatb_bsr_t A, int* n_block_rows, int* n_block_cols, int* block_size,
                   int64_t* nnz_blocks, int* dtype, unsigned* flags);
/* The pattern to host memory: row_ptr (n_block_rows + 1 entries) and
 * col_ind (nnz_blocks entries), vbcsr BlockSpMat::row_ptr() / col_ind().
 * Synchronises. */
RSATB_API int rsatb_bsr_pattern(rsatb_ctx_t ctx, rsatb_bsr_t A, int32_t* row_ptr,
                                int32_t* col_ind);
/* Device pointer to the values array (nnz_blocks*b*b elements). */
RSATB_API void* rsatb_bsr_values(rsatb_bsr_t A);
/* Overwrites the values from host (or device with RSATB_BSR_DEVICE_POINTERS). */
RSATB_API int rsatb_bsr_set_values(rsatb_ctx_t ctx, rsatb_bsr_t A, const void* values, unsigned flags);

/* Bloch sum of real-space images into the values of `out` (C128, its
 * pattern already set): block s = sum over the bonds e of slot s of
 * w_e (i if imag_unit) exp(-2 pi i k . R_e) V_e, summed in bond order.
 * BlochPhase / AddLocalBlock (rsatb/operator/block_assembly.hpp:31-100);
 * with w_e = (R + r_j - r_i)_a and imag_unit the commutator velocity
 * (rsatb/operator/commutator_velocity.hpp:114-255).  Device arrays: slot_ptr
 * (nnz_blocks + 1, int64: bonds slot_ptr[s] .. slot_ptr[s+1]-1 belong to
 * block s), shifts (3 doubles per bond, in the units k is given against),
 * image_values (b*b per bond, F64 or C128, row-major), weights (one per
 * bond, or NULL).  k: host, 3 doubles.  Stream-ordered, no sync. */
RSATB_API int rsatb_bloch_sum(rsatb_ctx_t ctx, rsatb_bsr_t out, const int64_t* slot_ptr,
                              const double* shifts, const void* image_values,
                              rsatb_dtype image_dtype, const double* weights, const double* k,
                              int imag_unit);

/* Solves S X = B for every column (rsatb::calc::LinearSolver::solve for a
 * multivector, rsatb/calc/solver.hpp:216-312): batched CG from X's
 * contents, per-column step lengths, a column below tol or at breakdown
 * frozen, stopping when the largest column residual |r| < tol or after
 * max_iter iterations.  With Z and ZH = Z^H (both or neither): symmetric
 * preconditioning by the graph-local factor (solver.hpp:329-338), the CG on
 * Z^H S Z Y = Z^H B from Y = 0 and X = Z Y, tol then bounding that
 * system's residual.  S square SPD (Hermitian), B and X device panels of
 * n_vectors (1..256) columns, distinct, 16-byte aligned.  iterations and
 * max_residual (host, may be NULL) receive the count and the final
 * residual.  Reads the residuals back every iteration (synchronises). */
RSATB_API int rsatb_cg_solve(rsatb_ctx_t ctx, rsatb_bsr_t S, rsatb_bsr_t Z, rsatb_bsr_t ZH,
                             const void* B, void* X, int n_vectors, rsatb_dtype vec_dtype,
                             double tol, int max_iter, int* iterations, double* max_residual);

/* Y = alpha * A X.  BlockSpMat::mult_dense (vbcsr), called by
 * Chebyshev::mult_by (rsatb/calc/cheby.hpp:599-606).  X, Y device, N x R of
 * vec_dtype; a real matrix may multiply a complex multivector. */
RSATB_API int rsatb_bsr_mult_dense(rsatb_ctx_t ctx, rsatb_bsr_t A, const void* X, void* Y,
                         int n_vectors, rsatb_dtype vec_dtype, double alpha);

/* ----------------------------------------------------- rescaled operator */

/* The operator a Chebyshev<T> iterates (rsatb/calc/cheby.hpp:147-201):
 * Orthogonal: H;  Sandwich: Z^H H Z with Z and its adjoint ZH;  Solve:
 * S^-1 H with the overlap S, one batched CG per application
 * (LinearSolver(1e-8, 1000), cheby.hpp:188-199; cg_tol and cg_max_iter 0
 * select those defaults), preconditioned symmetrically by Z when Z and ZH
 * are set (the reference's default route: the graph-local seed
 * preconditions an exact solve).
 * Every matrix must share one precision; the multivectors passed with the
 * operator must have that precision too (F64/C128 or F32/C64). */
typedef struct {
    int form;            /* rsatb_form */
    rsatb_bsr_t H;
    rsatb_bsr_t Z;       /* sandwich only */
    rsatb_bsr_t ZH;      /* sandwich only: Z^H (rsatb_bsr_adjoint) */
    double center;       /* (emax + emin)/2 */
    double half_width;   /* (emax - emin)/2 */
    rsatb_bsr_t S;       /* solve only: the overlap, SPD */
    double cg_tol;       /* solve only: largest column residual |r| at exit */
    int cg_max_iter;     /* solve only: CG iterations per application at most */
} rsatb_cheb_op;

/* Y = ((Op) X - center X) / half_width.  Chebyshev::apply_op NORMAL
 * (rsatb/calc/cheby.hpp:232-235, apply_form :555-591). */
RSATB_API int rsatb_cheb_apply_op(rsatb_ctx_t ctx, const rsatb_cheb_op* op, const void* X, void* Y,
                        int n_vectors, rsatb_dtype vec_dtype);

/* Y = scale * (V dressed by the operator form) X: V X (Orthogonal),
 * Z^H V Z X (Sandwich) or S^-1 V X (Solve: one CG with S, V X its target
 * and initial guess).  Chebyshev::apply_dual NORMAL (rsatb/calc/cheby.hpp:
 * 249-291) for a plain velocity matrix V (RSATB_BSR_IMAGINARY_UNIT for the
 * i W of a real k-point).  X, Y: device N x n_vectors panels, 16-byte
 * aligned, distinct. */
RSATB_API int rsatb_cheb_apply_dual(rsatb_ctx_t ctx, const rsatb_cheb_op* op, rsatb_bsr_t V,
                                    const void* X, void* Y, int n_vectors, rsatb_dtype vec_dtype,
                                    double scale);
/* The same in ChebyMode::ADJOINT: scale * V S^-1 X for the Solve form (the
 * CG from zero), equal to rsatb_cheb_apply_dual for the two Hermitian
 * forms. */
RSATB_API int rsatb_cheb_apply_dual_adjoint(rsatb_ctx_t ctx, const rsatb_cheb_op* op,
                                            rsatb_bsr_t V, const void* X, void* Y,
                                            int n_vectors, rsatb_dtype vec_dtype, double scale);

/* Y = sum_{n < n_coeffs} c_n T_n(Op~) X, Chebyshev::propagate
 * (rsatb/calc/cheby.hpp:367-441): coeffs holds n_coeffs complex values as
 * (re, im) pairs; a real panel takes Re(c_n), as the reference's CoeffCast
 * does for a real scalar type.  n_coeffs == 0 leaves Y unchanged.  X, Y:
 * device panels, 16-byte aligned, distinct.  The Solve form runs one CG per
 * application, each started from its output panel's previous contents
 * (T_{n-3}; the first two from zero). */
RSATB_API int rsatb_cheb_propagate(rsatb_ctx_t ctx, const rsatb_cheb_op* op, const void* X,
                                   void* Y, int n_vectors, rsatb_dtype vec_dtype,
                                   const double* coeffs, int n_coeffs);

/* KPM trace moments averaged over the R columns of psi,
 * rsatb::calc::kpm_dos_moments (rsatb/calc/dos.hpp:125-190): doubled
 * (two moments per matvec) when `doubled` != 0, else the plain recurrence
 * mu_n = <psi|T_n|psi> (Chebyshev::compute_moments, cheby.hpp:479-514).
 * The recurrence, its rescaling and the FP64 column dots all run on the
 * device; mu_out (host) receives n_moments complex values as 2*n_moments
 * doubles.  col_mu_out (host, may be NULL) receives the per-column
 * moments, [n_moments][R] complex. */
RSATB_API int rsatb_kpm_dos_moments(rsatb_ctx_t ctx, const rsatb_cheb_op* op, const void* psi,
                          int n_vectors, rsatb_dtype vec_dtype, int n_moments, int doubled,
                          double* mu_out, double* col_mu_out);

/* rsatb_kpm_dos_moments for callers that cannot allocate device memory:
 * for example a process whose device memory is reserved in full by another
 * allocator (a framework's caching pool sized to the whole GPU), where a new
 * cudaMalloc fails, or a latency-critical loop that cannot take the
 * device-wide synchronisation of cudaMalloc/cudaFree.  Same arguments,
 * arithmetic and results as rsatb_kpm_dos_moments; it allocates nothing:
 * all its temporaries live in one fixed 32 MiB static device array that
 * every GPU loading the library holds until exit.  The first call on a
 * device looks up that array's address (make it before any stream capture);
 * with lazy module loading (the CUDA 12.2+ default) that first call is also
 * what reserves the 32 MiB on the device, so a caller that hands the rest
 * of the device to another allocator makes it before that allocator takes
 * the memory.  A bounded wait of a step kernel that gives up fails the call
 * with RSATB_CUDA_ERROR (its fault word is in the static array too).
 * Problems whose temporaries exceed 32 MiB are rejected with
 * RSATB_INVALID_ARGUMENT; calls overlapping on the GPU share the array and
 * race, so serialise them.  No counterpart in the reference: RSATB runs on
 * the CPU and has no device allocations to avoid. */
RSATB_API int rsatb_kpm_dos_moments_noalloc(rsatb_ctx_t ctx, const rsatb_cheb_op* op,
                                            const void* psi, int n_vectors,
                                            rsatb_dtype vec_dtype, int n_moments, int doubled,
                                            double* mu_out, double* col_mu_out);

/* ------------------------------------------------------------ sample vectors */

/* Seeded sample vectors, the device half of SampleVectors::initialize
 * (rsatb/calc/observables.hpp:84-96, vbcsr set_random(seed, normalize,
 * atom_index)).  Element (row, col) of the N x R output is a function of
 * (seed, atom_index[atom], orbital-in-atom, col) only, through
 * Philox-4x32-10, so it does not depend on the launch shape, and
 * `normalize` scales by 1/sqrt(n_rows_global).  atom_index is a host array
 * of n_atoms stable ids; every atom has orbitals_per_atom rows.  Column j
 * of the output is global sample column first_column + j, so ranks that
 * split the samples by column draw disjoint columns of one global set. */
RSATB_API int rsatb_set_random(rsatb_ctx_t ctx, uint64_t seed, int kind, int normalize,
                     const int64_t* atom_index, int n_atoms, int orbitals_per_atom,
                     int64_t n_rows_global, int n_vectors, int64_t first_column,
                     rsatb_dtype dtype, void* out);

/* -------------------------------------------------------------- densities */

/* rho(x_j) = (g0 mu0 + 2 sum_n g_n mu_n T_n(x_j)) / (pi sqrt(1 - x_j^2)),
 * x clamped by edge_inset.  rsatb::calc::evaluate_kpm_density
 * (rsatb/calc/kpm.hpp:206-241) with kpm_kernel_weights (:52-85).
 * moments: host, 2*n_moments doubles (complex; real parts used);
 * x, rho_out: host arrays of nx doubles.  Computed on the device. */
RSATB_API int rsatb_evaluate_kpm_density(rsatb_ctx_t ctx, const double* moments, int n_moments,
                               const double* x, int nx, double edge_inset, int kernel,
                               double* rho_out);

/* Chebyshev coefficients of e^{-i x t} (forward != 0) or e^{+i x t}:
 * c_n = (2 - delta_n0) (-+i)^n J_n(t), truncated before the first n with
 * |J_n(t)| <= precision and |J_{n+1}(t)| <= precision.
 * rsatb::calc::timeprop_coeff (rsatb/calc/cheby.hpp:85-106) with
 * build_bessel_vector (rsatb/calc/bessel.hpp:9-52).  The Bessel values are
 * computed on the device (Miller's backward recurrence).  *n_coeffs gets the
 * full length; the first min(length, capacity) coefficients are written to
 * coeffs (host, (re, im) pairs).  t must be positive and below about 64,000
 * (the reference's order limit 65536), else RSATB_INVALID_ARGUMENT. */
RSATB_API int rsatb_timeprop_coeff(rsatb_ctx_t ctx, double time_step, double precision,
                                   int forward, int capacity, double* coeffs, int* n_coeffs);

/* The correlation-series DOS of ComputeDos(method = "corr")
 * (rsatb/calc/observables.hpp:393-428): C(j pi) = sum_n c_n(j pi) mu_n for
 * j = 1..nt with the coefficients above (corr_from_moments,
 * rsatb/calc/dos.hpp:30-46; C(0) = mu_0), a Hann window, the mirror
 * C(-t) = conj C(t), an unnormalised inverse FFT of 2 nt points (cuFFT) and
 * the reorder to energies (i - nt)/nt, i/nt.  moments: host, (re, im) x
 * n_moments (at least rsatb_timeprop_coeff(nt pi) terms for the full
 * expansion).  cdos_out (host, (re, im) x (nt + 1)) and dos_out (host,
 * 2 nt) may each be NULL. */
RSATB_API int rsatb_corr_dos(rsatb_ctx_t ctx, const double* moments, int n_moments, int nt,
                             double precision, double* cdos_out, double* dos_out);

/* sigma(mu, T) of the six tensor components from a zero-temperature
 * spectrum, rsatb::calc::integrate_dc_spectrum
 * (rsatb/calc/fftcheb_transport.hpp:950-1040): T <= 0 interpolates linearly
 * at mu (clamped to the grid's ends); T > 0 (kelvin) integrates the
 * piecewise-linear spectrum exactly against -df/dE.  sigma: host,
 * n_energy x 6; energy: host, n_energy values, strictly ascending when
 * T > 0 (else RSATB_INVALID_ARGUMENT); sigma_out: host, 6 values.
 * Computed on the device (one thread per component, energy order). */
RSATB_API int rsatb_integrate_dc_spectrum(rsatb_ctx_t ctx, const double* sigma,
                                          const double* energy, int n_energy, double mu,
                                          double temp, double* sigma_out);

/* ------------------------------------------------------------ adjoint KPM */

/* Counters of one rsatb_kpm_moments_vjp call. */
typedef struct {
    int checkpoint_stride;    /* moments per recomputed segment */
    int segments;             /* checkpoint segments */
    double forward_ms;        /* device time of the forward pass (moments, checkpoints) */
    double backward_ms;       /* device time of the recompute, adjoint recurrence and SDDMM */
    int panels_held;          /* N x R panels held at once */
} rsatb_adjoint_stats;

/* Gradient of f = sum_n dmu[n] mu_n with respect to every stored block value
 * of H, where mu_n = (1/R) sum_s psi_s^T T_n((H - center)/half_width) psi_s
 * are the plain KPM moments of Chebyshev::compute_moments
 * (rsatb/calc/cheby.hpp:479-514) averaged over the R columns.  No
 * counterpart in the reference, which has no differentiation code: this is
 * the hand-written adjoint Chebyshev recurrence
 *     lambda_n = (dmu_n / R) psi + 2 A lambda_{n+1} - lambda_{n+2},
 *     df/dA = lambda_1 t_0^T + 2 sum_{n>=1} lambda_{n+1} t_n^T,
 * with t_n = T_n(A) psi recomputed from checkpoints every checkpoint_stride
 * moments (0: ceil(sqrt(n_moments))), and df/dH = df/dA / half_width
 * sampled on H's pattern.  Orthogonal form, real H (F64 or F32) and real
 * psi (device N x n_vectors, the same precision); dmu: host, n_moments.
 * mu_out (host, may be NULL) receives the moments of the forward pass;
 * grad_values (device, FP64, nnz_blocks * b * b in the layout of H's
 * values) is overwritten.  Bounds are held fixed.  Synchronises the stream. */
RSATB_API int rsatb_kpm_moments_vjp(rsatb_ctx_t ctx, const rsatb_cheb_op* op, const void* psi,
                                    int n_vectors, rsatb_dtype vec_dtype, int n_moments,
                                    const double* dmu, int checkpoint_stride, double* mu_out,
                                    double* grad_values, rsatb_adjoint_stats* stats);

/* The same VJP for the sandwich form A = (Z^T H Z - center) / half_width
 * (real symmetric H, Z the graph-local S^-1/2 and ZH = Z^T, every matrix
 * and psi of one precision): with G = df/dA,
 *     grad_h = Z G Z^T / half_width   on H's pattern,
 *     grad_z = H Z (G + G^T) / half_width   on Z's pattern
 * (device, FP64, in the layouts of H's and Z's values; overwritten).  The
 * gradient with respect to S follows from grad_z through each row's local
 * inverse square root (rsatb_b200.adjoint.kpm_moments_vjp_sandwich).  No
 * counterpart in the reference.  Synchronises the stream. */
RSATB_API int rsatb_kpm_moments_vjp_sandwich(rsatb_ctx_t ctx, const rsatb_cheb_op* op,
                                             const void* psi, int n_vectors,
                                             rsatb_dtype vec_dtype, int n_moments,
                                             const double* dmu, int checkpoint_stride,
                                             double* mu_out, double* grad_h, double* grad_z,
                                             rsatb_adjoint_stats* stats);

/* ------------------------------------------------ FFT-Chebyshev transport */

/* Counters of one rsatb_dc_spectrum_fftcheb call. */
typedef struct {
    int sections;             /* row sections (the recurrence runs once per section) */
    int64_t fft_chunks;       /* row chunks of the transform stage */
    double recurrence_ms;     /* device time of the recurrences and stores */
    double transform_ms;      /* device time of the DCT-III and contraction stage */
    size_t store_bytes;       /* bytes of the moment stores of one section */
} rsatb_fftcheb_stats;

/* Kubo-Greenwood DC conductivity by the FFT-Chebyshev method,
 * rsatb::calc::dc_spectrum_fftcheb (rsatb/calc/fftcheb_transport.hpp:
 * 543-660) with accumulate_fftcheb_block (:270-525) for one block of all
 * n_vectors samples: left chain J_a T_m(Op~) psi and right chains
 * T_m(Op~) J_a psi, J_a = -(1/(2 half_width)) V_a (current, rsatb/calc/
 * ac.hpp:35-60; dressed as Z^H V_a Z in the Sandwich form), the DCT-III of
 * (g_m/pi) x_m per row, axis and sample (fft.hpp:125-154), and
 * K(E_k) = sum conj(L3) R3 / max(1e-14, 1 - eps_k^2), averaged over the
 * samples.  Vx, Vy, Vz: velocity matrices (RSATB_BSR_IMAGINARY_UNIT for the
 * i*W of a real k-point, or complex), H's shape and precision.  psi: device
 * N x n_vectors complex (C128, or C64 for FP32 vectors; the transform and
 * the contraction are FP64 either way).  formulation 0 Greenwood, 1
 * Bastin: beside phi3 the zero-padded 2M-point inverse FFTs phi1, phi2 of
 * the moments times the complex phase weights (:443-461), all six (a, b)
 * components of eps (conj(L3_a) R1_b + conj(L1_a) R3_b) + i sqrt(1 - eps^2)
 * (conj(L2_a) R3_b - conj(L3_a) R2_b) (:496-519), then the cumulative
 * trapezoid of Re(i zeta) over the ascending grid: sigma(mu, T = 0)
 * (:635-659).  partition_sections > 0 asks for at least that many row sections,
 * max_workspace_bytes bounds the device memory (0: 80 % of what is free).
 * sigma_out (host) receives n_moments x 6 (xx xy xz yy yz zz; Greenwood
 * fills xx, yy, zz) scaled by prefactor, energy_out (host) the ascending
 * energies c + hw cos(pi (M - 1 - k + 1/2) / M).  stats may be NULL.
 * Synchronises the context's stream. */
RSATB_API int rsatb_dc_spectrum_fftcheb(rsatb_ctx_t ctx, const rsatb_cheb_op* op,
                                        rsatb_bsr_t Vx, rsatb_bsr_t Vy, rsatb_bsr_t Vz,
                                        const void* psi, int n_vectors, rsatb_dtype vec_dtype,
                                        int n_moments, int formulation, double prefactor,
                                        int partition_sections, size_t max_workspace_bytes,
                                        int kernel, double* sigma_out, double* energy_out,
                                        rsatb_fftcheb_stats* stats);

/* Quasi-eigenstate Greenwood spectrum, rsatb::calc::dc_spectrum_qe
 * (rsatb/calc/fftcheb_transport.hpp:662-884): the fftcheb Greenwood
 * bilinear form evaluated at a window of grid nodes only, with no row store
 * and no row transform.  The right chains T_m(Op) J_b psi and the left
 * J_a T_m(Op) psi are summed into per-node vectors with the node weights
 * (g_m / pi)(2 - [m = 0]) T_m(e_j) in batches of moments, and each node's
 * value is one dot of its two vectors over rows and samples.  nodes (host,
 * n_nodes, may be NULL with n_nodes = 0 for every node) index the
 * ascending output grid; out-of-range indices are RSATB_INVALID_ARGUMENT.
 * sigma_out (n_moments x 6, zero outside the window: xx, yy, zz filled)
 * and energy_out (n_moments, ascending) as for rsatb_dc_spectrum_fftcheb.
 * Memory: two FP64 vectors of 3 x N x R complex per node.  Synchronises. */
RSATB_API int rsatb_dc_spectrum_qe(rsatb_ctx_t ctx, const rsatb_cheb_op* op, rsatb_bsr_t Vx,
                                   rsatb_bsr_t Vy, rsatb_bsr_t Vz, const void* psi,
                                   int n_vectors, rsatb_dtype vec_dtype, int n_moments,
                                   double prefactor, int kernel, const int32_t* nodes,
                                   int n_nodes, double* sigma_out, double* energy_out);

/* ------------------------------------------- batched dense inverse square root */

/* Arithmetic of the batched Newton-Schulz solve. */
typedef enum {
    RSATB_NS_FP64 = 0,     /* every iteration in FP64 */
    RSATB_NS_TF32X3 = 1,   /* tensor-core phase in split TF32 (hi*hi + hi*lo + lo*hi, FP32
                              accumulation in TMEM), then FP64 refinement iterations */
    RSATB_NS_TF32 = 2      /* tensor-core phase in plain TF32, then FP64 refinement */
} rsatb_ns_precision;

/* Options of rsatb_isqrt_columns_batched.  Zero fields take the defaults in
 * brackets. */
typedef struct {
    int precision;          /* rsatb_ns_precision [RSATB_NS_FP64 when zero] */
    int max_iter;           /* iterations of the tensor-core phase [30] */
    int max_fp64_iter;      /* FP64 iterations [6 after a tensor-core phase, 60 alone] */
    double tol;             /* stop when ||X - I||_F <= tol, X = Z S Z^T [1e-11] */
    double accept;          /* a problem whose final ||X - I||_F exceeds this is reported
                               RSATB_NUMERICAL_FAILURE [1e-6] */
    size_t workspace_bytes; /* device workspace per chunk of problems [8 GiB] */
    int no_graph;           /* 0: each chunk's iterations run as one captured CUDA graph */
    int tc_kernel;          /* tensor-core GEMM: 0 the built-in choice, 1 warp-specialised
                               (N tile <= 128), 2 single-role (N tile <= 256) */
    int n_tiles;            /* entries of the N-tile table (0: the built-in rule, the fewest
                               tiles of at most the kernel's widest N tile) */
    const int32_t* tile_n_pad; /* host: padded sizes (multiples of 32) of the table */
    const int32_t* tile_nt;    /* host: the N tile (multiple of 16) for each padded size;
                                  sizes absent from the table take the built-in rule */
} rsatb_isqrt_options;

/* Per-call statistics (host). */
typedef struct {
    int chunks;               /* chunks of problems the workspace allowed */
    int low_iterations;       /* tensor-core iterations run (max over problems) */
    int fp64_iterations;      /* FP64 iterations run (max over problems) */
    int n_failed;             /* problems whose status is not RSATB_SUCCESS */
    double max_residual;      /* max over problems of the final ||X - I||_F */
    double low_flops;         /* FLOPs the tensor-core tiles executed (2 M N K per product,
                                 padding included) */
    double fp64_flops;        /* FLOPs of the FP64 GEMMs (2 n^3 per product) */
    double useful_flops;      /* 8 n^3 per problem per iteration, both phases */
    int64_t gemm_launches;    /* GEMM kernel launches */
    double low_ms, fp64_ms;   /* device time of the two phases (CUDA events), all chunks */
} rsatb_isqrt_stats;

/* Columns [col_start, col_start + k_cols) of M^{-1/2} for a batch of
 * symmetric positive definite matrices: the per-subgraph action of
 * rsatb::calc::isqrt::inverse_sqrt_columns_inplace
 * (rsatb/calc/isqrt_action.hpp:1343-1422) as called by graph_inverse_sqrt
 * (rsatb/calc/isqrtm.hpp:149-232), for all subgraphs in one call.
 *
 * Problem p: n[p] x n[p] matrix at M + in_offset[p] (device, FP64,
 * column-major, only the upper triangle is read, as with the reference's
 * uplo 'U'); its result, n[p] x k_cols[p] column-major, goes to
 * out + out_offset[p] (device).  n, col_start, k_cols, in_offset and
 * out_offset are host arrays.  k_cols[p] <= 0 means all n[p] columns.
 *
 * Method: the Newton-Schulz iteration of rsatb::calc::inverse_sqrt
 * (rsatb/calc/isqrtm.hpp:620-807), X = Z S Z^T, P = 1.875 I - 1.25 X +
 * 0.375 X^2, Z <- P Z, from Z0 = I / sqrt(s) with s the Gershgorin bound
 * of lambda_max, stopped per problem by the reference's rules (tolerance,
 * 0.5 % plateau, iteration cap, divergence above 100); dense, per problem,
 * 1 <= n <= 1024.  The result is (Z + Z^T)/2 of the last iterate.
 *
 * status (host, may be NULL) receives one rsatb_status per problem
 * (RSATB_DIVERGED, or RSATB_NUMERICAL_FAILURE when the final residual
 * exceeds `accept`); the call itself fails only for invalid arguments or
 * device errors.  Synchronises the context's stream before returning. */
RSATB_API int rsatb_isqrt_columns_batched(rsatb_ctx_t ctx, int n_problems, const int32_t* n,
                                          const int32_t* col_start, const int32_t* k_cols,
                                          const int64_t* in_offset, const double* M,
                                          const int64_t* out_offset, double* out,
                                          const rsatb_isqrt_options* options, int32_t* status,
                                          rsatb_isqrt_stats* stats);

/* Autotuner of the tensor-core tiles of rsatb_isqrt_columns_batched.  For
 * each size in sizes[n_sizes] it builds problems_per_size well-conditioned
 * SPD matrices of that size on the device, times (CUDA events, best of two
 * after a warm-up) a fixed-length solve in `precision` (RSATB_NS_TF32X3 or
 * RSATB_NS_TF32) for each candidate: both tensor-core kernels, and for each
 * the N tiles that split the padded size into the fewest tiles of at most
 * 32, 64, 128 (and 256 for the single-role kernel) columns.  It returns the
 * kernel with the smallest summed time (*tc_kernel_out, 1 or 2) and, for
 * that kernel, the fastest N tile per size (nt_out[n_sizes]), which go into
 * rsatb_isqrt_options.tc_kernel / tile_n_pad / tile_nt.  ms_out (optional,
 * n_sizes x 8) receives every candidate's time: [size][kernel 0..1][tile
 * 0..3], -1 where the candidate does not exist. */
RSATB_API int rsatb_isqrt_autotune(rsatb_ctx_t ctx, int precision, int n_sizes,
                                   const int32_t* sizes, int problems_per_size,
                                   int* tc_kernel_out, int32_t* nt_out, double* ms_out);

/* Options of the global sparse Newton-Schulz refinement,
 * rsatb::calc::InverseSqrtOptions (rsatb/calc/isqrtm.hpp:235-240) plus the
 * route rule. */
typedef struct {
    double tol;    /* stop when max block ||(Z^H S Z - I)[i,j]||_F <= tol (1e-7) */
    double sptol;  /* Frobenius drop threshold of every product (1e-6); 0 keeps all */
    int maxit;     /* Newton-Schulz steps at most (20); 0 returns the seed */
    int route;     /* 0: advance X by P X P when cheaper (every 5th step and
                    * residuals >= 0.1 reform); 1: always reform X = Z^H S Z */
} rsatb_ns_refine_options;

/* What the refinement did, rsatb::calc::InverseSqrtReport (isqrtm.hpp:
 * 243-258), plus the final factor's size. */
typedef struct {
    int steps;
    int converged;             /* the loop residual reached tol */
    int hit_maxiter;
    int diverged;              /* residual above 100: the iteration left its radius */
    int last_advance_propagated;
    double residual;           /* loop metric: max block Frobenius of X - I */
    double applied_residual;   /* ||(Z^H S Z - I) v|| on a unit random probe */
    int64_t nnz_blocks;        /* blocks of the returned factor */
    int reforms, propagations; /* how X was advanced */
} rsatb_ns_refine_report;

/* S^-1/2 refined from a seed Z (the graph-local factor) by the cubic
 * Newton-Schulz purification of rsatb::calc::inverse_sqrt (rsatb/calc/
 * isqrtm.hpp:262-900): X = Z^H S Z, P = 1.875 I - 1.25 X + 0.375 X^2,
 * Z <- Z P, every product a block SpGEMM on the device whose blocks of
 * Frobenius norm below sptol are dropped; X advanced by reformation or by
 * P X P; stops on tol, a plateau (|norm_prev - norm| <= 0.005 norm), maxit or
 * divergence.  S and Z_seed: F64 BSR with equal block size (at most 8)
 * and rows.
 * *Z_out receives a new matrix (its pattern grows with the products).
 * report (may be NULL) as above.  Synchronises. */
RSATB_API int rsatb_inverse_sqrt_refine(rsatb_ctx_t ctx, rsatb_bsr_t S, rsatb_bsr_t Z_seed,
                                        const rsatb_ns_refine_options* options,
                                        rsatb_bsr_t* Z_out, rsatb_ns_refine_report* report);

/* ------------------------------------------------------- spectral bounds */

/* Options of rsatb_lanczos_extremes; zero fields take the defaults. */
typedef struct {
    int steps;          /* fixed Lanczos steps when tol <= 0 (0: 20) */
    double tol;         /* > 0: stop once both extreme Ritz pairs have residual
                           <= tol * max|theta| (PRIMME's 1e-3 in the reference) */
    int max_matvecs;    /* cap with tol (0: 10000); at most 400 basis vectors */
    uint64_t seed;      /* start vector of rsatb_set_random (0: 2) */
} rsatb_lanczos_options;

typedef struct {
    double theta_min, theta_max;  /* extreme Ritz values of the unscaled operator */
    double res_min, res_max;      /* their residual norms |beta_m y_m| */
    int matvecs;                  /* operator applications */
    int converged;                /* tol met (or an invariant subspace found) */
} rsatb_lanczos_result;

/* Extreme eigenvalues of the operator of `op` applied unscaled (its window is
 * ignored): Lanczos with full FP64 reorthogonalisation on the device, the
 * basis S-orthonormal for the Solve form (H x = lambda S x), the tridiagonal
 * eigenproblem on the host (implicit QL).  The spectral-bounds estimate of
 * rsatb/setup/spectral_bounds.hpp:311-490 (ExtremalEigenvalues) without
 * PRIMME; the caller pads and applies the fallback rules.  Allocates its
 * basis (n x m FP64) with cudaMalloc and frees it; synchronises. */
RSATB_API int rsatb_lanczos_extremes(rsatb_ctx_t ctx, const rsatb_cheb_op* op,
                                     const rsatb_lanczos_options* options,
                                     rsatb_lanczos_result* result);

/* Eigenvalues (ascending) of the symmetric tridiagonal matrix diag[0..m),
 * off[0..m-1) and the last components of its normalised eigenvectors (host
 * only; the Ritz solve of rsatb_lanczos_extremes). */
RSATB_API int rsatb_tridiag_eigen(int m, const double* diag, const double* off,
                                  double* eigenvalues, double* last_components);

/* ------------------------------------------------------------ measurement */

/* FMA-pipe throughput of this device in FLOP/s, from independent FMA chains
 * on every SM timed with CUDA events: the compute roofline of the block SpMM
 * at wide panels.  double_precision: 1 FP64, 0 FP32 (scalar FMAs), 2 FP32
 * issued as packed pairs (fma.rn.f32x2), 3 FP64 on the tensor cores
 * (mma.sync m8n8k4 f64 tiles), 4 TF32 on the tensor cores (mma.sync m16n8k8
 * tf32 tiles, FP32 accumulation). */
RSATB_API int rsatb_measure_fma_peak(rsatb_ctx_t ctx, int double_precision, double* flops);

#ifdef __cplusplus
}
#endif

#endif /* RSATB_B200_H */
