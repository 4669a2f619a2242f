/*
 * fastctqw_b200 — C ABI of the B200 expm(-iHt) engine.
 *
 * Plain C types only (pointers, sizes, ints).  Every entry point returns an fx_status;
 * fx_last_error() gives the message of the last failure on a handle (or globally when the
 * handle is NULL).  Matrices are dense, row-major ("C order", as numpy hands them over),
 * interleaved complex (real, imag) in the dtype the handle was created with.  Because
 * expm(A^T) = expm(A)^T, row- vs column-major storage does not change the result as long
 * as input and output use the same order.
 *
 * Reference interfaces replaced (Crinton/FastCTQW):
 *   fx_create  <- MatrixExpCalculator<T>::MatrixExpCalculator(size_t n)
 *                 (include/MatrixExpCalculator.h:36, :64, :92; bound src/main.cu:14-15,
 *                 :27-28, :40-41, :53-54 as ExpMatFloat32/Float64/Complex64/Complex128)
 *   fx_run_host <- MatrixExpCalculator<T>::run(py::array_t<T>&)
 *                 (include/MatrixExpCalculator.h:40, :68, :96; src/main.cu:17-19, :30-32,
 *                 :43-45, :56-58)
 *   fx_free    <- MatrixExpCalculator<T>::free()  (include/MatrixExpCalculator.h:42, :70, :98;
 *                 src/main.cu:21-22)
 *   fx_get_n   <- MatrixExpCalculator<T>::getN()  (include/MatrixExpCalculator.h:41, :69, :97)
 *   fx_destroy <- ~MatrixExpCalculator()          (include/MatrixExpCalculator.h:37, :65, :93)
 *   fx_walk_device / fx_walk_host <- Operator.buildExpmOperator(t) followed by the host
 *                 GEMV U @ psi0 in Ctqw.runWalk (FastCTQW/Operator.py:70-78,
 *                 FastCTQW/Ctqw.py:90-94), kept on the device.
 *   fx_run_device: device-pointer variant of run (no counterpart: the reference always
 *                 copies through host numpy arrays).
 *   fx_gpu_memory_gb <- get_current_gpu_memory_gb() (include/MatrixExpCalculator.h:101)
 */
#ifndef FASTCTQW_B200_H
#define FASTCTQW_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fx_engine* fx_handle;

/* Element types (ExpMatFloat32 / Float64 / Complex64 / Complex128). */
enum fx_dtype { FX_F32 = 0, FX_F64 = 1, FX_C64 = 2, FX_C128 = 3 };

enum fx_status {
  FX_OK = 0,
  FX_ERR_TYPE = 1,      /* bad dtype / handle kind          -> Python TypeError   */
  FX_ERR_VALUE = 2,     /* bad size, shape, option value    -> Python ValueError  */
  FX_ERR_NOMEM = 3,     /* device or host allocation failed -> Python MemoryError.  For
                           tests of that path, the environment variable
                           FX_INJECT_ALLOC_FAIL=k makes the k-th workspace allocation
                           (counted from when the variable took its value) fail this
                           way; no counterpart in the reference */
  FX_ERR_CUDA = 4,      /* CUDA runtime / launch error      -> RuntimeError       */
  FX_ERR_TIMEOUT = 5,   /* a bounded device wait ran out    -> RuntimeError       */
  FX_ERR_NONFINITE = 6, /* NaN/Inf in the input or a norm   -> ValueError         */
  FX_ERR_SINGULAR = 7,  /* exactly singular Pade denominator-> RuntimeError       */
  FX_ERR_NODEV = 8,     /* no sm_100 device                 -> RuntimeError       */
  FX_ERR_FREED = 9      /* handle used after fx_free        -> RuntimeError       */
};

/* Arithmetic forms for the matrix products (fx_set_option(FX_OPT_FORM, ...)). */
enum fx_form {
  FX_FORM_PLAIN = 0,  /* int8 tensor-core products of 5 (FP64 masters) or 4 (FP32)
                         Ozaki slices, exact int32 accumulation; default for complex64.
                         Walk generators: the powers, Pade and solve products split
                         their operands' diagonals off (added in FP64); walks padded to
                         4096 or more, or needing 8 or more squarings, square as three
                         split products Re^2, Im^2, (Re+Im)^2, the others as the exact
                         complex square                                               */
  FX_FORM_MIXED = 1,  /* reduced-precision products (complex64 / float32 handles).  Walk
                         generators X = i*(real symmetric) padded to 4096 or more: int8
                         slices on FP64 masters with the diagonals split off and added in
                         FP64, 4 slices for the powers and (when s <= 10) the Pade and
                         solve products (FX_OPT_PADE_SLICES), the solve by a
                         Newton-Schulz inverse, each squaring as three symmetric products
                         Re^2, Im^2, (Re+Im)^2 at 4 slices (5 for squarings before the
                         last FX_OPT_SQ_N4, 3 for the last FX_OPT_SQ_N3).  Smaller walk
                         generators take the plain form's schedule.
                         Other inputs: BF16 hi+lo split, 3 products (hi*hi, hi*lo,
                         lo*hi), FP32 accumulate, FP32 masters                        */
  FX_FORM_SIMT = 2,   /* CUDA-core FP32 FMA products, FP32 masters (checker)          */
  FX_FORM_FP64 = 3    /* CUDA-core FP64 products (default for complex128 / float64)   */
};

enum fx_option {
  FX_OPT_FORM = 0,        /* fx_form                                                   */
  FX_OPT_SHIFT = 1,       /* 0 none, 1 trace, 2 trace + rank-one (default 2)           */
  FX_OPT_STRUCTURE = 2,   /* 1: exploit X = i*(real symmetric) structure (default 1)   */
  FX_OPT_FORCE_S = 3,     /* >= 0: override the scaling s (with FX_OPT_FORCE_M)        */
  FX_OPT_FORCE_M = 4,     /* 3, 5, 7, 9, 13 or -1 (automatic)                          */
  FX_OPT_TIMEOUT_MS = 5,  /* bound of every device-side wait (default 2000)            */
  FX_OPT_IPE = 6,         /* 1: square in I+E form (default 1)                         */
  FX_OPT_REFINE = 7,      /* iterative-refinement steps of the Pade solve (default 0)  */
  FX_OPT_DEBUG_STAGE = 8, /* diagnostics: k > 0 makes run write intermediate k instead of
                             U (1 Y, 2-4 A2/A4/A6, 5 U_pade, 6 V_pade, 7 R, 8+j after j
                             squarings) and stop                                       */
  FX_OPT_PROFILE = 9,     /* 1: CUDA-event timing of every tensor-core product launch
                             (fx_stats.prod_*)                                         */
  FX_OPT_SELECTOR = 10,   /* (m, s) selection for walk generators X = i*(real symmetric):
                             0 Al-Mohy & Higham (default), 1 the cheapest (m, s) the
                             truncation bound certifies at phase error 1e-6 from the
                             rigorous spectral bound min(||Y||_1, d4, d6), 2 the learned
                             MLP proposal, used when it is cheaper than option 3's choice,
                             the phase bound at min(rigorous bound, 1.1 x the Lanczos
                             estimate) stays below 1e-5 (infidelity <= 1e-10 for every
                             state) and the result passes the a-posteriori checks (else
                             option 3), 3 the same phase bound at a Lanczos estimate of the
                             spectral radius (30 steps, two starts) raised by 10%, at 1e-6
                             (estimated selection)                                     */
  FX_OPT_INJECT_STALL = 11, /* diagnostics of the failure path (walk generators): k >= 0 makes
                             the k-th product launch of every run leave out the operand
                             loads of one K step, so that its bounded waits run out and
                             the run returns FX_ERR_TIMEOUT; -1 (default) off          */
  FX_OPT_SQ_N4 = 12,      /* mixed form, walk generators: how many squarings before the
                             3-slice ones run at 4 slices (default 8; the earlier ones,
                             whose errors later squarings amplify most, run at 5)      */
  FX_OPT_SQ_N3 = 13,      /* mixed form, walk generators: how many of the last squarings run
                             at 3 slices (default 0)                                   */
  FX_OPT_DRIFT = 14,      /* diagnostics (walk generators): 1 records the unitarity residual
                             ||U_k^H U_k - I||_F / sqrt(n) after every squaring k = 0..s
                             (fx_unitarity_drift), at the cost of two extra products per
                             squaring                                                  */
  FX_OPT_PADE_SLICES = 15, /* mixed form, walk generators: int8 slices of the powers, Pade and
                             solve products (4 default, 5 or 3; the Pade and solve
                             products take 5 when the selection needs more than 10
                             squarings)                                                */
  FX_OPT_NEWTON_SLICES = 16, /* walk generators: int8 slices of the Newton-Schulz steps of
                             the solve whose model residual stays above 1e-4 (3 default,
                             4 or 5; the later steps take the Pade products' count: the
                             iteration corrects the early steps' rounding)             */
  FX_OPT_SOLVE = 17,      /* walk generators: solve of the Pade step R = G^-1 P^2 (G SPD):
                             0 (default) Newton-Schulz for walks padded to 4096 or more,
                             blocked Cholesky otherwise; 1 Cholesky; 2 Newton-Schulz  */
  FX_OPT_APPROX = 18      /* walk generators X = iB: approximant of exp(X / 2^s) before the
                             squarings.  0 (default) the [m/m] Pade approximant and its
                             solve; 1 the Chebyshev-Bessel polynomial sum_k (2 - [k=0])
                             i^k J_k(a) T_k(B / rho), a = rho / 2^s, evaluated with
                             products of commuting real symmetric matrices only (no
                             solve); rho is the rigorous spectral bound min(||Y||_1, d4,
                             d6), or for the estimated and learned selections
                             min(that, 1.25 x the Lanczos estimate); (s, degree) are the
                             cheapest plan of fx_chebyshev_plan at error 1e-6 (1e-12 for
                             complex128 walks).  Reported
                             as m = 0, solver 3, fx_stats.degree, sel_outcome 5.  No
                             counterpart in the reference                             */
};

/* What the last run did. */
typedef struct fx_stats {
  int32_t m;            /* Pade degree                                   */
  int32_t s;            /* number of squarings                           */
  int32_t form;         /* fx_form used for the products                 */
  int32_t structured;   /* 1 if the X = i*(real symmetric) path was used */
  int32_t rank1_shift;  /* 1 if the rank-one commuting shift was applied */
  int32_t symmetric;    /* 1 if X^T == X (no transposes needed)          */
  int32_t gemm_launches;/* matrix-product kernel launches in the run     */
  int32_t launches;     /* all kernel launches of the run                */
  int32_t solver;       /* 0 pivoted LU, 1 Cholesky of Q^H Q (normal Q), 2 Newton-Schulz
                           inverse of Q^H Q, 3 none (Chebyshev polynomial, FX_OPT_APPROX) */
  int32_t degree;       /* degree of the Chebyshev polynomial (FX_OPT_APPROX = 1), else 0  */
  double norm1;         /* ||X - shifts||_1                              */
  double d[5];          /* d4, d6, d8, d10, log2 ||(|A|)^27||_1          */
  double ms_total;      /* device time of the last run (CUDA events)     */
  double flops;         /* algorithmic real flops of the last run        */
  double prod_ms;       /* summed duration of the int8 product launches  */
  double prod_ops;      /* int8 tensor ops they issued                   */
  double prod_flops;    /* real-arithmetic flops they computed           */
  int32_t prod_launches;
  int32_t reserved2;
  int32_t selector;     /* FX_OPT_SELECTOR of the run                                  */
  int32_t sel_outcome;  /* 0 plain, 1 certified, 2 learned accepted, 3 estimated (also a
                           learned proposal that was rejected or not cheaper), -1 learned
                           rejected by the bound with no estimated choice cheaper than plain, -2 failed an a-posteriori check
                           (Cholesky of Q^H Q or unitarity) and was redone with the plain
                           (m, s)                                                   */
  int32_t plain_m;      /* (m, s) of the Al-Mohy & Higham selection                    */
  int32_t plain_s;
} fx_stats;

int fx_create(size_t n, int dtype, fx_handle* out);
int fx_destroy(fx_handle h);
int fx_free(fx_handle h);
int fx_get_n(fx_handle h, size_t* n);
int fx_set_option(fx_handle h, int key, double value);
int fx_get_stats(fx_handle h, fx_stats* out);
const char* fx_last_error(fx_handle h);

/* Per product launch of the last run made with FX_OPT_PROFILE = 1 through the walk-generator
 * pipeline: its stage (0 powers, 1 Pade numerator / denominator, 2 the solve's V^2, W^2, VW,
 * 3 Cholesky, 4 triangular inverse, 5 triangular products, 6 squarings, 7 diagnostic unitarity
 * products, 8 Newton-Schulz inverse of the solve), its CUDA-event duration in ms and the int8
 * tensor ops it issued; then four timeline records of the whole run (ops 0): 9 phase 1, 10 the
 * gap between the phases (read-back, selection, graph launch), 11 phase 2, 12 the checks after
 * it.  Writes min(cap, records) records and the record count to *count (0 when no such run was
 * profiled).  Diagnostics; no counterpart in the reference. */
int fx_product_profile(fx_handle h, int32_t* tags, double* ms, double* ops, int32_t cap, int32_t* count);

/* The unitarity residuals of the last run made with FX_OPT_DRIFT = 1: out[k] =
 * ||U_k^H U_k - I||_F / sqrt(n) for the iterate U_k = I + E_k after k squarings (k = 0: the
 * Pade approximant of the scaled generator; k = s: the propagator before the shifts, which are
 * unitary), computed from exact-in-int32 products on 5 slices.  Writes min(cap, s + 1) values
 * and s + 1 to *count (0 when no such run was made).  Diagnostics; no counterpart in the
 * reference. */
int fx_unitarity_drift(fx_handle h, double* out, int32_t cap, int32_t* count);
/* Spectral-radius estimates of the shifted generator of the last walk-generator run: a Lanczos
 * estimate (30 steps from two pseudo-random starts; Ritz values lie inside the spectrum, so it
 * does not exceed the radius) and the rigorous upper bound min(||Y||_1, d4, d6).  The Lanczos
 * estimate runs only where it is used (the learned and estimated selections, the mixed form);
 * elsewhere *rho_lanczos is 0.  Diagnostics of the (m, s) selection; no counterpart in the
 * reference. */
int fx_spectral_radius(fx_handle h, double* rho_lanczos, double* rho_up);

/* U = expm(A), both host buffers of n*n elements of the handle's dtype. */
int fx_run_host(fx_handle h, const void* A, void* U);
/* Same with device buffers; the work is ordered on `stream` (a cudaStream_t or NULL). */
int fx_run_device(fx_handle h, const void* dA, void* dU, void* stream);
/* psi = expm(A) psi0 (and U if dU != NULL); device buffers. */
int fx_walk_device(fx_handle h, const void* dA, const void* dpsi0, void* dpsi, void* dU,
                   void* stream);
/* psi = expm(A) psi0 with host buffers.  U stays resident on the device (not copied back)
 * until fx_fetch_u asks for it. */
int fx_walk_host(fx_handle h, const void* A, const void* psi0, void* psi);
/* Copy the U of the last fx_walk_host call to a host buffer of n*n elements
 * (Operator.getOperator after Ctqw.runWalk, FastCTQW/Operator.py:165-166). */
int fx_fetch_u(fx_handle h, void* U);

/* Diagnostics (no counterpart in the reference): one real product through the engine's
 * product kernels, D = alpha A Bt^T + beta C + gamma I, on device buffers (row-major;
 * Bt is the right factor transposed, N x K).  form: FX_FORM_PLAIN / FX_FORM_MIXED
 * (tcgen05, BF16 split) or FX_FORM_SIMT (CUDA cores).  Allocates its split scratch. */
int fx_product_f32(int form, int64_t M, int64_t N, int64_t K, const float* A, int64_t lda,
                   const float* Bt, int64_t ldb, float alpha, float beta, const float* C,
                   int64_t ldc, float gamma, float* D, int64_t ldd, void* stream);
const char* fx_product_error(void);

/* Diagnostics (no counterpart in the reference): the grouped int8 slicer of the product kernels
 * on one block of `rows` rows of FP64 planes (device buffers, row pitch ld elements).  Each row
 * is scaled by 2^(7S - e), e its exponent (as the products use it), and cut into S signed
 * digits from the top with round-half-even.  kind 0: warp-per-row kernel, 1: the two passes the
 * products use (row exponents by a warp per row, then the digits over a block plan of the rows'
 * elements); both give the same digits.  im may be null; split_diag (single plane, dg non-null) leaves row
 * r's element at column r out of the slices and writes it to dg[r]; neg (im non-null) also
 * writes the digits of -im.  out: 3 S planes of rows x ldo bytes (re digits 0..S-1, im, -im;
 * ldo >= K, a multiple of 16), exps: rows int32.  Messages through fx_product_error. */
int fx_slice_rows_f64(int kind, int S, const double* re, const double* im, int64_t ld, int64_t rows,
                      int64_t K, int split_diag, int neg, int8_t* out, int64_t ldo, int32_t* exps,
                      double* dg, void* stream);

/* Measured dense tensor-core rate of the current GPU (diagnostics; no counterpart in the
 * reference): one CTA per SM issues `iters` (1..2^20) x 2 tcgen05.mma of M = 128, N = 256, K = 32 bytes
 * (kind 0: int8 x int8 -> int32; kind 1: BF16 x BF16 -> FP32) on operand tiles resident in
 * shared memory, timed with CUDA events on `stream`.  *tops = tensor ops (2 M N K per
 * instruction) per second / 1e12, *ms = the launch's duration.  Messages through
 * fx_product_error. */
int fx_tensor_peak(int kind, int64_t iters, double* tops, double* ms, void* stream);

/* Allocation-free form of fx_product_f32 with FX_FORM_PLAIN (4 int8 slices, exact int32
 * accumulation on the tensor cores); no counterpart in the reference.  For callers that must
 * not allocate device memory once they are running (a pool that owns the device, an
 * allocator callback, a host that sizes all GPU memory at start-up): the slice scratch lives
 * in one fixed 16 MiB array of device memory inside the library, present on every GPU that
 * loads it until the process exits.  Needs 4 (M + N) K + 4 (M + N) + 512 bytes of it (M, N
 * multiples of 16, K of 64 and at most 32768) and returns FX_ERR_VALUE beyond that.  The first
 * call on a device looks the array's device address up (make it before any stream capture).
 * All calls share the array: calls that overlap on the GPU race; order them on one stream.
 * Each call synchronises its stream before it returns (it reads the kernel's error word back).
 * Messages through fx_product_error. */
int fx_product_f32_noalloc(int64_t M, int64_t N, int64_t K, const float* A, int64_t lda,
                           const float* Bt, int64_t ldb, float alpha, float beta, const float* C,
                           int64_t ldc, float gamma, float* D, int64_t ldd, void* stream);

/* ---- Batched walks: many independent walks of uneven sizes in grouped launches.
 * No counterpart in the reference (it ran one matrix per MatrixExpCalculator object,
 * include/MatrixExpCalculator.h:17-103, one walk per Ctqw.runWalk, FastCTQW/Ctqw.py:90-94);
 * this is the batched form of fx_walk_device for walk generators X_w = i*(real symmetric)
 * (X = -iHt with real symmetric H).  Every phase of the pipeline is one grouped launch over
 * all walks (tensor-core products over a tile list spanning the walks, one-CTA-per-walk
 * Cholesky blocks and 1-norm estimates); everything after the (m, s) selection is replayed
 * as one CUDA graph.  Products: int8 Ozaki slices on FP64 masters (the plain form). */
typedef struct fx_batch* fx_batch_handle;
enum fx_batch_option {
  FX_BATCH_OPT_GRAPH = 0,       /* 1 (default): replay the post-selection phases as a CUDA graph */
  FX_BATCH_OPT_TIMEOUT_MS = 1,  /* bound of every device-side wait (default 2000)               */
  FX_BATCH_OPT_FORCE_M = 2,     /* diagnostics: force the Pade degree (-1 automatic)            */
  FX_BATCH_OPT_SELECTOR = 3,    /* as FX_OPT_SELECTOR                                           */
  FX_BATCH_OPT_ANALYZE_ONLY = 4, /* 1: stop after the selection (features and (m, s) only)      */
  FX_BATCH_OPT_DIAG_SPLIT = 5,   /* mask, default 7: products that take their operands'          */
                                 /* diagonals out of the int8 slices and add those terms in     */
                                 /* FP64; 1 the real products (V^2, W^2, VW; all of the mixed   */
                                 /* form's), 2 P2 L^-T and Z L^-1, 4 the plain form's powers     */
                                 /* and Pade products, 8 the plain form's squarings as three   */
                                 /* split products Re^2, Im^2, (Re+Im)^2 (as the mixed form's)  */
  FX_BATCH_OPT_AUTOTUNE = 6,     /* 1: at the next run, time the candidate schedules of the     */
                                 /* post-selection products on this batch and keep the fastest */
  FX_BATCH_OPT_TILE_GROUP = 7,   /* schedule: tiles in G x G blocks, G = 4, 8 (default) or 16    */
  FX_BATCH_OPT_TILE_ORDER = 8,   /* schedule: 0 (default) longest K ranges first, 1 by problem   */
  FX_BATCH_OPT_SAMPLE_WALKS = 9, /* walks (default 2, 0..64) of a non-plain selection re-run with */
                                 /* the plain (m, s) and compared after every run               */
  FX_BATCH_OPT_FORM = 10,        /* FX_FORM_PLAIN (default) or FX_FORM_MIXED (as FX_OPT_FORM)     */
  FX_BATCH_OPT_SQ_N4 = 11,       /* mixed form: squarings at 4 slices (as FX_OPT_SQ_N4)          */
  FX_BATCH_OPT_SQ_N3 = 12,       /* mixed form: last squarings at 3 slices (as FX_OPT_SQ_N3)     */
  FX_BATCH_OPT_DRIFT = 13,       /* diagnostics: per-squaring unitarity residual (as FX_OPT_DRIFT) */
  FX_BATCH_OPT_PADE_SLICES = 14, /* mixed form: slices of the Pade and solve products (as        */
                                 /* FX_OPT_PADE_SLICES)                                         */
  FX_BATCH_OPT_NEWTON_SLICES = 15, /* mixed form: slices of the early Newton-Schulz steps (as    */
                                  /* FX_OPT_NEWTON_SLICES)                                      */
  FX_BATCH_OPT_SOLVE = 16,        /* solve of the Pade step (as FX_OPT_SOLVE)                   */
  FX_BATCH_OPT_APPROX = 17        /* approximant: 0 Pade, 1 Chebyshev polynomial (as           */
                                  /* FX_OPT_APPROX)                                             */
};
/* count walks of sizes n[0..count); dtype FX_C64 or FX_C128 (of X, psi0 and psi). */
int fx_batch_create(size_t count, const int64_t* n, int dtype, fx_batch_handle* out);
int fx_batch_destroy(fx_batch_handle b);
int fx_batch_set_option(fx_batch_handle b, int key, double value);
/* psi_w = expm(X_w) psi0_w for all walks; arrays of `count` device pointers (X_w: n_w x n_w
 * row-major interleaved complex; psi0_w, psi_w: n_w). */
int fx_batch_walk_device(fx_batch_handle b, const void* const* dX, const void* const* dpsi0,
                         void* const* dpsi, void* stream);
/* The same with host buffers (copies in and out inside the call). */
int fx_batch_walk_host(fx_batch_handle b, const void* const* X, const void* const* psi0,
                       void* const* psi);
/* Unitarity residuals of walk w in the last run made with FX_BATCH_OPT_DRIFT = 1 (as
 * fx_unitarity_drift). */
int fx_batch_drift(fx_batch_handle b, int64_t w, double* out, int32_t cap, int32_t* count);
/* Per-walk forced (m, s) for the following runs (arrays of `count`; m[w] <= 0 leaves walk w to
 * the selector; m NULL clears): measured (m, s, error) sweeps for the learned selector's labels.
 * Forced walks report outcome 4.  No counterpart in the reference. */
int fx_batch_force_selection(fx_batch_handle b, const int32_t* m, const int32_t* s);
/* Per walk of the last run (arrays of `count`): the Lanczos spectral-radius estimate and the
 * rigorous bound (as fx_spectral_radius). */
int fx_batch_spectral(fx_batch_handle b, double* rho_lanczos, double* rho_up);
/* The plan of the Chebyshev approximant (FX_OPT_APPROX = 1) for a spectral bound rho >= 0 of B
 * and an error bound tol > 0 after the squarings: the number of squarings s, the degree D of
 * the polynomial in B / rho (its truncation error 2 sum_{k>D} |J_k(rho / 2^s)| <= tol / 2^s),
 * the baby steps m (T_1..T_m of C = 2 (B / rho)^2 - I) and the matrix products of the whole
 * walk (3 per squaring), the cheapest such plan; host arithmetic only, no device needed.  No
 * counterpart in the reference. */
int fx_chebyshev_plan(double rho, double tol, int32_t* s, int32_t* degree, int32_t* baby, int32_t* cost);
/* (m, s) chosen for every walk by the last run (arrays of `count`; m = 0: Chebyshev). */
int fx_batch_selection(fx_batch_handle b, int32_t* m, int32_t* s);
/* Device time (ms, CUDA events), algorithmic flops and kernel launches of the last run. */
int fx_batch_info(fx_batch_handle b, double* ms, double* flops, int32_t* launches);
/* Per walk of the last run: the 8 selector features (features[8 w ..]: log2 n, log2 ||Y||_1,
 * log2 (||X||_F / sqrt n), log2 (1 + max off-diagonal nonzeros of a row), log2 (Lanczos spectral radius),
 * rank-one shift flag, log2 d4, log2 d6), the Al-Mohy & Higham (m, s), the certified (m, s) and
 * the selection outcome (as fx_stats.sel_outcome). */
int fx_batch_details(fx_batch_handle b, double* features, int32_t* plain_m, int32_t* plain_s,
                     int32_t* cert_m, int32_t* cert_s, int32_t* outcome);
/* Weights of the learned selector for every handle of the process (5126 floats, host
 * pointer; copied to the current device). */
int fx_selector_set_weights(const float* w, int64_t n);
/* Sampled comparison of the last run: how many non-plain walks were re-run with the plain
 * (m, s) (the smallest ones, at most FX_BATCH_OPT_SAMPLE_WALKS, trimmed to a tenth of the
 * batch's N^3 but never below one; 0 when no walk took a non-plain (m, s); -1 when the
 * comparison was skipped because the batch holds a single walk), and the largest infidelity
 * between the two states.  Above 1e-10 every non-plain walk was redone with the plain (m, s)
 * (outcome -2). */
int fx_batch_sample_check(fx_batch_handle b, int32_t* sampled, double* max_infidelity);
/* The phase-2 schedule in use and, after an autotuned run, the candidates tried: ntuned rows
 * of (tile group, tile order, ms) in tuned (3 doubles each, at most 16 rows). */
int fx_batch_schedule(fx_batch_handle b, int32_t* tile_group, int32_t* tile_order, double* tuned,
                      int32_t* ntuned);
const char* fx_batch_last_error(fx_batch_handle b);

/* ---- Learned (m, s) selector: MLP 8 -> 64 -> 64 -> (5 Pade-degree logits + s), ReLU.
 * No counterpart in the reference (its scaling was chosen inside the absent prebuilt core).
 * 5126 FP32 weights in the order W1 [64 x 8], b1, W2 [64 x 64], b2, W3 [6 x 64], b3.
 * All pointers are device pointers.  Inference runs with BF16 weights, FP32 accumulation;
 * training with fused forward/backward kernels and Adam, all on the device. */
int fx_mlp_param_count(void);
/* out[n x 6] = MLP(x[n x 8]). */
int fx_mlp_infer(const float* w, const float* x, int64_t n, float* out, void* stream);
/* Mean loss over the n samples (cross-entropy of the class ym in 0..4 + lambda (s_hat - ys)^2)
 * and its gradient w.r.t. the weights (grad: 5126 floats, loss: 1 float). */
int fx_mlp_loss_grad(const float* w, const float* x, const int32_t* ym, const float* ys, int64_t n,
                     float lambda, float* grad, float* loss, void* stream);
/* Adam training in place of w: `epochs` passes over seeded permutations in minibatches of
 * `batch`; epoch_loss (host, epochs floats, may be NULL) receives the mean loss per epoch. */
int fx_mlp_train(float* w, const float* x, const int32_t* ym, const float* ys, int64_t n, int epochs,
                 int batch, float lr, float lambda, uint64_t seed, float* epoch_loss, void* stream);
const char* fx_mlp_error(void);

/* ---- Device-side set-up and read-out around the propagator (device pointers; stream may be
 * NULL).  These replace O(N^2) host steps of the reference's walk.  No device allocation.
 *
 * X = -1j * H * t for H = -gamma A (laplacian = 0) or -gamma (D - A) (laplacian = 1) of the
 * undirected graph whose m edges are the int64 pairs edges[2k], edges[2k + 1] (repeated edges
 * count once; a self-loop sets A_uu = 1).  Replaces Operator._buildHamiltonian and
 * _buildUnitory (FastCTQW/Operator.py:49-56) on nx.to_numpy_array of the graph
 * (FastCTQW/Ctqw.py:57; Ctqw.from_adjacency_list, FastCTQW/Ctqw.py:60-71, is a stub in the
 * reference).  X: n x n row-major, FX_C64 or FX_C128; entries rounded as numpy rounds those
 * expressions in that dtype.  Synchronises the stream; FX_ERR_VALUE if an endpoint is outside
 * 0..n-1. */
int fx_build_generator(int64_t n, const int64_t* edges, int64_t m, double gamma, int laplacian,
                       double t, int dtype, void* X, void* stream);
/* *hermitian = np.allclose(H, H^H, rtol, atol) for an n x n row-major H of any fx_dtype, in one
 * pass over H (Operator._is_hermitian, FastCTQW/Operator.py:92-103); with skew = 1 the same
 * test of H against -H^H (a walk's X = -iHt is skew-Hermitian exactly when H is Hermitian).
 * Synchronises the stream. */
int fx_check_hermitian(int64_t n, int dtype, const void* H, double rtol, double atol, int skew,
                       int32_t* hermitian, void* stream);
/* psi_out = U psi_in (the GEMV of Ctqw.runWalk, FastCTQW/Ctqw.py:90-94), complex64 or
 * complex128, FP64 accumulation; for stepping a state along a time grid with one U. */
int fx_apply_propagator(int64_t n, int dtype, const void* U, const void* psi_in, void* psi_out,
                        void* stream);
/* prob[k] = |psi[nodes[k]]|^2 in FP64 for k < count, or |psi[k]|^2 for every k < n when nodes is
 * NULL (State.getProbabilities, FastCTQW/State.py:50-51).  A node outside 0..n-1 gives NaN. */
int fx_probabilities(int64_t n, int dtype, const void* psi, const int64_t* nodes, int64_t count,
                     double* prob, void* stream);
const char* fx_graph_error(void);

/* Device memory currently in use on the current device, GB. */
double fx_gpu_memory_gb(void);
/* 1 if a device with compute capability 10.x is present. */
int fx_device_ok(void);
/* Library build string. */
const char* fx_version(void);

#ifdef __cplusplus
}
#endif
#endif /* FASTCTQW_B200_H */
