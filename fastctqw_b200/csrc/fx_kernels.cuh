// Launchers of the bandwidth-bound kernels, the LU kernels and the matrix-product
// kernels (internal header).  All pointers are device pointers; all work is ordered on
// the given stream.  Matrices are planar complex: separate real and imaginary planes,
// row-major with leading dimension `ld`; an imaginary plane of nullptr means "zero".
#pragma once
#include <vector>

#include "fx_common.cuh"

namespace fx {

// ---------------------------------------------------------------- input / structure
// Line sums, trace and exact structure flags of the interleaved input (n x n, row-major,
// element type given by dtype).  row/col: n doubles each (real,imag interleaved => 2n).
struct InputStats {
  double* rowsum;   // 2n (re, im)
  double* colsum;   // 2n
  double* diag;     // 2n (diagonal entries, re/im)
  int* flags;       // [0] any Re != 0, [1] any Im != 0, [2] not symmetric,
                    // [3] not skew-Hermitian, [4] non-finite seen
};
void launch_input_stats(const void* X, int dtype, int64_t n, InputStats st, cudaStream_t s);

// Y = X - mu I - (nu/n) J on the n x n block, zero padding elsewhere, planar T.
template <typename T>
void launch_load_shifted(const void* X, int dtype, int64_t n, int64_t np, double mu_re,
                         double mu_im, double nu_re, double nu_im, T* yre, T* yim,
                         cudaStream_t s);

// --------------------------------------------------------------------------- norms
// colsum[j] += sum_i |M_ij| (double, 2 planes -> complex modulus), columns 0..np-1.
template <typename T>
void launch_col_abs_sums(const T* re, const T* im, int64_t np, int64_t ld, double* colsum,
                         cudaStream_t s);
// Block products for the 1-norm estimator: Y = M X, Z = M^H S with X, S: np x 2 complex
// stored as (re, im) double arrays of length 2*np per column, column-major.
template <typename T>
void launch_matvec2(const T* re, const T* im, int64_t np, const double* X, double* Y,
                    cudaStream_t s);
template <typename T>
void launch_matvec2_h(const T* re, const T* im, int64_t np, const double* S, double* Z,
                      cudaStream_t s);
// w = v |M| (row vector times the entrywise modulus), w zeroed by the launcher.
template <typename T>
void launch_vec_absmat(const T* re, const T* im, int64_t np, const double* v, double* w,
                       cudaStream_t s);

// --------------------------------------------------------------------- elementwise
// D = c0 M0 + c1 M1 + c2 M2 + c3 M3 + g I   (one real plane; null Mk are skipped).
template <typename T>
void launch_combo(T* D, const T* M0, double c0, const T* M1, double c1, const T* M2,
                  double c2, const T* M3, double c3, double g, int64_t np, cudaStream_t s);
// Zero fill of a plane.
template <typename T>
void launch_zero(T* D, int64_t count, cudaStream_t s);
// Out-of-place transpose of an rows x cols block (ld_in / ld_out).
template <typename T>
void launch_transpose(const T* in, int64_t ld_in, T* out, int64_t ld_out, int64_t rows,
                      int64_t cols, cudaStream_t s);
// BF16 split planes of an rows x cols FP32 block: out[p] gets part p (p < nparts); with
// `transpose` the block is written transposed (cols x rows).
void launch_split(const float* in, int64_t ld_in, __nv_bfloat16* const* out, int nparts,
                  int64_t ld_out, int64_t rows, int64_t cols, bool transpose, cudaStream_t s);

// ------------------------------------------------------------------------- output
// U = e^mu (E + ipe*I + rank1 * (e^nu - 1)/n J) on the n x n block -> interleaved dtype.
struct OutputMap {
  double emu_re, emu_im;     // e^mu
  double cj_re, cj_im;       // (e^nu - 1)/n, 0 when no rank-one shift
  int ipe;                   // 1 if E stores R - I
};
template <typename T>
void launch_output(const T* ere, const T* eim, int64_t n, int64_t np, OutputMap om,
                   void* U, int dtype, cudaStream_t s);
// psi = e^mu (E psi0 + ipe psi0 + rank1 * (e^nu-1)/n (1^T psi0) 1), psi0/psi interleaved
// complex of the handle's dtype (complex64 for real handles is not used).
template <typename T>
void launch_apply(const T* ere, const T* eim, int64_t n, int64_t np, OutputMap om,
                  const void* psi0, void* psi, int dtype, double* scratch2, cudaStream_t s);

// ----------------------------------------------------------------------------- LU
// Right-looking panel factorisation with partial pivoting of columns [k0, k0+nb) of the
// planar complex np x np matrix, rows [k0, np).  ipiv[k] = pivot row of column k.
template <typename T>
void launch_lu_panel(T* re, T* im, int64_t np, int64_t k0, int nb, int* ipiv, int* err,
                     cudaStream_t s);
// Apply the row interchanges ipiv[k0..k0+nb) to columns [c0, c1) of a planar matrix.
template <typename T>
void launch_row_swaps(T* re, T* im, int64_t ld, int64_t c0, int64_t c1, const int* ipiv,
                      int64_t k0, int nb, cudaStream_t s);
// In place B <- L^-1 B (L unit lower, nb x nb at (r0, r0) of the factored matrix) for the
// nb x cols block B at rows [r0, r0+nb), columns [c0, c0+cols) of (bre, bim, ldb).
template <typename T>
void launch_trsm_lower_unit(const T* lre, const T* lim, int64_t ldl, int64_t r0, int nb,
                            T* bre, T* bim, int64_t ldb, int64_t c0, int64_t cols,
                            cudaStream_t s);
// In place B <- U^-1 B (U upper non-unit, nb x nb at (r0, r0)).
template <typename T>
void launch_trsm_upper(const T* ure, const T* uim, int64_t ldu, int64_t r0, int nb, T* bre,
                       T* bim, int64_t ldb, int64_t c0, int64_t cols, int* err,
                       cudaStream_t s);

// A <- P A P with P = I - J/n on the n x n block (removes the components along the all-ones
// vector on both sides).  scratch: at least 34 n + 8 doubles.
template <typename T>
void launch_project_ones(T* a, int64_t n, int64_t ld, double* scratch, cudaStream_t s);

// Cholesky diagonal block: G_kk -> L_kk in place, Linv = L_kk^-1, LinvT = L_kk^-T (nb x nb).
template <typename T>
void launch_potrf_inv(T* G, int64_t ld, int64_t k0, int nb, T* Linv, T* LinvT, int* err,
                      cudaStream_t s);

// ----------------------------------------------------------------- matrix products
// D = alpha * sum_t sign_t * A_t * Bt_t^T + beta * C + gamma * I_diag
// A_t: M x K row-major (lda), Bt_t: N x K row-major (ldb) -- i.e. the right factor is
// given transposed, K contiguous, for both operands.  C may alias D.  `diag` adds gamma at
// (i, i) of the M x N block.
template <typename T>
struct GemmTerm {
  const T* a;
  const T* b;
  float sign;
};
template <typename T>
void launch_gemm_simt(int64_t M, int64_t N, int64_t K, const GemmTerm<T>* terms, int nterms,
                      int64_t lda, int64_t ldb, double alpha, double beta, const T* C,
                      int64_t ldc, double gamma, T* D, int64_t ldd, cudaStream_t s);

// tcgen05 (5th-gen tensor core) product on BF16 split planes with FP32 accumulation in
// TMEM.  Each term carries `nplanes` split planes of A and of Bt; the products (i, j) with
// i + j < nplanes are accumulated (3 for nplanes = 2, 6 for nplanes = 3).
struct TcTerm {
  const __nv_bfloat16* a[4];
  const __nv_bfloat16* b[4];
  int neg;
};
struct TcOut {
  float* d;                       // FP32 result (may be null)
  int64_t ldd;
  __nv_bfloat16* split[4];        // optional BF16 split planes of the result
  int nsplit;
  int64_t lds;
};
void launch_gemm_tc(int64_t M, int64_t N, int64_t K, const TcTerm* terms, int nterms,
                    int nplanes, int64_t lda, int64_t ldb, float alpha, float beta,
                    const float* C, int64_t ldc, float gamma, TcOut out, int* err,
                    unsigned timeout_ms, cudaStream_t s);
bool tc_available();

// Int8 slices (Ozaki splitting) of an operand: S = 4 or 5 slices per plane, row exponents
// shared by the real and imaginary planes; optional negated imaginary slices.
struct I8Slices {
  int8_t* re[5];
  int8_t* im[5];
  int8_t* neg_im[5];
  int* exp;
  int64_t ld;   // bytes between rows of a slice
  double* dg;   // grouped slicing: per row, the diagonal element left out of the slices
};
template <typename TI>
void launch_slice_rows(int S, const TI* re, const TI* im, int64_t ld, int64_t rows, int64_t K,
                       I8Slices out, bool want_neg_im, cudaStream_t s);
// Grouped int8 product: many independent problems D_p = alpha_p A_p Bt_p^T + beta_p C_p +
// gamma_p I in one launch.  The A (Bt) slices of every problem are rows of the same stacked
// slice planes (one common pitch); each problem names its first rows there.
struct GProblem {
  int a_row0, b_row0;   // first slice row of A_p / Bt_p in the stacked planes
  int M, N, K;          // M, N multiples of 16; K multiple of 64 and <= the pitch
  int sym;              // symmetric output: only tiles touching the upper triangle are listed
  double alpha, beta, gamma;
  const void* C;        // element type of the launch (T)
  int64_t ldc;
  void* D;
  int64_t ldd;
  void* Dt;             // optional: also store D^T here (non-symmetric problems only)
  int64_t ldt;
  // Diagonal split (square problems whose slabs left the diagonal out, GSlab::diag0 = 0):
  // A Bt^T = A' B'^T + a_ii B_ij + A'_ij b_jj with the diagonals a, b from I8Slices::dg and the
  // FP64 masters A (ldam) and Bt (ldbm) read in the epilogue.  split: 0 off; 1 on; 2 on, and A
  // is symmetric (read by columns; Am 16-byte aligned with ldam even for split 1).
  int split;
  const void* Am;
  int64_t ldam;
  const void* Btm;
  int64_t ldbm;
};
// One output tile of a grouped launch: problem, tile coordinates (BM = 128, BN = the launch's
// tile width: 128 for 4 slices, 96 for 5), and the K steps [kb0, kb1) of 64 bytes to run (a
// triangular factor has zero blocks that need no K steps).
struct GTile {
  int prob, mb, nb, kb0, kb1, pad;
};
int i8_tile_bn(int S);
struct I8Term {
  const int8_t* a[5];
  const int8_t* b[5];
};
// D = alpha * 2^(ea_i + eb_j) * sum_t A_t Bt_t^T + beta C + gamma I with exact int32 accumulation
// of the slice products (S slices, products p + q <= S + 1); `sym`: the result is symmetric,
// only tiles touching the upper triangle are computed and mirrored (M == N).
template <typename TO>
void launch_gemm_i8(int S, int64_t M, int64_t N, int64_t K, const I8Term* terms, int nterms,
                    int64_t lda, int64_t ldb, const int* aexp, const int* bexp, double alpha,
                    double beta, const TO* C, int64_t ldc, double gamma, TO* D, int64_t ldd, bool sym,
                    int* err, unsigned timeout_ms, cudaStream_t s);
// Grouped Cholesky block step: one job per matrix (nb <= 128; every job's block is nb wide).
// A block that is not positive definite sets kDevSingular in err and, when job_err is given,
// job_err[tag] = 1.
struct GChol {
  void* G;
  int64_t ld, k0;
  int nb, tag;
  void* Linv;
  void* LinvT;
};
template <typename T>
void launch_potrf_inv_grouped(const GChol* jobs, int njobs, int* err, int* job_err, cudaStream_t s);
// Set the kernels' shared-memory attributes ahead of a stream capture.
void prepare_potrf_inv_grouped();
void prepare_gemm_i8_grouped(int S);
// Grouped pipeline of fx_batch.cu, as a one-walk pipeline for the per-walk engine: walk
// generators X = i*(real symmetric), plain form (int8 slices on FP64 masters).  Any of dpsi0 /
// dpsi / dU may be null.  Throws fx::Error (FX_ERR_VALUE when X is not of that form).
class BatchPipeline;
// Stage of a product launch, for the per-launch timing of a profiled run.
enum ProdTag {
  kTagPowers = 0,      // A2, A4, A6 (and A8)
  kTagPade = 1,        // Pade numerator / denominator products
  kTagSolve = 2,       // V^2, W^2, VW of the solve
  kTagCholesky = 3,    // Cholesky panel and trailing updates
  kTagInverse = 4,     // explicit inverse of the Cholesky factor
  kTagTriangular = 5,  // Z = P2 L^-T, R^T = Z L^-1
  kTagSquare = 6,      // squarings
  kTagDrift = 7,       // diagnostic unitarity products
  kTagNewton = 8,      // Newton-Schulz inverse of the solve
  // whole-run timeline records (profile mode, no ops): phase 1, the host gap between the two
  // phases (read-back, selection, recording or graph launch), phase 2, the checks after it
  kTagPhase1 = 9,
  kTagHostGap = 10,
  kTagPhase2 = 11,
  kTagChecks = 12
};
struct ProdRecord {
  int tag;
  double ms, ops, flops;
};
BatchPipeline* batch_pipeline_create(int64_t n, int dtype);
void batch_pipeline_destroy(BatchPipeline* p);
// Options of one run of the one-walk pipeline.
struct PipeOpts {
  bool profile = false;      // CUDA-event timing of every product launch
  unsigned timeout_ms = 2000;
  int selector = 0;          // 0 Al-Mohy & Higham, 1 certified bound, 2 learned, 3 estimated
  int inject_stall = -1;     // diagnostics: k >= 0 makes product launch k of every run skip the
                             // operand loads of its first K step, so that the bounded waits run out
  int form = FX_FORM_PLAIN;  // FX_FORM_MIXED: two-product squarings with the slice schedule below
  int sq_n4 = 0, sq_n3 = 0;  // mixed form: the last sq_n3 squarings at 3 slices, the sq_n4 before at 4
  int pade_slices = 5;       // mixed form: slices of the Pade and solve products
  int newton_slices = 5;     // mixed form: slices of the Newton-Schulz steps that leave a residual
                             // above 1e-3 (the later ones take pade_slices)
  int solve = 0;             // Pade solve: 0 by form and size, 1 Cholesky, 2 Newton-Schulz
  bool drift = false;        // diagnostics: unitarity residual after every squaring
  int approx = 0;            // 0 Pade, 1 Chebyshev-Bessel polynomial (walk generators)
};
// Default slice schedule of the mixed form (see fx_batch.cu, BatchPipeline::sq_slices and
// BatchPipeline::newton_solve).
constexpr int kMixedN4 = 8, kMixedN3 = 0, kMixedPade = 4, kMixedNewton = 3;
void batch_pipeline_run(BatchPipeline* p, const void* dX, const void* dpsi0, void* dpsi, void* dU,
                        const PipeOpts& o, cudaStream_t s);
void batch_pipeline_stats(const BatchPipeline* p, fx_stats* st);
const std::vector<ProdRecord>& batch_pipeline_products(const BatchPipeline* p);
std::vector<double> batch_pipeline_drift(const BatchPipeline* p);
void batch_pipeline_spectral(const BatchPipeline* p, double* rho_lanczos, double* rho_up);
// Host <-> device copies of large host buffers (fx_hostcopy.cu): a buffer the driver knows as
// page-locked is copied by DMA directly; any other goes through two page-locked chunk buffers,
// the host side of a chunk (split over threads) overlapping the DMA of the previous one.
bool host_is_pinned(const void* p);
// First touch of every page of a (pageable) host buffer, split over the copy workers.
void prefault_host(void* p, size_t bytes);
struct HostStage {
  void* buf[2] = {nullptr, nullptr};
  cudaEvent_t ev[2] = {nullptr, nullptr};
  HostStage() = default;
  HostStage(const HostStage&) = delete;
  HostStage& operator=(const HostStage&) = delete;
  ~HostStage();
  void release();
  void ensure();
  // device dst <- host src, ordered on s; src may be reused once it returns.
  void h2d(void* dst, const void* src, size_t bytes, cudaStream_t s);
  // host dst <- device src after the work already on s; dst holds the data when it returns.
  void d2h(void* dst, const void* src, size_t bytes, cudaStream_t s);
};
// Learned selector inference (fx_selector.cu): out[n x 6] = MLP(x[n x 8]), device pointers.
void launch_mlp_infer(const float* w, const float* x, int n, float* out, cudaStream_t s);
// Records the message returned by fx_product_error (fx_debug.cu).
void set_product_error(const std::string& msg);
// Grouped form of launch_gemm_i8: `probs` and `tiles` are device arrays; the slice planes of
// `terms` are the stacked planes (pitch bytes per row, a_rows / b_rows rows); aexp / bexp are
// indexed by stacked row.
template <typename TO>
void launch_gemm_i8_grouped(int S, const I8Term* terms, int nterms, int64_t pitch, int64_t a_rows,
                            int64_t b_rows, const int* aexp, const int* bexp, const GProblem* probs,
                            const GTile* tiles, int ntiles, int* err, unsigned timeout_ms, cudaStream_t s,
                            const double* adg = nullptr, const double* bdg = nullptr, int skip_tile = -1);
// Grouped slicing: slab k copies rows [0, rows_k) of a planar (re, im) source with leading
// dimension ld_k, K_k columns, into stacked rows [row0_k, row0_k + rows_k).  Slabs are sorted
// by row0 and do not overlap; rows between slabs are left alone.
struct GSlab {
  const void* re;
  const void* im;
  int64_t ld;
  int rows, K, row0;
  int diag0;            // kNoDiag, or: local row r holds its diagonal element at column r + diag0,
                        // which is left out of the slices and written to I8Slices::dg
};
constexpr int kNoDiag = -(1 << 30);
// Block plan of the two-pass slicer over slabs sorted by row0 (device copy of slice_plan's
// prefix: plan[i] = first digit-pass block of slab i, plan[nslabs] = blocks).
constexpr int kPlanGroups = 2048;   // 4-column groups per digit-pass block
struct SlicePlan {
  const int* plan = nullptr;
  int blocks = 0;
};
std::vector<int> slice_plan(const std::vector<GSlab>& sorted);
// With a plan: two passes, row exponents (a warp per row) and then the digits over the plan's
// blocks (each slab's rows x K elements in row-major order); without one: a warp per row that
// reads the row twice.  kind: -1 by the plan, 0 / 1 to choose (both give the same digits; the
// choice is for the kernel tests).
template <typename TI>
void launch_slice_rows_grouped(int S, const GSlab* slabs, int nslabs, int64_t total_rows, I8Slices out,
                               bool want_neg_im, cudaStream_t s, SlicePlan plan = SlicePlan(), int kind = -1);
// In place A <- (A + A^T) / 2 of an n x n plane (exact symmetry of a result known to be
// symmetric in exact arithmetic).
template <typename T>
void launch_symmetrize(T* a, int64_t n, int64_t ld, cudaStream_t s);

}  // namespace fx
