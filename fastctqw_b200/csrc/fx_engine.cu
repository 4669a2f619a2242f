// Host orchestration of the expm(X) pipeline and the C ABI (include/fastctqw_b200.h).
//
// One fx_engine owns, from fx_create until fx_free, everything a run needs: the device
// workspace of padded planar matrices, a stream, CUDA events and the device error word --
// the same ownership as the reference's MatrixExpCalculator<T>
// (include/MatrixExpCalculator.h:17-103), whose arithmetic lived in a prebuilt library.
//
// Pipeline of one run (Al-Mohy & Higham 2009, scaling and squaring with Pade):
//   1. input statistics in FP64: line sums, diagonal, exact structure flags
//   2. exact shifts  X = mu I + nu J/n + Y  (trace shift; rank-one commuting shift when
//      every row and column sum is the same number)          -> planar Y, zero padded
//   3. A2 = Y^2, A4 = A2^2, A6 = A4 A2; ||Y||_1, d4, d6 exact; d8, d10 by the
//      deterministic block 1-norm estimator; l(A, m) from ||(|Y|)^p||_1 unless Y is normal
//   4. (m, s) selection (theta_m of the 2009 paper)
//   5. Pade: U (odd part), V (even part) with the powers scaled by 2^-s (folded into the
//      coefficients), Q = V - U, P = V + U
//   6. blocked right-looking LU with partial pivoting of Q, R = Q^-1 P
//   7. s squarings, in I+E form (E <- 2E + E^2); for X = i*(real symmetric) the real and
//      imaginary parts of R commute and each squaring is two real products:
//      Re' = (Re+Im)(Re-Im), Im' = 2 Re Im
//   8. U = e^mu (I + E + (e^nu - 1) J/n), written in the caller's dtype; optional psi = U psi0
// The products run on the tcgen05 kernel (BF16 split planes, FP32 accumulate) for the
// complex64/float32 handles and on the CUDA-core FP64 kernel for complex128/float64.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <memory>
#include <mutex>
#include <thread>
#include <string>
#include <vector>

#include "fx_kernels.cuh"

namespace fx {
namespace {

// Al-Mohy & Higham (2009), Table 3.1 (theta_13 = 4.25 of their Algorithm 6.1).
const double kTheta3 = 1.495585217958292e-2, kTheta5 = 2.539398330063230e-1,
             kTheta7 = 9.504178996162932e-1, kTheta9 = 2.097847961257068e0, kTheta13 = 4.25;

double factorial(int k) {
  double f = 1;
  for (int i = 2; i <= k; ++i) f *= i;
  return f;
}
// b_j = (2m - j)! / (j! (m - j)!)
std::vector<double> pade_coeffs(int m) {
  std::vector<double> b(m + 1);
  for (int j = 0; j <= m; ++j) b[j] = factorial(2 * m - j) / (factorial(j) * factorial(m - j));
  return b;
}
// 1 / |c_{2m+1}| = (2m)! (2m+1)! / (m!)^2
double ell_const(int m) { return factorial(2 * m) * factorial(2 * m + 1) / (factorial(m) * factorial(m)); }
int pade_products(int m) { return m == 3 ? 2 : m == 5 ? 3 : m == 7 ? 4 : m == 9 ? 5 : 6; }

// Deterministic second probe column: +1 when bit 31 of i*0x9E3779B1 (mod 2^32) is clear.
double probe_sign(int64_t i) {
  uint32_t h = (uint32_t)((uint64_t)i * 0x9E3779B1ull);
  return (h >> 31) & 1 ? -1.0 : 1.0;
}

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  void alloc(size_t b) {
    if (inject_alloc_failure() || cudaMalloc(&p, b) != cudaSuccess) {
      p = nullptr;
      cudaGetLastError();
      throw Error{FX_ERR_NOMEM, "device allocation of " + std::to_string(b) + " bytes failed"};
    }
    bytes = b;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
};

struct RunOpts {
  int form;
  int shift;
  int structure;
  int force_s, force_m;
  unsigned timeout_ms;
  int ipe;
  int debug_stage;   // 0: normal output; k > 0: output an intermediate (diagnostics)
  int profile;       // 1: time every int8 product launch with CUDA events
  int selector;      // (m, s) selection of the grouped path: 0 plain, 1 certified, 2 learned
  int inject_stall;  // diagnostics of the grouped path: product launch that skips a K step (-1 off)
  int sq_n4, sq_n3;  // mixed form of the grouped path: squarings at 4 and at 3 slices
  int pade_slices;   // mixed form of the grouped path: slices of the Pade and solve products
  int newton_slices; // mixed form of the grouped path: slices of the early Newton-Schulz steps
  int solve;         // grouped path: Pade solve, 0 by form and size, 1 Cholesky, 2 Newton-Schulz
  int drift;         // diagnostics of the grouped path: unitarity residual after every squaring
  int approx;        // grouped path: 0 Pade, 1 Chebyshev-Bessel polynomial
};

// Planar complex matrix view over owned storage; a missing plane is identically zero.
template <typename T>
struct CM {
  T* rb = nullptr;
  T* ib = nullptr;
  bool hr = false, hi = false;
  T* re() const { return hr ? rb : nullptr; }
  T* im() const { return hi ? ib : nullptr; }
};

template <typename T>
class Pipeline {
 public:
  Pipeline(int64_t n, int dtype) : n_(n), np_(pad_n(n > 0 ? n : 1)), dtype_(dtype) {
    const size_t plane = sizeof(T) * (size_t)np_ * (size_t)np_;
    const int nmat = kNumMats;
    mats_.alloc(plane * 2 * nmat);
    T* base = (T*)mats_.p;
    for (int i = 0; i < nmat; ++i) {
      slot_[i].rb = base + (size_t)(2 * i) * np_ * np_;
      slot_[i].ib = base + (size_t)(2 * i + 1) * np_ * np_;
    }
    if (std::is_same<T, float>::value) {
      // BF16 split planes (mixed form): 2 operands x 2 planes x up to 4 parts.
      split_.alloc(sizeof(__nv_bfloat16) * (size_t)np_ * (size_t)np_ * kSplitPlanes);
    }
    // int8 slices (plain form): A (re, im) and Bt (re, im, -im), up to 5 slices each, + exponents.
    slices_.alloc((size_t)np_ * (size_t)np_ * kSlicePlanes + sizeof(int) * 2 * (size_t)np_ + 4096);
    small_.alloc(sizeof(double) * (size_t)np_ * 48 + 4096);
    ipiv_.alloc(sizeof(int) * (size_t)np_);
    err_.alloc(sizeof(int) * 8);
    const size_t tbytes = sizeof(T) * (size_t)np_ * kPanel;
    panel_t_.alloc(tbytes * 2);
    chol_.alloc(sizeof(T) * (size_t)np_ * kCholNb * 6);
  }
  ~Pipeline() {
    mats_.release();
    split_.release();
    slices_.release();
    small_.release();
    ipiv_.release();
    err_.release();
    panel_t_.release();
    chol_.release();
  }

  using Opts = RunOpts;

  // Runs the pipeline on the device input dX; writes dU (interleaved, n x n) if non-null and
  // psi = U psi0 if dpsi0/dpsi are non-null.
  void run(const void* dX, void* dU, const void* dpsi0, void* dpsi, const Opts& o,
           cudaStream_t s, fx_stats& st) {
    st = fx_stats{};
    gemm_count_ = 0;
    launches_ = 0;
    opts_ = o;
    stream_ = s;
    const bool fp32 = std::is_same<T, float>::value;
    form_ = o.form;
    if (fp32 && form_ == FX_FORM_FP64) throw Error{FX_ERR_VALUE, "FP64 form needs the FP64 pipeline"};
    if (!fp32 && form_ == FX_FORM_MIXED) throw Error{FX_ERR_VALUE, "mixed form needs the FP32 pipeline"};
    if (!fp32 && form_ == FX_FORM_SIMT) form_ = FX_FORM_FP64;
    if ((form_ == FX_FORM_PLAIN || form_ == FX_FORM_MIXED) && !tc_available())
      throw Error{FX_ERR_NODEV, "tcgen05 products need an sm_100 device"};
    nplanes_ = form_ == FX_FORM_MIXED ? 2 : 3;
    FX_CUDA(cudaMemsetAsync(err_.p, 0, sizeof(int) * 8, s));

    // ---- 1. statistics of the input
    double* d_small = (double*)small_.p;
    InputStats is{d_small, d_small + 2 * n_, d_small + 4 * n_, (int*)(d_small + 6 * n_)};
    FX_CUDA(cudaMemsetAsync(is.flags, 0, sizeof(int) * 8, s));
    launch_input_stats(dX, dtype_, n_, is, s);
    launches_ += 4;
    std::vector<double> h_small(6 * n_);
    int h_flags[8];
    FX_CUDA(cudaMemcpyAsync(h_small.data(), d_small, sizeof(double) * 6 * n_, cudaMemcpyDeviceToHost, s));
    FX_CUDA(cudaMemcpyAsync(h_flags, is.flags, sizeof(int) * 8, cudaMemcpyDeviceToHost, s));
    FX_CUDA(cudaStreamSynchronize(s));
    if (h_flags[4]) throw Error{FX_ERR_NONFINITE, "input contains NaN or Inf"};
    const bool re_zero = !h_flags[0];
    const bool symmetric = !h_flags[2];
    const bool skewh = !h_flags[3];
    const bool real_in = dtype_ == FX_F32 || dtype_ == FX_F64;
    std::complex<double> tr(0, 0);
    for (int64_t i = 0; i < n_; ++i) tr += std::complex<double>(h_small[4 * n_ + 2 * i], h_small[4 * n_ + 2 * i + 1]);
    std::complex<double> mu(0, 0), nu(0, 0);
    bool rank1 = false;
    if (o.shift >= 1 && n_ > 0) mu = tr / (double)n_;
    if (o.shift >= 2 && n_ > 1) {
      const double c0r = h_small[0], c0i = h_small[1];
      bool eq = true;
      for (int64_t i = 0; i < n_ && eq; ++i)
        eq = h_small[2 * i] == c0r && h_small[2 * i + 1] == c0i &&
             h_small[2 * n_ + 2 * i] == c0r && h_small[2 * n_ + 2 * i + 1] == c0i;
      if (eq) {
        rank1 = true;
        nu = std::complex<double>(c0r, c0i) - mu;
      }
    }
    structured_ = o.structure && re_zero && symmetric && !real_in;
    normal_ = o.structure && skewh;
    sym_ = symmetric;
    st.structured = structured_;
    st.rank1_shift = rank1;
    st.symmetric = symmetric;

    // ---- 2. shifted, padded planar Y
    CM<T>& Y = slot_[kY];
    Y.hr = true;
    Y.hi = !real_in;
    const std::complex<double> nu_n = n_ > 0 ? nu / (double)n_ : std::complex<double>(0, 0);
    launch_load_shifted<T>(dX, dtype_, n_, np_, mu.real(), mu.imag(), nu_n.real(), nu_n.imag(), Y.rb,
                           Y.hi ? Y.ib : nullptr, s);
    ++launches_;
    if (structured_) Y.hr = false;  // X - shifts is purely imaginary: drop the zero plane
    if (dump(1, Y, dU)) return;

    // ---- 3. norms and powers
    const double anorm = onenorm(Y);
    st.norm1 = anorm;
    CM<T>& A2 = slot_[kA2];
    CM<T>& A4 = slot_[kA4];
    CM<T>& A6 = slot_[kA6];
    mm(A2, Y, Y, 1.0, nullptr, 0.0, 0.0);
    mm(A4, A2, A2, 1.0, nullptr, 0.0, 0.0);
    mm(A6, A4, A2, 1.0, nullptr, 0.0, 0.0);
    if (dump(2, A2, dU) || dump(3, A4, dU) || dump(4, A6, dU)) return;
    const double d4 = std::pow(onenorm(A4), 0.25);
    const double d6 = std::pow(onenorm(A6), 1.0 / 6.0);
    st.d[0] = d4;
    st.d[1] = d6;

    // log2 ||(|Y|)^p||_1 for p = 7, 11, 15, 19, 27 (only when l is needed)
    std::vector<double> abslog;
    auto ell = [&](int m, int sc) -> int {
      if (normal_) return 0;
      if (abslog.empty()) abslog = abs_power_log2(27);
      const double lp = abslog[2 * m + 1];
      if (!std::isfinite(lp) || anorm == 0.0) return 0;
      const double l2a = lp - std::log2(anorm) - std::log2(ell_const(m)) - 2.0 * m * sc;
      const int v = (int)std::ceil((l2a + 53.0) / (2.0 * m));
      return v > 0 ? v : 0;
    };
    int m = 13, sq = 0;
    double d8 = -1, d10 = -1;
    if (std::max(d4, d6) < kTheta3 && ell(3, 0) == 0) {
      m = 3;
    } else if (std::max(d4, d6) < kTheta5 && ell(5, 0) == 0) {
      m = 5;
    } else {
      d8 = std::pow(normest({&A4, &A4}), 0.125);
      const double eta3 = std::max(d6, d8);
      if (eta3 < kTheta7 && ell(7, 0) == 0) {
        m = 7;
      } else if (eta3 < kTheta9 && ell(9, 0) == 0) {
        m = 9;
      } else {
        d10 = std::pow(normest({&A4, &A6}), 0.1);
        const double eta5 = std::min(eta3, std::max(d8, d10));
        sq = eta5 == 0.0 ? 0 : std::max((int)std::ceil(std::log2(eta5 / kTheta13)), 0);
        sq += ell(13, sq);
      }
    }
    st.d[2] = d8;
    st.d[3] = d10;
    st.d[4] = abslog.empty() ? -1.0 : abslog[27];
    if (o.force_m > 0) m = o.force_m;
    if (o.force_s >= 0) sq = o.force_s;
    if (m != 13) sq = (o.force_s >= 0 && o.force_m == m) ? sq : 0;
    st.m = m;
    st.s = sq;

    // ---- 5. Pade numerator / denominator
    CM<T>& U = slot_[kU];
    CM<T>& V = slot_[kV];
    CM<T>& T1 = slot_[kT1];
    CM<T>& T2 = slot_[kT2];
    const std::vector<double> b = pade_coeffs(m);
    const double c = std::ldexp(1.0, -sq), c2 = c * c, c4 = c2 * c2, c6 = c4 * c2;
    if (m == 13) {
      combo(T1, {{&A6, b[13] * c6}, {&A4, b[11] * c4}, {&A2, b[9] * c2}}, 0.0);
      mm(T2, A6, T1, c6, nullptr, 0.0, 0.0);                      // W1 = B6 (..)
      combo(T1, {{&T2, 1.0}, {&A6, b[7] * c6}, {&A4, b[5] * c4}, {&A2, b[3] * c2}}, b[1]);
      mm(U, Y, T1, c, nullptr, 0.0, 0.0);                         // U = B (W1 + ..)
      combo(T1, {{&A6, b[12] * c6}, {&A4, b[10] * c4}, {&A2, b[8] * c2}}, 0.0);
      combo(T2, {{&A6, b[6] * c6}, {&A4, b[4] * c4}, {&A2, b[2] * c2}}, 0.0);
      mm(V, A6, T1, c6, &T2, 1.0, b[0]);                          // V = B6 (..) + ..
    } else {
      // m in {3,5,7,9}: s = 0, powers A2, A4, A6 (A8 = A4^2 for m = 9).
      CM<T>& A8 = slot_[kT2];
      std::vector<CM<T>*> pw = {nullptr, &A2, &A4, &A6};
      if (m == 9) {
        mm(A8, A4, A4, 1.0, nullptr, 0.0, 0.0);
        pw.push_back(&A8);
      }
      const int h = m / 2;
      std::vector<std::pair<CM<T>*, double>> odd, even;
      for (int k = 1; k <= h; ++k) {
        odd.push_back({pw[k], b[2 * k + 1]});
        even.push_back({pw[k], b[2 * k]});
      }
      combo(T1, odd, b[1]);
      mm(U, Y, T1, 1.0, nullptr, 0.0, 0.0);
      combo(V, even, b[0]);
    }

    if (dump(5, U, dU) || dump(6, V, dU)) return;
    CM<T>& Q = slot_[kQ];
    CM<T>& R = slot_[kR];
    // FP64 masters only: in FP32 storage the kappa(Q)^2 of the normal equations costs accuracy.
    const bool chol = std::is_same<T, double>::value && structured_ && normal_ && V.hr && !V.hi && U.hi && !U.hr;
    st.solver = chol ? 1 : 0;
    if (chol) {
      // ---- 6'. X = i*(real symmetric): P = conj(Q) = Q^H, so R = Q^-1 P = G^-1 (Q^H)^2 with
      // G = Q^H Q = V^2 + W^2 real SPD (V even part, U = iW odd part; V and W commute).
      CM<T>& VV = slot_[kT1];
      CM<T>& WW = slot_[kT2];
      CM<T>& VW = slot_[kTmp];
      cproduct(np_, np_, np_, V.rb, nullptr, np_, V.rb, nullptr, np_, 1.0, nullptr, nullptr, np_, 0.0, 0.0,
               VV.rb, nullptr, np_, true);
      cproduct(np_, np_, np_, U.ib, nullptr, np_, U.ib, nullptr, np_, 1.0, nullptr, nullptr, np_, 0.0, 0.0,
               WW.rb, nullptr, np_, true);
      cproduct(np_, np_, np_, V.rb, nullptr, np_, U.ib, nullptr, np_, 1.0, nullptr, nullptr, np_, 0.0, 0.0,
               VW.rb, nullptr, np_, true);
      launch_combo<T>(Q.rb, VV.rb, 1.0, WW.rb, 1.0, nullptr, 0, nullptr, 0, 0.0, np_, s);
      launch_combo<T>(R.rb, VV.rb, 1.0, WW.rb, -1.0, nullptr, 0, nullptr, 0, 0.0, np_, s);
      launch_combo<T>(R.ib, VW.rb, 2.0, nullptr, 0, nullptr, 0, nullptr, 0, 0.0, np_, s);
      launches_ += 3;
      Q.hr = true;
      Q.hi = false;
      R.hr = R.hi = true;
      chol_solve(Q.rb, R.rb, R.ib);
    } else {
      // Q = V - U into the LU slot, P = V + U into the solution slot.
      combo(Q, {{&V, 1.0}, {&U, -1.0}}, 0.0);
      combo(R, {{&V, 1.0}, {&U, 1.0}}, 0.0);
      // The solver works on full planes: materialise a zero imaginary plane if needed.
      ensure_planes(Q, !real_in);
      ensure_planes(R, !real_in);
      // ---- 6. R = Q^-1 P
      lu_solve(Q, R);
    }
    if (sym_) {
      // R = Q^-1 P is symmetric in exact arithmetic (P, Q commute and are symmetric); the
      // solve leaves an antisymmetric rounding part that the squarings would amplify.
      launch_symmetrize<T>(R.rb, np_, np_, s);
      if (R.hi) launch_symmetrize<T>(R.ib, np_, np_, s);
      launches_ += R.hi ? 2 : 1;
    }
    if (dump(7, R, dU)) return;

    // ---- 7. squarings in I+E form
    const bool ipe = o.ipe != 0;
    if (ipe) add_identity(R, -1.0);
    // With the rank-one shift, Y 1 = 0 = 1^T Y, hence E 1 = 0 = 1^T E exactly (E = R - I):
    // restore that invariant after the solve and after every squaring (an exact identity of
    // the iterates, O(N^2); rounding otherwise accumulates along the all-ones direction).
    const bool project = rank1 && ipe;
    auto proj = [&]() {
      if (!project) return;
      double* scr = (double*)small_.p + 8 * np_;
      if (R.hr) launch_project_ones<T>(R.rb, n_, np_, scr, s);
      if (R.hi) launch_project_ones<T>(R.ib, n_, np_, scr, s);
      launches_ += 5 * ((int)R.hr + (int)R.hi);
    };
    proj();
    for (int k = 0; k < sq; ++k) {
      if (dump(8 + k, R, dU)) return;
      square(R, ipe);
      proj();
    }
    if (dump(8 + sq, R, dU)) return;

    // ---- 8. output
    OutputMap om{};
    const std::complex<double> emu = std::exp(mu);
    om.emu_re = emu.real();
    om.emu_im = emu.imag();
    if (rank1) {
      const std::complex<double> cj = (std::exp(nu) - 1.0) / (double)n_;
      om.cj_re = cj.real();
      om.cj_im = cj.imag();
    }
    om.ipe = ipe ? 1 : 0;
    if (dU) {
      launch_output<T>(R.re(), R.im(), n_, np_, om, dU, dtype_, s);
      ++launches_;
    }
    if (dpsi0 && dpsi) {
      launch_apply<T>(R.re(), R.im(), n_, np_, om, dpsi0, dpsi, dtype_ == FX_C128 || dtype_ == FX_F64 ? FX_C128 : FX_C64,
                      d_small + 14 * np_, s);
      launches_ += 2;
    }
    int h_err[8];
    FX_CUDA(cudaMemcpyAsync(h_err, err_.p, sizeof(int) * 8, cudaMemcpyDeviceToHost, s));
    FX_CUDA(cudaStreamSynchronize(s));
    if (h_err[0] & kDevTimeout) throw Error{FX_ERR_TIMEOUT, "a device-side wait timed out"};
    if (h_err[0] & kDevSingular) throw Error{FX_ERR_SINGULAR, "Pade denominator is singular"};
    prof_collect(st);
    st.form = form_;
    st.gemm_launches = gemm_count_;
    st.launches = launches_;
    const double N3 = (double)n_ * n_ * n_;
    st.flops = 8.0 * N3 * (pade_products(m) + sq) + (8.0 / 3.0) * N3 + 8.0 * N3;
  }

  int64_t n() const { return n_; }

  // Diagnostics: write intermediate matrix M (no shifts undone) to dU and stop the run.
  bool dump(int stage, const CM<T>& M, void* dU) {
    if (opts_.debug_stage != stage || !dU) return false;
    OutputMap om{};
    om.emu_re = 1.0;
    launch_output<T>(M.re() ? M.re() : zero_plane(), M.im(), n_, np_, om, dU, dtype_, stream_);
    FX_CUDA(cudaStreamSynchronize(stream_));
    return true;
  }

 private:
  enum { kY, kA2, kA4, kA6, kT1, kT2, kU, kV, kQ, kR, kTmp, kS1, kS2, kBt, kNumMats };
  static constexpr int kSplitPlanes = 16;
  static constexpr int kSlicePlanes = 25;
  static constexpr int kPanel = 128;
  static constexpr int kCholNb = 128;

  int64_t n_, np_;
  int dtype_;
  DevBuf mats_, split_, slices_, small_, ipiv_, err_, panel_t_, chol_;
  CM<T> slot_[kNumMats];
  Opts opts_{};
  cudaStream_t stream_ = nullptr;
  int form_ = FX_FORM_PLAIN, nplanes_ = 3;
  bool structured_ = false, normal_ = false, sym_ = false;
  int gemm_count_ = 0, launches_ = 0;

  int* derr() const { return (int*)err_.p; }

  // ---- live timing of the int8 product launches (CUDA events on the launch stream)
  std::vector<cudaEvent_t> ev_pool_;
  std::vector<std::pair<double, double>> ev_work_;   // (issued int8 ops, useful real flops)
  size_t ev_used_ = 0;
  void prof_begin() {
    if (!opts_.profile) return;
    if (ev_used_ + 2 > ev_pool_.size()) {
      for (int i = 0; i < 64; ++i) {
        cudaEvent_t e;
        FX_CUDA(cudaEventCreate(&e));
        ev_pool_.push_back(e);
      }
    }
    FX_CUDA(cudaEventRecord(ev_pool_[ev_used_], stream_));
  }
  void prof_end(double ops, double flops) {
    if (!opts_.profile) return;
    FX_CUDA(cudaEventRecord(ev_pool_[ev_used_ + 1], stream_));
    ev_work_.push_back({ops, flops});
    ev_used_ += 2;
  }
  void prof_collect(fx_stats& st) {
    if (!opts_.profile) return;
    FX_CUDA(cudaStreamSynchronize(stream_));
    double ms = 0, ops = 0, fl = 0;
    for (size_t i = 0; i < ev_work_.size(); ++i) {
      float t = 0;
      FX_CUDA(cudaEventElapsedTime(&t, ev_pool_[2 * i], ev_pool_[2 * i + 1]));
      ms += t;
      ops += ev_work_[i].first;
      fl += ev_work_[i].second;
    }
    st.prod_ms = ms;
    st.prod_ops = ops;
    st.prod_flops = fl;
    st.prod_launches = (int)ev_work_.size();
    ev_work_.clear();
    ev_used_ = 0;
  }
  static double sym_tile_fraction(int64_t n, int S) {
    const int bn = S == 4 ? 128 : 96;
    const int64_t tm = (n + 127) / 128, tn = (n + bn - 1) / bn;
    int64_t cnt = 0;
    for (int64_t r = 0; r < tm; ++r) cnt += tn - (r * 128) / bn;
    return (double)cnt / (double)(tm * tn);
  }
  __nv_bfloat16* split_plane(int i, int64_t elems) const {
    if (elems > np_ * np_) throw Error{FX_ERR_VALUE, "split plane overflow"};
    return (__nv_bfloat16*)split_.p + (size_t)i * np_ * np_;
  }
  int8_t* slice_plane(int i, int64_t elems) const {
    if (elems > np_ * np_) throw Error{FX_ERR_VALUE, "slice plane overflow"};
    return (int8_t*)slices_.p + (size_t)i * np_ * np_;
  }
  int* slice_exp(int side) const {
    return (int*)((int8_t*)slices_.p + (size_t)np_ * np_ * kSlicePlanes) + side * np_;
  }

  double onenorm(const CM<T>& A) {
    if (!A.re() && !A.im()) return 0.0;
    double* col = (double*)small_.p + 8 * np_;
    launch_col_abs_sums<T>(A.re() ? A.re() : A.im(), A.re() ? A.im() : nullptr, np_, np_, col, stream_);
    launches_ += 2;
    std::vector<double> h(np_);
    FX_CUDA(cudaMemcpyAsync(h.data(), col, sizeof(double) * np_, cudaMemcpyDeviceToHost, stream_));
    FX_CUDA(cudaStreamSynchronize(stream_));
    double mx = 0;
    for (double v : h) mx = std::max(mx, v);
    if (!std::isfinite(mx)) throw Error{FX_ERR_NONFINITE, "non-finite norm in the pipeline"};
    return mx;
  }

  void ensure_planes(CM<T>& A, bool want_im) {
    if (!A.hr) {
      launch_zero<T>(A.rb, np_ * np_, stream_);
      A.hr = true;
      ++launches_;
    }
    if (want_im && !A.hi) {
      launch_zero<T>(A.ib, np_ * np_, stream_);
      A.hi = true;
      ++launches_;
    }
  }

  // D = sum c_k M_k + g I, planewise.
  void combo(CM<T>& D, std::vector<std::pair<CM<T>*, double>> terms, double g) {
    const T* r[4] = {nullptr, nullptr, nullptr, nullptr};
    const T* i_[4] = {nullptr, nullptr, nullptr, nullptr};
    double cr[4] = {0, 0, 0, 0};
    bool any_r = g != 0.0, any_i = false;
    int k = 0;
    for (auto& t : terms) {
      if (k >= 4) throw Error{FX_ERR_VALUE, "combo: too many terms"};
      r[k] = t.first->re();
      i_[k] = t.first->im();
      cr[k] = t.second;
      any_r |= r[k] != nullptr;
      any_i |= i_[k] != nullptr;
      ++k;
    }
    // Reading and writing the same plane is fine (elementwise).
    if (any_r) {
      launch_combo<T>(D.rb, r[0], cr[0], r[1], cr[1], r[2], cr[2], r[3], cr[3], g, np_, stream_);
      ++launches_;
    }
    if (any_i) {
      launch_combo<T>(D.ib, i_[0], cr[0], i_[1], cr[1], i_[2], cr[2], i_[3], cr[3], 0.0, np_, stream_);
      ++launches_;
    }
    D.hr = any_r;
    D.hi = any_i;
  }

  void add_identity(CM<T>& A, double g) {
    ensure_planes(A, false);
    launch_combo<T>(A.rb, A.rb, 1.0, nullptr, 0, nullptr, 0, nullptr, 0, g, np_, stream_);
    ++launches_;
  }

  // ---- matrix products -------------------------------------------------------------
  // D (M x N, ldd) = alpha * A (M x K, lda) * Bt^T (Bt: N x K, ldb) + beta C + gamma I, complex
  // planar (null planes are zero).  `sym`: the result is known to be symmetric (all products of
  // the expm pipeline for a symmetric X are polynomials in X); it is then computed / stored
  // exactly symmetric.  Returns which output planes were written.
  std::pair<bool, bool> cproduct(int64_t M, int64_t N, int64_t K, const T* ar, const T* ai, int64_t lda,
                                 const T* btr, const T* bti, int64_t ldb, double alpha, const T* cr,
                                 const T* ci, int64_t ldc, double beta, double gamma, T* dr, T* di,
                                 int64_t ldd, bool sym) {
    struct P2 {
      int a;   // 0 re, 1 im
      int b;   // 0 re, 1 im
      int neg;
    };
    std::vector<P2> tr, ti;
    if (ar && btr) tr.push_back({0, 0, 0});
    if (ai && bti) tr.push_back({1, 1, 1});
    if (ar && bti) ti.push_back({0, 1, 0});
    if (ai && btr) ti.push_back({1, 0, 0});
    const bool want_r = dr && (!tr.empty() || (cr && beta != 0.0) || gamma != 0.0);
    const bool want_i = di && (!ti.empty() || (ci && beta != 0.0));
    const T* A2[2] = {ar, ai};
    const T* B2[2] = {btr, bti};
    auto plain_combo = [&](T* d, const T* c, double bt, double g) {
      // D = bt C + g I on the M x N block (only used for full np x np blocks)
      if (M != np_ || N != np_ || ldd != np_) throw Error{FX_ERR_VALUE, "combo on a sub-block"};
      launch_combo<T>(d, c, bt, nullptr, 0, nullptr, 0, nullptr, 0, g, np_, stream_);
      ++launches_;
    };

    if (form_ == FX_FORM_SIMT || form_ == FX_FORM_FP64) {
      auto run = [&](T* d, const std::vector<P2>& terms, const T* c, double g) {
        if (terms.empty()) return plain_combo(d, c, beta, g);
        std::vector<GemmTerm<T>> gt;
        for (auto& t : terms) gt.push_back(GemmTerm<T>{A2[t.a], B2[t.b], t.neg ? -1.f : 1.f});
        launch_gemm_simt<T>(M, N, K, gt.data(), (int)gt.size(), lda, ldb, alpha, c ? beta : 0.0, c, ldc, g,
                            d, ldd, stream_);
        ++gemm_count_;
        ++launches_;
        if (sym) {
          launch_symmetrize<T>(d, M, ldd, stream_);
          ++launches_;
        }
      };
      if (want_r) run(dr, tr, cr, gamma);
      if (want_i) run(di, ti, ci, 0.0);
      return {want_r, want_i};
    }
    if constexpr (std::is_same<T, float>::value) {
      if (form_ == FX_FORM_MIXED) {
        // BF16 hi+lo split planes of A (re, im) and Bt (re, im).
        __nv_bfloat16* ap[2][4] = {};
        __nv_bfloat16* bp[2][4] = {};
        for (int pl = 0; pl < 2; ++pl) {
          for (int q = 0; q < nplanes_; ++q) {
            ap[pl][q] = split_plane((pl * 2 + 0) * 4 + q, M * K);
            bp[pl][q] = split_plane((pl * 2 + 1) * 4 + q, N * K);
          }
          if (A2[pl]) launch_split(A2[pl], lda, ap[pl], nplanes_, K, M, K, false, stream_);
          if (B2[pl]) launch_split(B2[pl], ldb, bp[pl], nplanes_, K, N, K, false, stream_);
          launches_ += (A2[pl] != nullptr) + (B2[pl] != nullptr);
        }
        auto run = [&](T* d, const std::vector<P2>& terms, const T* c, double g) {
          if (terms.empty()) return plain_combo(d, c, beta, g);
          std::vector<TcTerm> tt;
          for (auto& t : terms) {
            TcTerm x{};
            for (int q = 0; q < 4; ++q) {
              x.a[q] = ap[t.a][q];
              x.b[q] = bp[t.b][q];
            }
            x.neg = t.neg;
            tt.push_back(x);
          }
          TcOut out{};
          out.d = d;
          out.ldd = ldd;
          launch_gemm_tc(M, N, K, tt.data(), (int)tt.size(), nplanes_, K, K, (float)alpha,
                         c ? (float)beta : 0.f, c, ldc, (float)g, out, derr(), opts_.timeout_ms, stream_);
          ++gemm_count_;
          ++launches_;
          if (sym) {
            launch_symmetrize<T>(d, M, ldd, stream_);
            ++launches_;
          }
        };
        if (want_r) run(dr, tr, cr, gamma);
        if (want_i) run(di, ti, ci, 0.0);
        return {want_r, want_i};
      }
    }
    if (form_ == FX_FORM_PLAIN) {
      // int8 slices with exact accumulation (S = 5 on FP64 masters, 4 on FP32 masters).
      const int S = std::is_same<T, double>::value ? 5 : 4;
      I8Slices sa{}, sb{};
      for (int q = 0; q < S; ++q) {
        sa.re[q] = slice_plane(0 * 5 + q, M * K);
        sa.im[q] = slice_plane(1 * 5 + q, M * K);
        sb.re[q] = slice_plane(2 * 5 + q, N * K);
        sb.im[q] = slice_plane(3 * 5 + q, N * K);
        sb.neg_im[q] = slice_plane(4 * 5 + q, N * K);
      }
      sa.exp = slice_exp(0);
      sb.exp = slice_exp(1);
      sa.ld = sb.ld = K;
      const bool need_a = ar || ai, need_b = btr || bti;
      if (need_a && !(need_b && ar == btr && ai == bti && lda == ldb && M == N)) {
        launch_slice_rows<T>(S, ar ? ar : ai, ar ? ai : nullptr, lda, M, K, sa, false, stream_);
        ++launches_;
      }
      // The same matrix on both sides (squarings, powers): slice it once.
      const bool same = need_a && need_b && ar == btr && ai == bti && lda == ldb && M == N;
      if (same) {
        sb.re[0] = nullptr;  // marker: B side uses the A slices
        I8Slices sab = sa;
        for (int q = 0; q < S; ++q) sab.neg_im[q] = sb.neg_im[q];
        launch_slice_rows<T>(S, ar ? ar : ai, ar ? ai : nullptr, lda, M, K, sab, ai != nullptr && ar != nullptr,
                             stream_);
        ++launches_;
        for (int q = 0; q < S; ++q) {
          sb.re[q] = sa.re[q];
          sb.im[q] = sa.im[q];
        }
        sb.exp = sa.exp;
      } else if (need_b) {
        launch_slice_rows<T>(S, btr ? btr : bti, btr ? bti : nullptr, ldb, N, K, sb,
                             bti != nullptr && btr != nullptr, stream_);
        ++launches_;
      }
      // A lone imaginary plane was sliced into the "re" slots: negate by slicing -Bt.im when needed.
      auto run = [&](T* d, const std::vector<P2>& terms, const T* c, double g) {
        if (terms.empty()) return plain_combo(d, c, beta, g);
        std::vector<I8Term> tt;
        double sgn = 1.0;
        for (auto& t : terms) {
          I8Term x{};
          for (int q = 0; q < S; ++q) {
            x.a[q] = (t.a == 0 || ar == nullptr) ? sa.re[q] : sa.im[q];
            if (t.b == 0 || btr == nullptr) x.b[q] = sb.re[q];
            else x.b[q] = t.neg ? sb.neg_im[q] : sb.im[q];
          }
          // With only imaginary planes on both sides the single term is -(Ai Bti^T).
          if (t.neg && (btr == nullptr)) sgn = -1.0;
          tt.push_back(x);
        }
        prof_begin();
        launch_gemm_i8<T>(S, M, N, K, tt.data(), (int)tt.size(), K, K, sa.exp, sb.exp, alpha * sgn,
                          c ? beta : 0.0, c, ldc, g, d, ldd, sym, derr(), opts_.timeout_ms, stream_);
        // Issued int8 MMA work: 2 M N K ops per slice product and term; a symmetric product
        // computes only the tiles touching the upper triangle.
        const double frac = sym ? sym_tile_fraction(M, S) : 1.0;
        prof_end(2.0 * (double)M * (double)N * (double)K * (S * (S + 1) / 2) * tt.size() * frac,
                 2.0 * (double)M * (double)N * (double)K * tt.size() * frac);
        ++gemm_count_;
        ++launches_;
      };
      if (want_r) run(dr, tr, cr, gamma);
      if (want_i) run(di, ti, ci, 0.0);
      return {want_r, want_i};
    }
    throw Error{FX_ERR_VALUE, "form not available for this precision"};
  }

  // D = alpha A B + beta C + gamma I  (complex, planar, np x np).  D must not alias A or B.
  void mm(CM<T>& D, const CM<T>& A, const CM<T>& B, double alpha, const CM<T>* C, double beta,
          double gamma) {
    if (&D == &A || &D == &B) throw Error{FX_ERR_VALUE, "product output aliases an operand"};
    const T* btr = B.re();
    const T* bti = B.im();
    if (!sym_) {
      // Right factor transposed into scratch (K contiguous).
      CM<T>& Bt = slot_[kBt];
      if (btr) launch_transpose<T>(btr, np_, Bt.rb, np_, np_, np_, stream_);
      if (bti) launch_transpose<T>(bti, np_, Bt.ib, np_, np_, np_, stream_);
      launches_ += (btr != nullptr) + (bti != nullptr);
      btr = btr ? Bt.rb : nullptr;
      bti = bti ? Bt.ib : nullptr;
    }
    auto w = cproduct(np_, np_, np_, A.re(), A.im(), np_, btr, bti, np_, alpha, C ? C->re() : nullptr,
                      C ? C->im() : nullptr, np_, beta, gamma, D.rb, D.ib, np_, sym_);
    D.hr = w.first;
    D.hi = w.second;
  }

  // One squaring of R (or of E = R - I when ipe).
  void square(CM<T>& R, bool ipe) {
    CM<T>& Tmp = slot_[kTmp];
    const double beta = ipe ? 2.0 : 0.0;
    if (structured_ && R.hr && R.hi && (form_ != FX_FORM_PLAIN || opts_.structure >= 2)) {
      // Re and Im of R commute (both are functions of the same real symmetric matrix), so
      // Re' = (Re + Im)(Re - Im) and Im' = 2 Re Im.  The computed parts commute only up to
      // rounding; the forms that symmetrise by averaging, (M + M^T)/2, remove that commutator
      // part.  The int8 form stores the upper triangle exactly instead and therefore uses the
      // general formula below (Re^2 - Im^2, Re Im + Im Re: symmetric by construction), which
      // in triangle mode costs the same two full-product equivalents.
      CM<T>& S1 = slot_[kS1];
      CM<T>& S2 = slot_[kS2];
      launch_combo<T>(S1.rb, R.rb, 1.0, R.ib, 1.0, nullptr, 0, nullptr, 0, 0.0, np_, stream_);
      launch_combo<T>(S2.rb, R.rb, 1.0, R.ib, -1.0, nullptr, 0, nullptr, 0, 0.0, np_, stream_);
      launches_ += 2;
      cproduct(np_, np_, np_, R.rb, nullptr, np_, R.ib, nullptr, np_, 2.0, ipe ? R.ib : nullptr, nullptr, np_,
               beta, 0.0, Tmp.ib, nullptr, np_, true);
      cproduct(np_, np_, np_, S1.rb, nullptr, np_, S2.rb, nullptr, np_, 1.0, ipe ? R.rb : nullptr, nullptr, np_,
               beta, 0.0, R.rb, nullptr, np_, true);
      std::swap(R.ib, Tmp.ib);
      return;
    }
    mm(Tmp, R, R, 1.0, ipe ? &R : nullptr, beta, 0.0);
    std::swap(R.rb, Tmp.rb);
    std::swap(R.ib, Tmp.ib);
    std::swap(R.hr, Tmp.hr);
    std::swap(R.hi, Tmp.hi);
  }

  // ---- 1-norm estimator (mirror of the oracle's deterministic Higham-Tisseur t = 2).
  double normest(std::vector<CM<T>*> mats) {
    const int64_t n = n_, np = np_;
    double* dX = (double*)small_.p + 8 * np_;   // 4 np doubles (2 complex columns)
    double* dY = dX + 4 * np_;
    std::vector<double> X(4 * np, 0.0), Y(4 * np);
    auto apply = [&](bool herm) {
      FX_CUDA(cudaMemcpyAsync(dX, X.data(), sizeof(double) * 4 * np, cudaMemcpyHostToDevice, stream_));
      double* in = dX;
      double* out = dY;
      if (!herm) {
        for (int k = (int)mats.size() - 1; k >= 0; --k) {
          launch_matvec2<T>(mats[k]->re() ? mats[k]->re() : zero_plane(), mats[k]->im(), np, in, out, stream_);
          ++launches_;
          std::swap(in, out);
        }
      } else {
        for (size_t k = 0; k < mats.size(); ++k) {
          launch_matvec2_h<T>(mats[k]->re() ? mats[k]->re() : zero_plane(), mats[k]->im(), np, in, out, stream_);
          launches_ += 2;
          std::swap(in, out);
        }
      }
      FX_CUDA(cudaMemcpyAsync(Y.data(), in, sizeof(double) * 4 * np, cudaMemcpyDeviceToHost, stream_));
      FX_CUDA(cudaStreamSynchronize(stream_));
    };
    if (n == 0) return 0.0;
    const int t = n > 1 ? 2 : 1;
    for (int64_t i = 0; i < n; ++i) {
      X[2 * i] = 1.0 / n;
      if (t == 2) X[2 * np + 2 * i] = probe_sign(i) / n;
    }
    double est_old = 0.0;
    std::vector<char> visited(n, 0);
    int64_t ind_best = 0;
    const int itmax = 5;
    for (int k = 1; k <= itmax; ++k) {
      apply(false);
      double col[2] = {0, 0};
      for (int c = 0; c < t; ++c)
        for (int64_t i = 0; i < n; ++i) col[c] += std::hypot(Y[c * 2 * np + 2 * i], Y[c * 2 * np + 2 * i + 1]);
      const int j = (t == 2 && col[1] > col[0]) ? 1 : 0;
      const double est = col[j];
      if (k >= 2 && est <= est_old) return est_old;
      est_old = est;
      if (k == itmax) break;
      // S = sign(Y)
      std::fill(X.begin(), X.end(), 0.0);
      for (int c = 0; c < t; ++c)
        for (int64_t i = 0; i < n; ++i) {
          const double a = Y[c * 2 * np + 2 * i], b = Y[c * 2 * np + 2 * i + 1];
          const double m = std::hypot(a, b);
          X[c * 2 * np + 2 * i] = m > 0 ? a / m : 1.0;
          X[c * 2 * np + 2 * i + 1] = m > 0 ? b / m : 0.0;
        }
      apply(true);
      std::vector<double> h(n);
      double hmax = 0;
      for (int64_t i = 0; i < n; ++i) {
        double v = 0;
        for (int c = 0; c < t; ++c) v = std::max(v, std::hypot(Y[c * 2 * np + 2 * i], Y[c * 2 * np + 2 * i + 1]));
        h[i] = v;
        hmax = std::max(hmax, v);
      }
      if (k >= 2 && hmax <= h[ind_best]) break;
      std::vector<int64_t> order(n);
      for (int64_t i = 0; i < n; ++i) order[i] = i;
      std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b2) { return h[a] > h[b2]; });
      std::vector<int64_t> picks;
      for (int64_t i : order) {
        if (!visited[i]) picks.push_back(i);
        if ((int)picks.size() == t) break;
      }
      if ((int)picks.size() < t) break;
      ind_best = picks[0];
      std::fill(X.begin(), X.end(), 0.0);
      for (int c = 0; c < t; ++c) {
        visited[picks[c]] = 1;
        X[c * 2 * np + 2 * picks[c]] = 1.0;
      }
    }
    return est_old;
  }

  T* zero_plane() {
    CM<T>& Z = slot_[kS2];
    launch_zero<T>(Z.ib, np_ * np_, stream_);
    ++launches_;
    return Z.ib;
  }

  // log2 ||(|Y|)^p||_1 for p = 0..maxp (index p), by normalised vector iterations.
  std::vector<double> abs_power_log2(int maxp) {
    const CM<T>& Y = slot_[kY];
    std::vector<double> out(maxp + 1, 0.0);
    double* dv = (double*)small_.p + 8 * np_;
    double* dw = dv + np_;
    std::vector<double> v(np_, 0.0);
    for (int64_t i = 0; i < n_; ++i) v[i] = 1.0;
    double logacc = 0.0;
    for (int p = 1; p <= maxp; ++p) {
      FX_CUDA(cudaMemcpyAsync(dv, v.data(), sizeof(double) * np_, cudaMemcpyHostToDevice, stream_));
      launch_vec_absmat<T>(Y.re() ? Y.re() : Y.im(), Y.re() ? Y.im() : nullptr, np_, dv, dw, stream_);
      launches_ += 2;
      FX_CUDA(cudaMemcpyAsync(v.data(), dw, sizeof(double) * np_, cudaMemcpyDeviceToHost, stream_));
      FX_CUDA(cudaStreamSynchronize(stream_));
      double mx = 0;
      for (double x : v) mx = std::max(mx, x);
      if (mx == 0.0) {
        for (int q = p; q <= maxp; ++q) out[q] = -INFINITY;
        return out;
      }
      for (double& x : v) x /= mx;
      logacc += std::log2(mx);
      out[p] = logacc;
    }
    return out;
  }

  // ---- blocked Cholesky G = L L^T (real SPD, in place) and R <- G^-1 R for the two planes of R.
  void chol_solve(T* G, T* rr, T* ri) {
    const int nb = kCholNb;
    const int64_t np = np_;
    T* Linv = (T*)chol_.p;               // block k at rows [k0, k0+nb), ld nb
    T* LinvT = Linv + (size_t)np * nb;
    T* P21 = LinvT + (size_t)np * nb;    // np x nb
    T* At = P21 + (size_t)np * nb;       // np x nb
    T* Btr = At + (size_t)np * nb;       // np x nb (two planes)
    T* Bti = Btr + (size_t)np * nb;
    for (int64_t k0 = 0; k0 < np; k0 += nb) {
      launch_potrf_inv<T>(G, np, k0, nb, Linv + k0 * nb, LinvT + k0 * nb, derr(), stream_);
      ++launches_;
      const int64_t rest = np - k0 - nb;
      if (rest <= 0) continue;
      T* G21 = G + (k0 + nb) * np + k0;
      // L21 = G21 L11^-T  (A = G21, Bt = L11^-1)
      cproduct(rest, nb, nb, G21, nullptr, np, Linv + k0 * nb, nullptr, nb, 1.0, nullptr, nullptr, nb, 0.0, 0.0,
               P21, nullptr, nb, false);
      FX_CUDA(cudaMemcpy2DAsync(G21, sizeof(T) * np, P21, sizeof(T) * nb, sizeof(T) * nb, rest,
                                cudaMemcpyDeviceToDevice, stream_));
      // G22 -= L21 L21^T  (symmetric result)
      T* G22 = G + (k0 + nb) * np + (k0 + nb);
      cproduct(rest, rest, nb, P21, nullptr, nb, P21, nullptr, nb, -1.0, G22, nullptr, np, 1.0, 0.0, G22, nullptr,
               np, true);
    }
    // Triangular solves by recursive halving: the off-diagonal updates are large-K
    // products, the leaves apply the inverted 128 x 128 diagonal blocks.
    CM<T>& Sc = slot_[kBt];   // transposed right-hand-side blocks (two planes, np x np)
    CM<T>& Sa = slot_[kS1];   // transposed L blocks
    fwd_solve(G, Linv, rr, ri, 0, np, Sc);
    bwd_solve(G, LinvT, rr, ri, 0, np, Sc, Sa);
  }

  // Rows [r0, r1) of R hold T; solve L[r0:r1, r0:r1] Z = T in place.
  void fwd_solve(const T* G, const T* Linv, T* rr, T* ri, int64_t r0, int64_t r1, CM<T>& Sc) {
    const int nb = kCholNb;
    const int64_t np = np_;
    if (r1 - r0 <= nb) {
      launch_transpose<T>(rr + r0 * np, np, Sc.rb, nb, nb, np, stream_);
      launch_transpose<T>(ri + r0 * np, np, Sc.ib, nb, nb, np, stream_);
      launches_ += 2;
      cproduct(nb, np, nb, Linv + r0 * nb, nullptr, nb, Sc.rb, Sc.ib, nb, 1.0, nullptr, nullptr, np, 0.0, 0.0,
               rr + r0 * np, ri + r0 * np, np, false);
      return;
    }
    const int64_t mid = r0 + ((r1 - r0) / nb / 2) * nb;
    fwd_solve(G, Linv, rr, ri, r0, mid, Sc);
    const int64_t K = mid - r0, M = r1 - mid;
    launch_transpose<T>(rr + r0 * np, np, Sc.rb, K, K, np, stream_);
    launch_transpose<T>(ri + r0 * np, np, Sc.ib, K, K, np, stream_);
    launches_ += 2;
    cproduct(M, np, K, G + mid * np + r0, nullptr, np, Sc.rb, Sc.ib, K, -1.0, rr + mid * np, ri + mid * np, np, 1.0,
             0.0, rr + mid * np, ri + mid * np, np, false);
    fwd_solve(G, Linv, rr, ri, mid, r1, Sc);
  }

  // Rows [r0, r1) of R hold Z; solve L^T[r0:r1, r0:r1] R = Z in place.
  void bwd_solve(const T* G, const T* LinvT, T* rr, T* ri, int64_t r0, int64_t r1, CM<T>& Sc, CM<T>& Sa) {
    const int nb = kCholNb;
    const int64_t np = np_;
    if (r1 - r0 <= nb) {
      launch_transpose<T>(rr + r0 * np, np, Sc.rb, nb, nb, np, stream_);
      launch_transpose<T>(ri + r0 * np, np, Sc.ib, nb, nb, np, stream_);
      launches_ += 2;
      cproduct(nb, np, nb, LinvT + r0 * nb, nullptr, nb, Sc.rb, Sc.ib, nb, 1.0, nullptr, nullptr, np, 0.0, 0.0,
               rr + r0 * np, ri + r0 * np, np, false);
      return;
    }
    const int64_t mid = r0 + ((r1 - r0) / nb / 2) * nb;
    bwd_solve(G, LinvT, rr, ri, mid, r1, Sc, Sa);
    // Z[r0:mid] -= L[mid:r1, r0:mid]^T R[mid:r1]
    const int64_t M = mid - r0, K = r1 - mid;
    launch_transpose<T>(G + mid * np + r0, np, Sa.rb, K, K, M, stream_);   // (M x K) = L block^T
    launch_transpose<T>(rr + mid * np, np, Sc.rb, K, K, np, stream_);
    launch_transpose<T>(ri + mid * np, np, Sc.ib, K, K, np, stream_);
    launches_ += 3;
    cproduct(M, np, K, Sa.rb, nullptr, K, Sc.rb, Sc.ib, K, -1.0, rr + r0 * np, ri + r0 * np, np, 1.0, 0.0,
             rr + r0 * np, ri + r0 * np, np, false);
    bwd_solve(G, LinvT, rr, ri, r0, mid, Sc, Sa);
  }

  // ---- blocked LU with partial pivoting and the two triangular solves (in place).
  void lu_solve(CM<T>& Q, CM<T>& P) {
    const int nb = 64;
    const int64_t np = np_;
    T* qr = Q.rb;
    T* qi = Q.hi ? Q.ib : nullptr;
    T* pr = P.rb;
    T* pi = P.hi ? P.ib : nullptr;
    int* ipiv = (int*)ipiv_.p;
    for (int64_t k0 = 0; k0 < np; k0 += nb) {
      launch_lu_panel<T>(qr, qi, np, k0, nb, ipiv, derr(), stream_);
      launch_row_swaps<T>(qr, qi, np, 0, k0, ipiv, k0, nb, stream_);
      launch_row_swaps<T>(qr, qi, np, k0 + nb, np, ipiv, k0, nb, stream_);
      launch_row_swaps<T>(pr, pi, np, 0, np, ipiv, k0, nb, stream_);
      launches_ += 4;
      const int64_t rest = np - k0 - nb;
      if (rest > 0) {
        launch_trsm_lower_unit<T>(qr, qi, np, k0, nb, qr, qi, np, k0 + nb, rest, stream_);
        ++launches_;
        // Q22 -= L21 U12
        sub_product(rest, rest, nb, qr + (k0 + nb) * np + k0, qi ? qi + (k0 + nb) * np + k0 : nullptr,
                    qr + k0 * np + (k0 + nb), qi ? qi + k0 * np + (k0 + nb) : nullptr,
                    qr + (k0 + nb) * np + (k0 + nb), qi ? qi + (k0 + nb) * np + (k0 + nb) : nullptr);
      }
    }
    // forward: L Y = P
    for (int64_t k0 = 0; k0 < np; k0 += nb) {
      launch_trsm_lower_unit<T>(qr, qi, np, k0, nb, pr, pi, np, 0, np, stream_);
      ++launches_;
      const int64_t rest = np - k0 - nb;
      if (rest > 0)
        sub_product(rest, np, nb, qr + (k0 + nb) * np + k0, qi ? qi + (k0 + nb) * np + k0 : nullptr,
                    pr + k0 * np, pi ? pi + k0 * np : nullptr, pr + (k0 + nb) * np,
                    pi ? pi + (k0 + nb) * np : nullptr);
    }
    // backward: U R = Y
    for (int64_t k0 = np - nb; k0 >= 0; k0 -= nb) {
      launch_trsm_upper<T>(qr, qi, np, k0, nb, pr, pi, np, 0, np, derr(), stream_);
      ++launches_;
      if (k0 > 0)
        sub_product(k0, np, nb, qr + k0, qi ? qi + k0 : nullptr, pr + k0 * np, pi ? pi + k0 * np : nullptr,
                    pr, pi);
    }
  }

  // D(M x N, ld np) -= A(M x K, ld np) * B(K x N, ld np), complex planar (imag may be null).
  void sub_product(int64_t M, int64_t N, int64_t K, const T* ar, const T* ai, const T* br,
                   const T* bi, T* dr, T* di) {
    // Right factor transposed into scratch: N x K, ld K.
    T* btr = (T*)panel_t_.p;
    T* bti = btr + (size_t)np_ * kPanel;
    if (N > np_ || K > kPanel) throw Error{FX_ERR_VALUE, "sub_product: block too large"};
    launch_transpose<T>(br, np_, btr, K, K, N, stream_);
    if (bi) launch_transpose<T>(bi, np_, bti, K, K, N, stream_);
    launches_ += bi ? 2 : 1;
    cproduct(M, N, K, ar, ai, np_, btr, bi ? bti : nullptr, K, -1.0, dr, di, np_, 1.0, 0.0, dr, di, np_, false);
  }
};

}  // namespace
}  // namespace fx

// ================================================================== C ABI
struct fx_engine {
  int64_t n = 0;
  int dtype = FX_C64;
  bool freed = false;
  std::unique_ptr<fx::Pipeline<float>> p32;
  std::unique_ptr<fx::Pipeline<double>> p64;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  void* h_in = nullptr;   // device staging for host runs
  void* h_out = nullptr;
  void* h_psi = nullptr;
  bool u_valid = false;   // h_out holds the U of the last fx_walk_host
  size_t elem = 8;
  fx::BatchPipeline* grouped = nullptr;   // grouped pipeline for walk generators (lazy)
  void* check_buf = nullptr;              // input statistics of the routing check
  fx::HostStage stage;                    // page-locked chunks for copies of host buffers
  fx::RunOpts opts{FX_FORM_PLAIN, 2, 1, -1, -1, 2000, 1, 0, 0, 0, -1, fx::kMixedN4, fx::kMixedN3, fx::kMixedPade,
                      fx::kMixedNewton, 0, 0, 0};
  fx_stats stats{};
  std::string last_error;
};

namespace {
std::mutex g_err_mu;
std::string g_last_error;

int fail(fx_handle h, const fx::Error& e) {
  if (h) h->last_error = e.msg;
  std::lock_guard<std::mutex> lk(g_err_mu);
  g_last_error = e.msg;
  return e.code;
}

size_t elem_size(int dtype) {
  switch (dtype) {
    case FX_F32: return 4;
    case FX_F64: return 8;
    case FX_C64: return 8;
    case FX_C128: return 16;
  }
  return 0;
}

template <typename F>
int guarded(fx_handle h, F&& f) {
  try {
    f();
    return FX_OK;
  } catch (const fx::Error& e) {
    return fail(h, e);
  } catch (const std::bad_alloc&) {
    return fail(h, fx::Error{FX_ERR_NOMEM, "host allocation failed"});
  } catch (const std::exception& e) {
    return fail(h, fx::Error{FX_ERR_CUDA, e.what()});
  }
}

// FP64 masters for the int8 (plain) and FP64 forms; FP32 masters for the BF16 (mixed) and
// CUDA-core FP32 (simt) forms of complex64 / float32 handles.  Allocated on first use.
void ensure_pipeline(fx_handle h) {
  const bool single = h->dtype == FX_C64 || h->dtype == FX_F32;
  const bool want32 = single && (h->opts.form == FX_FORM_MIXED || h->opts.form == FX_FORM_SIMT);
  if (want32 && !h->p32) {
    h->p64.reset();
    h->p32.reset(new fx::Pipeline<float>(h->n, h->dtype));
  } else if (!want32 && !h->p64) {
    h->p32.reset();
    h->p64.reset(new fx::Pipeline<double>(h->n, h->dtype));
  }
}

// Walk generators X = i*(real symmetric) in complex storage with the default plain-form options
// run through the grouped pipeline (fx_batch.cu) as a batch of one: blocked Cholesky of
// Q^H Q, explicit triangular inverse and triangle-aware products for the Pade solve, and
// device-side norm estimation (no host round trips after the selection).  Everything else
// (general complex or real inputs, other forms or options) runs the pipeline of this file.
bool grouped_eligible(fx_handle h) {
  const fx::RunOpts& o = h->opts;
  return (h->dtype == FX_C64 || h->dtype == FX_C128) && (o.form == FX_FORM_PLAIN || o.form == FX_FORM_MIXED) &&
         o.shift == 2 && o.structure == 1 && o.ipe == 1 && o.debug_stage == 0 && o.force_m < 0 && o.force_s < 0;
}
bool input_is_walk_generator(fx_handle h, const void* dA, cudaStream_t s) {
  const int64_t n = h->n;
  if (!h->check_buf) fx::dev_malloc(&h->check_buf, sizeof(double) * (6 * (size_t)n + 16));
  double* b = (double*)h->check_buf;
  fx::InputStats is{b, b + 2 * n, b + 4 * n, (int*)(b + 6 * n)};
  FX_CUDA(cudaMemsetAsync(is.flags, 0, sizeof(int) * 8, s));
  fx::launch_input_stats(dA, h->dtype, n, is, s);
  int f[8];
  FX_CUDA(cudaMemcpyAsync(f, is.flags, sizeof(int) * 8, cudaMemcpyDeviceToHost, s));
  FX_CUDA(cudaStreamSynchronize(s));
  if (f[4]) throw fx::Error{FX_ERR_NONFINITE, "input contains NaN or Inf"};
  return !f[0] && !f[2];
}

void run_device(fx_handle h, const void* dA, void* dU, const void* dpsi0, void* dpsi, cudaStream_t s) {
  if (h->freed) throw fx::Error{FX_ERR_FREED, "handle was freed"};
  if (h->n == 0) return;
  if (grouped_eligible(h) && fx_device_ok() && input_is_walk_generator(h, dA, s)) {
    if (!h->grouped) h->grouped = fx::batch_pipeline_create(h->n, h->dtype);
    FX_CUDA(cudaEventRecord(h->ev0, s));
    fx::PipeOpts po;
    po.profile = h->opts.profile != 0;
    po.timeout_ms = h->opts.timeout_ms;
    po.selector = h->opts.selector;
    po.inject_stall = h->opts.inject_stall;
    po.form = h->opts.form;
    po.sq_n4 = h->opts.sq_n4;
    po.sq_n3 = h->opts.sq_n3;
    po.pade_slices = h->opts.pade_slices;
    po.newton_slices = h->opts.newton_slices;
    po.solve = h->opts.solve;
    po.approx = h->opts.approx;
    po.drift = h->opts.drift != 0;
    fx::batch_pipeline_run(h->grouped, dA, dpsi0, dpsi, dU, po, s);
    FX_CUDA(cudaEventRecord(h->ev1, s));
    FX_CUDA(cudaEventSynchronize(h->ev1));
    float ms = 0;
    FX_CUDA(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
    h->stats = fx_stats{};
    fx::batch_pipeline_stats(h->grouped, &h->stats);
    h->stats.form = h->opts.form;
    h->stats.ms_total = ms;
    return;
  }
  ensure_pipeline(h);
  FX_CUDA(cudaEventRecord(h->ev0, s));
  if (h->p32)
    h->p32->run(dA, dU, dpsi0, dpsi, h->opts, s, h->stats);
  else
    h->p64->run(dA, dU, dpsi0, dpsi, h->opts, s, h->stats);
  FX_CUDA(cudaEventRecord(h->ev1, s));
  FX_CUDA(cudaEventSynchronize(h->ev1));
  float ms = 0;
  FX_CUDA(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
  h->stats.ms_total = ms;
}
}  // namespace

extern "C" {

int fx_device_ok(void) {
  int cnt = 0;
  if (cudaGetDeviceCount(&cnt) != cudaSuccess || cnt == 0) {
    cudaGetLastError();
    return 0;
  }
  int dev = 0, major = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
  return major == 10 ? 1 : 0;
}

const char* fx_version(void) { return "fastctqw_b200 0.1 (sm_100a, tcgen05)"; }

double fx_gpu_memory_gb(void) {
  size_t fr = 0, tot = 0;
  if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
    cudaGetLastError();
    return -1.0;
  }
  return (double)(tot - fr) / 1e9;
}

int fx_create(size_t n, int dtype, fx_handle* out) {
  if (!out) return fail(nullptr, fx::Error{FX_ERR_VALUE, "null output handle"});
  *out = nullptr;
  if (elem_size(dtype) == 0) return fail(nullptr, fx::Error{FX_ERR_TYPE, "unknown dtype"});
  if (n > (size_t)1 << 20) return fail(nullptr, fx::Error{FX_ERR_VALUE, "matrix order too large"});
  if (!fx_device_ok()) return fail(nullptr, fx::Error{FX_ERR_NODEV, "no sm_100 CUDA device"});
  fx_handle h = new (std::nothrow) fx_engine();
  if (!h) return fail(nullptr, fx::Error{FX_ERR_NOMEM, "host allocation failed"});
  int rc = guarded(h, [&] {
    h->n = (int64_t)n;
    h->dtype = dtype;
    h->elem = elem_size(dtype);
    FX_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    FX_CUDA(cudaEventCreate(&h->ev0));
    FX_CUDA(cudaEventCreate(&h->ev1));
    if (dtype == FX_C128 || dtype == FX_F64) h->opts.form = FX_FORM_FP64;
    // the general pipeline's workspace is allocated at the first run that needs it: walk
    // generators run the grouped pipeline instead
  });
  if (rc != FX_OK) {
    std::string msg = h->last_error;
    fx_destroy(h);
    std::lock_guard<std::mutex> lk(g_err_mu);
    g_last_error = msg;
    return rc;
  }
  *out = h;
  return FX_OK;
}

int fx_free(fx_handle h) {
  if (!h) return fail(nullptr, fx::Error{FX_ERR_VALUE, "null handle"});
  return guarded(h, [&] {
    h->p32.reset();
    h->p64.reset();
    if (h->grouped) fx::batch_pipeline_destroy(h->grouped);
    h->grouped = nullptr;
    if (h->check_buf) cudaFree(h->check_buf);
    h->check_buf = nullptr;
    if (h->h_in) cudaFree(h->h_in);
    if (h->h_out) cudaFree(h->h_out);
    if (h->h_psi) cudaFree(h->h_psi);
    h->h_in = h->h_out = h->h_psi = nullptr;
    h->stage.release();
    h->freed = true;
  });
}

int fx_destroy(fx_handle h) {
  if (!h) return FX_OK;
  fx_free(h);
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return FX_OK;
}

int fx_get_n(fx_handle h, size_t* n) {
  if (!h || !n) return fail(h, fx::Error{FX_ERR_VALUE, "null argument"});
  *n = (size_t)h->n;
  return FX_OK;
}

int fx_set_option(fx_handle h, int key, double value) {
  if (!h) return fail(nullptr, fx::Error{FX_ERR_VALUE, "null handle"});
  const int v = (int)value;
  switch (key) {
    case FX_OPT_FORM:
      if (v < FX_FORM_PLAIN || v > FX_FORM_FP64) return fail(h, fx::Error{FX_ERR_VALUE, "bad form"});
      if ((h->dtype == FX_C128 || h->dtype == FX_F64) && v == FX_FORM_MIXED)
        return fail(h, fx::Error{FX_ERR_VALUE, "the BF16 mixed form is for complex64/float32 handles"});
      if ((h->dtype == FX_C64 || h->dtype == FX_F32) && v == FX_FORM_FP64)
        return fail(h, fx::Error{FX_ERR_VALUE, "the FP64 form is for complex128/float64 handles"});
      h->opts.form = v;
      return FX_OK;
    case FX_OPT_SHIFT:
      if (v < 0 || v > 2) return fail(h, fx::Error{FX_ERR_VALUE, "shift must be 0, 1 or 2"});
      h->opts.shift = v;
      return FX_OK;
    case FX_OPT_STRUCTURE:
      if (v < 0 || v > 2) return fail(h, fx::Error{FX_ERR_VALUE, "structure must be 0, 1 or 2"});
      h->opts.structure = v;
      return FX_OK;
    case FX_OPT_FORCE_S: h->opts.force_s = v; return FX_OK;
    case FX_OPT_FORCE_M:
      if (v != -1 && v != 3 && v != 5 && v != 7 && v != 9 && v != 13)
        return fail(h, fx::Error{FX_ERR_VALUE, "Pade degree must be 3, 5, 7, 9 or 13"});
      h->opts.force_m = v;
      return FX_OK;
    case FX_OPT_TIMEOUT_MS:
      if (value < 1) return fail(h, fx::Error{FX_ERR_VALUE, "timeout must be >= 1 ms"});
      h->opts.timeout_ms = (unsigned)value;
      return FX_OK;
    case FX_OPT_IPE: h->opts.ipe = v != 0; return FX_OK;
    case FX_OPT_REFINE: return v == 0 ? FX_OK : fail(h, fx::Error{FX_ERR_VALUE, "refinement not available"});
    case FX_OPT_DEBUG_STAGE: h->opts.debug_stage = v; return FX_OK;
    case FX_OPT_PROFILE: h->opts.profile = v != 0; return FX_OK;
    case FX_OPT_SELECTOR:
      if (v < 0 || v > 3) return fail(h, fx::Error{FX_ERR_VALUE, "selector must be 0, 1, 2 or 3"});
      h->opts.selector = v;
      return FX_OK;
    case FX_OPT_INJECT_STALL:
      if (v < -1) return fail(h, fx::Error{FX_ERR_VALUE, "stall injection takes a launch index >= 0, or -1"});
      h->opts.inject_stall = v;
      return FX_OK;
    case FX_OPT_SQ_N4:
    case FX_OPT_SQ_N3:
      if (v < 0 || v > 64) return fail(h, fx::Error{FX_ERR_VALUE, "squaring counts must be 0..64"});
      (key == FX_OPT_SQ_N4 ? h->opts.sq_n4 : h->opts.sq_n3) = v;
      return FX_OK;
    case FX_OPT_DRIFT: h->opts.drift = v != 0; return FX_OK;
    case FX_OPT_PADE_SLICES:
      if (v != 3 && v != 4 && v != 5) return fail(h, fx::Error{FX_ERR_VALUE, "Pade slice count must be 3, 4 or 5"});
      h->opts.pade_slices = v;
      return FX_OK;
    case FX_OPT_SOLVE:
      if (v != 0 && v != 1 && v != 2) return fail(h, fx::Error{FX_ERR_VALUE, "solve must be 0, 1 or 2"});
      h->opts.solve = v;
      return FX_OK;
    case FX_OPT_NEWTON_SLICES:
      if (v != 3 && v != 4 && v != 5) return fail(h, fx::Error{FX_ERR_VALUE, "Newton slice count must be 3, 4 or 5"});
      h->opts.newton_slices = v;
      return FX_OK;
    case FX_OPT_APPROX:
      if (v != 0 && v != 1) return fail(h, fx::Error{FX_ERR_VALUE, "approximant must be 0 (Pade) or 1 (Chebyshev)"});
      h->opts.approx = v;
      return FX_OK;
  }
  return fail(h, fx::Error{FX_ERR_VALUE, "unknown option"});
}

int fx_product_profile(fx_handle h, int32_t* tags, double* ms, double* ops, int32_t cap, int32_t* count) {
  if (!h || !count || (cap > 0 && (!tags || !ms || !ops))) return fail(h, fx::Error{FX_ERR_VALUE, "null argument"});
  *count = 0;
  if (!h->grouped) return FX_OK;
  const std::vector<fx::ProdRecord>& v = fx::batch_pipeline_products(h->grouped);
  for (int32_t i = 0; i < cap && i < (int32_t)v.size(); ++i) {
    tags[i] = v[i].tag;
    ms[i] = v[i].ms;
    ops[i] = v[i].ops;
  }
  *count = (int32_t)v.size();
  return FX_OK;
}

int fx_spectral_radius(fx_handle h, double* rho_lanczos, double* rho_up) {
  if (!h || !rho_lanczos || !rho_up) return fail(h, fx::Error{FX_ERR_VALUE, "null argument"});
  *rho_lanczos = *rho_up = 0.0;
  if (h->grouped) fx::batch_pipeline_spectral(h->grouped, rho_lanczos, rho_up);
  return FX_OK;
}

int fx_unitarity_drift(fx_handle h, double* out, int32_t cap, int32_t* count) {
  if (!h || !count || (cap > 0 && !out)) return fail(h, fx::Error{FX_ERR_VALUE, "null argument"});
  *count = 0;
  if (!h->grouped) return FX_OK;
  const std::vector<double> v = fx::batch_pipeline_drift(h->grouped);
  for (int32_t i = 0; i < cap && i < (int32_t)v.size(); ++i) out[i] = v[i];
  *count = (int32_t)v.size();
  return FX_OK;
}

int fx_get_stats(fx_handle h, fx_stats* out) {
  if (!h || !out) return fail(h, fx::Error{FX_ERR_VALUE, "null argument"});
  *out = h->stats;
  return FX_OK;
}

const char* fx_last_error(fx_handle h) {
  if (h) return h->last_error.c_str();
  std::lock_guard<std::mutex> lk(g_err_mu);
  return g_last_error.c_str();
}

int fx_run_device(fx_handle h, const void* dA, void* dU, void* stream) {
  if (!h) return fail(nullptr, fx::Error{FX_ERR_VALUE, "null handle"});
  return guarded(h, [&] {
    cudaStream_t s = stream ? (cudaStream_t)stream : h->stream;
    run_device(h, dA, dU, nullptr, nullptr, s);
  });
}

int fx_walk_device(fx_handle h, const void* dA, const void* dpsi0, void* dpsi, void* dU, void* stream) {
  if (!h) return fail(nullptr, fx::Error{FX_ERR_VALUE, "null handle"});
  return guarded(h, [&] {
    cudaStream_t s = stream ? (cudaStream_t)stream : h->stream;
    run_device(h, dA, dU, dpsi0, dpsi, s);
  });
}

int fx_run_host(fx_handle h, const void* A, void* U) {
  if (!h) return fail(nullptr, fx::Error{FX_ERR_VALUE, "null handle"});
  return guarded(h, [&] {
    if (h->freed) throw fx::Error{FX_ERR_FREED, "handle was freed"};
    if (h->n == 0) return;
    const size_t bytes = (size_t)h->n * h->n * h->elem;
    if (!h->h_in) fx::dev_malloc(&h->h_in, bytes);
    if (!h->h_out) fx::dev_malloc(&h->h_out, bytes);
    {
      fx::NvtxRange nr("fx_run_host: copy in");
      h->stage.h2d(h->h_in, A, bytes, h->stream);
    }
    h->u_valid = false;
    {
      fx::NvtxRange nr("fx_run_host: expm");
      // the caller's output array is usually fresh (numpy allocates it untouched): its page
      // faults are taken on another thread while the device computes
      std::thread pre([U, bytes] { fx::prefault_host(U, bytes); });
      try {
        run_device(h, h->h_in, h->h_out, nullptr, nullptr, h->stream);
      } catch (...) {
        pre.join();
        throw;
      }
      pre.join();
    }
    fx::NvtxRange nr("fx_run_host: copy out");
    h->stage.d2h(U, h->h_out, bytes, h->stream);
  });
}

int fx_walk_host(fx_handle h, const void* A, const void* psi0, void* psi) {
  if (!h) return fail(nullptr, fx::Error{FX_ERR_VALUE, "null handle"});
  return guarded(h, [&] {
    if (h->freed) throw fx::Error{FX_ERR_FREED, "handle was freed"};
    if (h->n == 0) return;
    const size_t bytes = (size_t)h->n * h->n * h->elem;
    const size_t vbytes = (size_t)h->n * ((h->dtype == FX_C128 || h->dtype == FX_F64) ? 16 : 8);
    if (!h->h_in) fx::dev_malloc(&h->h_in, bytes);
    if (!h->h_out) fx::dev_malloc(&h->h_out, bytes);
    if (!h->h_psi) fx::dev_malloc(&h->h_psi, 2 * vbytes);
    char* dpsi0 = (char*)h->h_psi;
    char* dpsi = dpsi0 + vbytes;
    h->stage.h2d(h->h_in, A, bytes, h->stream);
    FX_CUDA(cudaMemcpyAsync(dpsi0, psi0, vbytes, cudaMemcpyHostToDevice, h->stream));
    h->u_valid = false;
    run_device(h, h->h_in, h->h_out, dpsi0, dpsi, h->stream);
    h->u_valid = true;
    FX_CUDA(cudaMemcpyAsync(psi, dpsi, vbytes, cudaMemcpyDeviceToHost, h->stream));
    FX_CUDA(cudaStreamSynchronize(h->stream));
  });
}

int fx_fetch_u(fx_handle h, void* U) {
  if (!h || !U) return fail(h, fx::Error{FX_ERR_VALUE, "null argument"});
  return guarded(h, [&] {
    if (h->freed) throw fx::Error{FX_ERR_FREED, "handle was freed"};
    if (h->n == 0) return;
    if (!h->u_valid || !h->h_out) throw fx::Error{FX_ERR_VALUE, "no walk result on the device"};
    const size_t bytes = (size_t)h->n * h->n * h->elem;
    h->stage.d2h(U, h->h_out, bytes, h->stream);
  });
}

}  // extern "C"
