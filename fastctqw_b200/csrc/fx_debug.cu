// Diagnostic entry point: one real matrix product through the engine's product kernels, on
// caller-owned device buffers.  Used by the kernel tests (compared with a torch FP64 / FP32
// matmul) and by the benchmark's kernel-level roofline; not part of the walk path.
//
// form: FX_FORM_PLAIN (4 int8 slices, exact accumulation), 6 (the same in symmetric-output
// mode), 7 / 8 (5 slices, plain / symmetric), FX_FORM_MIXED (BF16 hi+lo), 4 (one BF16
// plane), 5 (three BF16 planes), FX_FORM_SIMT (CUDA-core FP32).
#include "fx_kernels.cuh"

#include <string>

namespace {
std::string g_dbg_err;
}

namespace fx {
// Message of the last failed diagnostic product call (read back by fx_product_error).
void set_product_error(const std::string& msg) { g_dbg_err = msg; }
}  // namespace fx

extern "C" {

int fx_product_f32(int form, int64_t M, int64_t N, int64_t K, const float* A, int64_t lda,
                   const float* Bt, int64_t ldb, float alpha, float beta, const float* C,
                   int64_t ldc, float gamma, float* D, int64_t ldd, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  void* scratch = nullptr;
  int* err = nullptr;
  try {
    FX_CUDA(cudaMalloc(&err, sizeof(int) * (1 + M + N)));
    FX_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
    if (form == FX_FORM_SIMT) {
      fx::GemmTerm<float> t{A, Bt, 1.f};
      fx::launch_gemm_simt<float>(M, N, K, &t, 1, lda, ldb, alpha, beta, C, ldc, gamma, D, ldd, s);
    } else if (form == FX_FORM_PLAIN || form == 6 || form == 7 || form == 8) {
      const int S = (form == 7 || form == 8) ? 5 : 4;
      const bool sym = form == 6 || form == 8;
      FX_CUDA(cudaMalloc(&scratch, S * (size_t)(M + N) * K));
      int8_t* sl = (int8_t*)scratch;
      fx::I8Slices sa{}, sb{};
      for (int q = 0; q < S; ++q) {
        sa.re[q] = sl + (size_t)q * M * K;
        sb.re[q] = sl + (size_t)S * M * K + (size_t)q * N * K;
      }
      sa.exp = err + 1;
      sb.exp = err + 1 + M;
      sa.ld = sb.ld = K;
      fx::launch_slice_rows<float>(S, A, nullptr, lda, M, K, sa, false, s);
      fx::launch_slice_rows<float>(S, Bt, nullptr, ldb, N, K, sb, false, s);
      fx::I8Term t{};
      for (int q = 0; q < S; ++q) {
        t.a[q] = sa.re[q];
        t.b[q] = sb.re[q];
      }
      fx::launch_gemm_i8<float>(S, M, N, K, &t, 1, K, K, sa.exp, sb.exp, alpha, beta, C, ldc, gamma, D, ldd,
                                sym, err, 2000, s);
    } else {
      const int P = form == FX_FORM_MIXED ? 2 : (form == 4 ? 1 : 3);
      const size_t asz = (size_t)M * K, bsz = (size_t)N * K;
      FX_CUDA(cudaMalloc(&scratch, sizeof(__nv_bfloat16) * P * (asz + bsz)));
      __nv_bfloat16* planes = (__nv_bfloat16*)scratch;
      __nv_bfloat16* ap[4] = {nullptr, nullptr, nullptr, nullptr};
      __nv_bfloat16* bp[4] = {nullptr, nullptr, nullptr, nullptr};
      for (int q = 0; q < P; ++q) {
        ap[q] = planes + q * asz;
        bp[q] = planes + P * asz + q * bsz;
      }
      fx::launch_split(A, lda, ap, P, K, M, K, false, s);
      fx::launch_split(Bt, ldb, bp, P, K, N, K, false, s);
      fx::TcTerm t{};
      for (int q = 0; q < 4; ++q) {
        t.a[q] = ap[q];
        t.b[q] = bp[q];
      }
      t.neg = 0;
      fx::TcOut out{};
      out.d = D;
      out.ldd = ldd;
      fx::launch_gemm_tc(M, N, K, &t, 1, P, K, K, alpha, beta, C, ldc, gamma, out, err, 2000, s);
    }
    int h_err = 0;
    FX_CUDA(cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, s));
    FX_CUDA(cudaStreamSynchronize(s));
    if (h_err) throw fx::Error{FX_ERR_TIMEOUT, "device wait timed out in the product kernel"};
  } catch (const fx::Error& e) {
    g_dbg_err = e.msg;
    if (scratch) cudaFree(scratch);
    if (err) cudaFree(err);
    return e.code;
  }
  if (scratch) cudaFree(scratch);
  if (err) cudaFree(err);
  return FX_OK;
}

// Diagnostic: the grouped int8 slicer on one block of rows of FP64 planes (device buffers).
// kind 0 / 1 picks the warp-per-row or the two-pass streaming kernel; S slices; split_diag
// leaves row r's element at column r out of the slices (single plane only) and writes it to dg;
// neg also writes the slices of -im.  out holds 3 S planes of rows x ldo bytes (re, im, -im).
int fx_slice_rows_f64(int kind, int S, const double* re, const double* im, int64_t ld, int64_t rows, int64_t K,
                      int split_diag, int neg, int8_t* out, int64_t ldo, int32_t* exps, double* dg, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  fx::GSlab* d_slab = nullptr;
  try {
    if ((kind != 0 && kind != 1) || S < 3 || S > 5 || !re || !out || !exps || rows <= 0 || K <= 0 || K > ld ||
        ldo < K || ldo % 16 != 0 || rows > (1 << 30) || K > (1 << 30) || (split_diag && (im || !dg)) ||
        (neg && !im))
      throw fx::Error{FX_ERR_VALUE, "fx_slice_rows_f64: invalid arguments"};
    fx::GSlab h{re, im, ld, (int)rows, (int)K, 0, split_diag ? 0 : fx::kNoDiag};
    const std::vector<int> plan = fx::slice_plan(std::vector<fx::GSlab>{h});
    // one allocation: the slab, then its block plan
    FX_CUDA(cudaMalloc(&d_slab, sizeof(fx::GSlab) + sizeof(int) * plan.size()));
    int* d_plan = reinterpret_cast<int*>(d_slab + 1);
    FX_CUDA(cudaMemcpyAsync(d_slab, &h, sizeof(h), cudaMemcpyHostToDevice, s));
    FX_CUDA(cudaMemcpyAsync(d_plan, plan.data(), sizeof(int) * plan.size(), cudaMemcpyHostToDevice, s));
    fx::I8Slices o{};
    const size_t plane = (size_t)rows * ldo;
    for (int q = 0; q < S; ++q) {
      o.re[q] = out + (size_t)q * plane;
      if (im) o.im[q] = out + (size_t)(S + q) * plane;
      if (neg) o.neg_im[q] = out + (size_t)(2 * S + q) * plane;
    }
    o.exp = exps;
    o.ld = ldo;
    o.dg = split_diag ? dg : nullptr;
    fx::launch_slice_rows_grouped<double>(S, d_slab, 1, rows, o, neg != 0, s, fx::SlicePlan{d_plan, plan.back()},
                                          kind);
    FX_CUDA(cudaStreamSynchronize(s));
  } catch (const fx::Error& e) {
    g_dbg_err = e.msg;
    if (d_slab) cudaFree(d_slab);
    return e.code;
  }
  cudaFree(d_slab);
  return FX_OK;
}

const char* fx_product_error(void) { return g_dbg_err.c_str(); }

}  // extern "C"
