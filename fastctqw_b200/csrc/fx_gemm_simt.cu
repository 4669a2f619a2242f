// CUDA-core (FFMA / DFMA) matrix product with the same operand convention as the
// tensor-core kernel: D = alpha * sum_t sign_t A_t Bt_t^T + beta C + gamma I.
//
// Used by the FP64 engine (complex128 / float64 handles) and as an independent on-device
// checker of the tcgen05 kernel.  128x128 tiles, 256 threads, 8x8 outputs per thread,
// K step 8, operand tiles transposed into shared memory so that the inner loop reads
// contiguous rows.
#include "fx_kernels.cuh"

namespace fx {
namespace {

constexpr int kBM = 128, kBN = 128, kBK = 8;
constexpr int kMaxTerms = 4;

template <typename T>
struct TermsArg {
  const T* a[kMaxTerms];
  const T* b[kMaxTerms];
  T sign[kMaxTerms];
  int n;
};

template <typename T>
__global__ void __launch_bounds__(256) k_gemm_simt(int64_t M, int64_t N, int64_t K, TermsArg<T> terms,
                                                   int64_t lda, int64_t ldb, T alpha, T beta,
                                                   const T* C, int64_t ldc, T gamma, T* D,
                                                   int64_t ldd) {
  __shared__ T As[kBK][kBM + 4];
  __shared__ T Bs[kBK][kBN + 4];
  const int tid = threadIdx.x;
  const int tx = tid % 16, ty = tid / 16;
  const int64_t m0 = (int64_t)blockIdx.y * kBM, n0 = (int64_t)blockIdx.x * kBN;
  T acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = (T)0;

  // Loader mapping: 256 threads x 4 elements = 128 rows x 8 k.
  const int lr = tid / 2, lk = (tid % 2) * 4;
  for (int t = 0; t < terms.n; ++t) {
    const T* A = terms.a[t];
    const T* B = terms.b[t];
    const T sg = terms.sign[t];
    for (int64_t k0 = 0; k0 < K; k0 += kBK) {
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int64_t kk = k0 + lk + q;
        const int64_t ra = m0 + lr, rb = n0 + lr;
        As[lk + q][lr] = (ra < M && kk < K) ? A[ra * lda + kk] * sg : (T)0;
        Bs[lk + q][lr] = (rb < N && kk < K) ? B[rb * ldb + kk] : (T)0;
      }
      __syncthreads();
#pragma unroll
      for (int kk = 0; kk < kBK; ++kk) {
        T a[8], b[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) a[i] = As[kk][ty * 8 + i];
#pragma unroll
        for (int j = 0; j < 8; ++j) b[j] = Bs[kk][tx * 8 + j];
#pragma unroll
        for (int i = 0; i < 8; ++i)
#pragma unroll
          for (int j = 0; j < 8; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
      }
      __syncthreads();
    }
  }
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int64_t r = m0 + ty * 8 + i;
    if (r >= M) continue;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int64_t c = n0 + tx * 8 + j;
      if (c >= N) continue;
      T v = alpha * acc[i][j];
      if (beta != (T)0) v += beta * C[r * ldc + c];
      if (r == c) v += gamma;
      D[r * ldd + c] = v;
    }
  }
}

}  // namespace

template <typename T>
void launch_gemm_simt(int64_t M, int64_t N, int64_t K, const GemmTerm<T>* terms, int nterms,
                      int64_t lda, int64_t ldb, double alpha, double beta, const T* C,
                      int64_t ldc, double gamma, T* D, int64_t ldd, cudaStream_t s) {
  if (nterms < 0 || nterms > kMaxTerms) throw Error{FX_ERR_VALUE, "too many product terms"};
  if (M <= 0 || N <= 0) return;
  TermsArg<T> ta{};
  ta.n = nterms;
  for (int i = 0; i < nterms; ++i) {
    ta.a[i] = terms[i].a;
    ta.b[i] = terms[i].b;
    ta.sign[i] = (T)terms[i].sign;
  }
  dim3 grid(cdiv(N, kBN), cdiv(M, kBM));
  k_gemm_simt<T><<<grid, 256, 0, s>>>(M, N, K, ta, lda, ldb, (T)alpha, (T)beta, C, ldc, (T)gamma,
                                      D, ldd);
  FX_LAUNCH_CHECK();
}

template void launch_gemm_simt<float>(int64_t, int64_t, int64_t, const GemmTerm<float>*, int,
                                      int64_t, int64_t, double, double, const float*, int64_t,
                                      double, float*, int64_t, cudaStream_t);
template void launch_gemm_simt<double>(int64_t, int64_t, int64_t, const GemmTerm<double>*, int,
                                       int64_t, int64_t, double, double, const double*, int64_t,
                                       double, double*, int64_t, cudaStream_t);

}  // namespace fx
