// Diagonal-block kernel of the blocked Cholesky solve used for normal Pade denominators.
//
// For X = i*(real symmetric) the Pade numerator is P = conj(Q) = Q^H and the solve
// R = Q^-1 P becomes R = G^-1 (Q^H)^2 with G = Q^H Q = V^2 + W^2 real symmetric positive
// definite (V, W = even / odd Pade parts, commuting).  The blocked right-looking Cholesky
// G = L L^T is driven from the host: this kernel factors one nb x nb diagonal block in shared
// memory and also returns its inverse and the transpose of the inverse, so that the panel
// solve L21 = G21 L11^-T and both triangular solves of the right-hand sides run as
// tensor-core matrix products.
#include "fx_kernels.cuh"

namespace fx {
namespace {

// One CTA of 1024 threads: G_kk (rows/cols [k0, k0+nb), nb <= 128) -> L_kk in place (zeros
// above the diagonal), Linv = L_kk^-1 and LinvT = L_kk^-T (nb x nb, ld nb).
//
// The block lives in shared memory with a padded leading dimension (nb + 1), so that column
// walks (lanes on different rows) hit different banks.  Threads form a 32 x 32 grid; thread
// (ty, tx) owns the elements (ty + 32 a, tx + 32 b).
//   Cholesky, right-looking, one barrier per column: step j subtracts a_rj a_cj / a_jj from
//   every (r, c) with j < c <= r, reading the unscaled column j (no column of index <= j is
//   written after step j), and a last pass scales L_rc = a_rc / sqrt(a_cc).
//   Inverse, by rows: X_ii = 1 / L_ii, X_ic = -X_ii sum_{m=c..i-1} L_im X_mc (c < i), eight
//   threads per column reduce with shuffles; row i of X is stored transposed in the (unused)
//   strict upper triangle, X_ic -> a[c][i].
template <typename T>
__device__ __forceinline__ void potrf_inv_block(T* G, int64_t ld, int64_t k0, int nb, T* Linv, T* LinvT,
                                                int* err, int* own_err = nullptr) {
  extern __shared__ unsigned char smem_raw[];
  const int sld = nb + 1;
  T* a = reinterpret_cast<T*>(smem_raw);   // nb x sld
  T* xdiag = a + nb * sld;                  // nb
  __shared__ int s_bad;
  const int tid = threadIdx.x, tx = tid & 31, ty = tid >> 5;
  if (tid == 0) s_bad = 0;
  for (int idx = tid; idx < nb * nb; idx += 1024) {
    const int i = idx / nb, j = idx - i * nb;
    a[i * sld + j] = G[(k0 + i) * ld + k0 + j];
  }
  __syncthreads();
  for (int j = 0; j < nb; ++j) {
    const T d = a[j * sld + j];
    if (!(d > (T)0)) {
      if (tid == 0) {
        atomicOr(err, kDevSingular);
        if (own_err) *own_err = 1;
      }
      s_bad = 1;
      break;
    }
    const T inv_d = (T)1 / d;
#pragma unroll
    for (int ra = 0; ra < 4; ++ra) {
      const int r = ty + 32 * ra;
      if (r <= j || r >= nb) continue;
      const T ar = a[r * sld + j] * inv_d;
#pragma unroll
      for (int cb = 0; cb < 4; ++cb) {
        const int c = tx + 32 * cb;
        if (c > j && c <= r) a[r * sld + c] -= ar * a[c * sld + j];
      }
    }
    __syncthreads();
  }
  if (s_bad) return;
  // Scale: L_rc = a_rc / sqrt(a_cc) for r > c, L_cc = sqrt(a_cc).
  for (int idx = tid; idx < nb * nb; idx += 1024) {
    const int r = idx / nb, c = idx - r * nb;
    if (c < r) a[r * sld + c] /= sqrt(a[c * sld + c]);
  }
  __syncthreads();
  for (int c = tid; c < nb; c += 1024) {
    const T l = sqrt(a[c * sld + c]);
    a[c * sld + c] = l;
    xdiag[c] = (T)1 / l;
  }
  __syncthreads();
  // Write L back (zeros above the diagonal).
  for (int idx = tid; idx < nb * nb; idx += 1024) {
    const int i = idx / nb, j = idx - i * nb;
    G[(k0 + i) * ld + k0 + j] = j <= i ? a[i * sld + j] : (T)0;
  }
  // X = L^-1 row by row.
  const int c = tid >> 3, part = tid & 7;
  for (int i = 1; i < nb; ++i) {
    T sum = (T)0;
    if (c < i) {
      for (int m = c + part; m < i; m += 8) {
        const T xm = (m == c) ? xdiag[c] : a[c * sld + m];
        sum += a[i * sld + m] * xm;
      }
    }
    sum += __shfl_xor_sync(0xffffffffu, sum, 1);
    sum += __shfl_xor_sync(0xffffffffu, sum, 2);
    sum += __shfl_xor_sync(0xffffffffu, sum, 4);
    __syncthreads();   // every read of row i's inputs is done before a[c][i] is written
    if (c < i && part == 0) a[c * sld + i] = -sum * xdiag[i];
    __syncthreads();
  }
  for (int idx = tid; idx < nb * nb; idx += 1024) {
    const int i = idx / nb, j = idx - i * nb;
    const T x = j < i ? a[j * sld + i] : (j == i ? xdiag[i] : (T)0);
    Linv[i * nb + j] = x;
    LinvT[j * nb + i] = x;
  }
}

template <typename T>
__global__ void __launch_bounds__(1024) k_potrf_inv(T* G, int64_t ld, int64_t k0, int nb, T* Linv, T* LinvT,
                                                    int* err) {
  potrf_inv_block<T>(G, ld, k0, nb, Linv, LinvT, err);
}

// One CTA per job: the same block factorisation for many independent matrices.
template <typename T>
__global__ void __launch_bounds__(1024) k_potrf_inv_grouped(const GChol* jobs, int* err, int* job_err) {
  const GChol j = jobs[blockIdx.x];
  potrf_inv_block<T>((T*)j.G, j.ld, j.k0, j.nb, (T*)j.Linv, (T*)j.LinvT, err, job_err ? job_err + j.tag : nullptr);
}

}  // namespace

void prepare_potrf_inv_grouped() {
  static bool attr = false;
  if (!attr) {
    FX_CUDA(cudaFuncSetAttribute(k_potrf_inv_grouped<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 200 * 1024));
    attr = true;
  }
}

template <typename T>
void launch_potrf_inv_grouped(const GChol* jobs, int njobs, int* err, int* job_err, cudaStream_t s) {
  if (njobs <= 0) return;
  const size_t sm = sizeof(T) * ((size_t)128 * 129 + 128);
  prepare_potrf_inv_grouped();
  k_potrf_inv_grouped<T><<<njobs, 1024, sm, s>>>(jobs, err, job_err);
  FX_LAUNCH_CHECK();
}
template void launch_potrf_inv_grouped<double>(const GChol*, int, int*, int*, cudaStream_t);

template <typename T>
void launch_potrf_inv(T* G, int64_t ld, int64_t k0, int nb, T* Linv, T* LinvT, int* err, cudaStream_t s) {
  // nb x (nb + 1) block + the nb reciprocal diagonal entries.
  if (nb <= 0 || nb > 128) throw Error{FX_ERR_VALUE, "Cholesky block must be 1..128 wide"};
  const size_t sm = sizeof(T) * ((size_t)nb * (nb + 1) + nb);
  static bool attr = false;
  if (!attr) {
    FX_CUDA(cudaFuncSetAttribute(k_potrf_inv<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    attr = true;
  }
  k_potrf_inv<T><<<1, 1024, sm, s>>>(G, ld, k0, nb, Linv, LinvT, err);
  FX_LAUNCH_CHECK();
}

template void launch_potrf_inv<float>(float*, int64_t, int64_t, int, float*, float*, int*, cudaStream_t);
template void launch_potrf_inv<double>(double*, int64_t, int64_t, int, double*, double*, int*, cudaStream_t);

}  // namespace fx
