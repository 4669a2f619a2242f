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

// One CTA: G_kk (rows/cols [k0, k0+nb)) -> L_kk in place (zeros above the diagonal),
// Linv = L_kk^-1 and LinvT = L_kk^-T (nb x nb, ld nb).
template <typename T>
__global__ void __launch_bounds__(1024) k_potrf_inv(T* G, int64_t ld, int64_t k0, int nb, T* Linv, T* LinvT,
                                                    int* err) {
  extern __shared__ unsigned char smem_raw[];
  T* a = reinterpret_cast<T*>(smem_raw);  // nb x nb, row-major
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int idx = tid; idx < nb * nb; idx += nt) {
    const int i = idx / nb, j = idx % nb;
    a[idx] = G[(k0 + i) * ld + k0 + j];
  }
  __syncthreads();
  // Right-looking Cholesky (lower).
  for (int j = 0; j < nb; ++j) {
    const T d = a[j * nb + j];
    if (!(d > (T)0)) {
      if (tid == 0) atomicOr(err, kDevSingular);
      return;
    }
    const T ljj = sqrt(d);
    __syncthreads();
    for (int i = j + 1 + tid; i < nb; i += nt) a[i * nb + j] /= ljj;
    if (tid == 0) a[j * nb + j] = ljj;
    __syncthreads();
    const int rem = nb - j - 1;
    for (int idx = tid; idx < rem * rem; idx += nt) {
      const int i = j + 1 + idx / rem, c = j + 1 + idx % rem;
      if (c <= i) a[i * nb + c] -= a[i * nb + j] * a[c * nb + j];
    }
    __syncthreads();
  }
  // Write L back (zeros above the diagonal).
  for (int idx = tid; idx < nb * nb; idx += nt) {
    const int i = idx / nb, j = idx % nb;
    G[(k0 + i) * ld + k0 + j] = j <= i ? a[idx] : (T)0;
  }
  // Inverse of L by forward substitution, one warp per column of the identity, the column
  // being built in shared memory (batches of nwarps columns).
  __syncthreads();
  T* xs = a + nb * nb;  // nwarps x nb
  const int warp = tid / 32, lane = tid % 32, nwarps = nt / 32;
  for (int c0 = 0; c0 < nb; c0 += nwarps) {
    const int c = c0 + warp;
    if (c < nb) {
      T* x = xs + warp * nb;
      for (int i = 0; i < nb; ++i) {
        T part = (T)0;
        for (int m = c + lane; m < i; m += 32) part += a[i * nb + m] * x[m];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
        if (lane == 0) x[i] = (i < c) ? (T)0 : (((i == c) ? (T)1 : (T)0) - part) / a[i * nb + i];
        __syncwarp();
      }
      for (int i = lane; i < nb; i += 32) {
        Linv[i * nb + c] = x[i];
        LinvT[c * nb + i] = x[i];
      }
    }
    __syncthreads();
  }
}

}  // namespace

template <typename T>
void launch_potrf_inv(T* G, int64_t ld, int64_t k0, int nb, T* Linv, T* LinvT, int* err, cudaStream_t s) {
  // nb x nb block + one nb-column per warp (32 warps) for the inverse.
  const size_t sm = sizeof(T) * (size_t)nb * (nb + 32);
  if (sm > 200 * 1024) throw Error{FX_ERR_VALUE, "Cholesky block too large"};
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
