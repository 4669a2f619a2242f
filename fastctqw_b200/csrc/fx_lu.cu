// Pivoted LU pieces for the Pade solve Q X = P (planar complex).
//
// The blocked right-looking factorisation is driven from the host (fx_engine.cu): a panel
// of nb columns is factored here with partial pivoting, the interchanges are applied to
// the rest of the rows, U12 comes from a unit-lower triangular solve, and the trailing
// update A22 -= L21 U12 goes through the matrix-product kernels.  Pivot choice follows
// LAPACK's getrf: the largest |Re| + |Im| in the column, first index on ties.
#include "fx_kernels.cuh"

namespace fx {
namespace {

template <typename T>
__device__ __forceinline__ T cabs1(T a, T b) {
  return fabs(a) + fabs(b);
}

// One CTA factors the panel in global memory (the panel is L2-resident).
template <typename T>
__global__ void __launch_bounds__(1024) k_lu_panel(T* re, T* im, int64_t np, int64_t k0, int nb,
                                                   int* ipiv, int* err) {
  __shared__ T s_val[32];
  __shared__ int s_idx[32];
  __shared__ T s_prow_re[128], s_prow_im[128];
  __shared__ int s_piv;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t kend = (k0 + nb < np) ? k0 + nb : np;
  for (int64_t j = k0; j < kend; ++j) {
    // --- pivot search over rows j..np-1 of column j
    T best = (T)-1;
    int64_t bidx = np;
    for (int64_t i = j + tid; i < np; i += blockDim.x) {
      T v = cabs1(re[i * np + j], im ? im[i * np + j] : (T)0);
      if (v > best || (v == best && i < bidx)) {
        best = v;
        bidx = i;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      T ov = __shfl_xor_sync(0xffffffffu, best, o);
      int64_t oi = __shfl_xor_sync(0xffffffffu, bidx, o);
      if (ov > best || (ov == best && oi < bidx)) {
        best = ov;
        bidx = oi;
      }
    }
    if (lane == 0) {
      s_val[warp] = best;
      s_idx[warp] = (int)bidx;
    }
    __syncthreads();
    if (warp == 0) {
      const int nw = blockDim.x >> 5;
      best = lane < nw ? s_val[lane] : (T)-1;
      bidx = lane < nw ? s_idx[lane] : np;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        T ov = __shfl_xor_sync(0xffffffffu, best, o);
        int64_t oi = __shfl_xor_sync(0xffffffffu, bidx, o);
        if (ov > best || (ov == best && oi < bidx)) {
          best = ov;
          bidx = oi;
        }
      }
      if (lane == 0) {
        if (bidx >= np) bidx = j;
        s_piv = (int)bidx;
        ipiv[j] = (int)bidx;
        if (!(best > (T)0)) atomicOr(err, kDevSingular);
      }
    }
    __syncthreads();
    const int64_t p = s_piv;
    // --- swap rows j and p inside the panel columns, stage the pivot row in smem
    for (int64_t c = k0 + tid; c < kend; c += blockDim.x) {
      T a = re[j * np + c], b = re[p * np + c];
      re[j * np + c] = b;
      re[p * np + c] = a;
      s_prow_re[c - k0] = b;
      if (im) {
        T ai = im[j * np + c], bi = im[p * np + c];
        im[j * np + c] = bi;
        im[p * np + c] = ai;
        s_prow_im[c - k0] = bi;
      } else {
        s_prow_im[c - k0] = (T)0;
      }
    }
    __syncthreads();
    // --- scale below the pivot and rank-1 update of the remaining panel columns
    const T pr = s_prow_re[j - k0], pi = s_prow_im[j - k0];
    const T den = pr * pr + pi * pi;
    if (den > (T)0) {
      const T inv_r = pr / den, inv_i = -pi / den;  // 1 / pivot
      for (int64_t i = j + 1 + tid; i < np; i += blockDim.x) {
        T ar = re[i * np + j], ai = im ? im[i * np + j] : (T)0;
        T lr = ar * inv_r - ai * inv_i;
        T li = ar * inv_i + ai * inv_r;
        re[i * np + j] = lr;
        if (im) im[i * np + j] = li;
        for (int64_t c = j + 1; c < kend; ++c) {
          T ur = s_prow_re[c - k0], ui = s_prow_im[c - k0];
          re[i * np + c] -= lr * ur - li * ui;
          if (im) im[i * np + c] -= lr * ui + li * ur;
        }
      }
    }
    __syncthreads();
  }
}

// Row interchanges for columns [c0, c1): one thread per column, swaps applied in order.
template <typename T>
__global__ void k_row_swaps(T* re, T* im, int64_t ld, int64_t c0, int64_t c1, const int* ipiv,
                            int64_t k0, int nb) {
  const int64_t c = c0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= c1) return;
  for (int k = 0; k < nb; ++k) {
    const int64_t j = k0 + k, p = ipiv[j];
    if (p != j) {
      T a = re[j * ld + c];
      re[j * ld + c] = re[p * ld + c];
      re[p * ld + c] = a;
      if (im) {
        T b = im[j * ld + c];
        im[j * ld + c] = im[p * ld + c];
        im[p * ld + c] = b;
      }
    }
  }
}

// B <- L^-1 B, L unit lower nb x nb; one thread per column of B.
template <typename T>
__global__ void k_trsm_lower_unit(const T* lre, const T* lim, int64_t ldl, int64_t r0, int nb,
                                  T* bre, T* bim, int64_t ldb, int64_t c0, int64_t cols) {
  extern __shared__ unsigned char smem_raw[];
  T* sl_re = reinterpret_cast<T*>(smem_raw);
  T* sl_im = sl_re + nb * nb;
  for (int idx = threadIdx.x; idx < nb * nb; idx += blockDim.x) {
    const int i = idx / nb, k = idx % nb;
    sl_re[idx] = lre[(r0 + i) * ldl + r0 + k];
    sl_im[idx] = lim ? lim[(r0 + i) * ldl + r0 + k] : (T)0;
  }
  __syncthreads();
  const int64_t c = c0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= c0 + cols) return;
  for (int i = 1; i < nb; ++i) {
    T ar = bre[(r0 + i) * ldb + c], ai = bim ? bim[(r0 + i) * ldb + c] : (T)0;
    for (int k = 0; k < i; ++k) {
      const T xr = bre[(r0 + k) * ldb + c], xi = bim ? bim[(r0 + k) * ldb + c] : (T)0;
      const T l_r = sl_re[i * nb + k], l_i = sl_im[i * nb + k];
      ar -= l_r * xr - l_i * xi;
      ai -= l_r * xi + l_i * xr;
    }
    bre[(r0 + i) * ldb + c] = ar;
    if (bim) bim[(r0 + i) * ldb + c] = ai;
  }
}

// B <- U^-1 B, U upper non-unit nb x nb; one thread per column of B.
template <typename T>
__global__ void k_trsm_upper(const T* ure, const T* uim, int64_t ldu, int64_t r0, int nb, T* bre,
                             T* bim, int64_t ldb, int64_t c0, int64_t cols, int* err) {
  extern __shared__ unsigned char smem_raw[];
  T* su_re = reinterpret_cast<T*>(smem_raw);
  T* su_im = su_re + nb * nb;
  for (int idx = threadIdx.x; idx < nb * nb; idx += blockDim.x) {
    const int i = idx / nb, k = idx % nb;
    su_re[idx] = ure[(r0 + i) * ldu + r0 + k];
    su_im[idx] = uim ? uim[(r0 + i) * ldu + r0 + k] : (T)0;
  }
  __syncthreads();
  const int64_t c = c0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= c0 + cols) return;
  for (int i = nb - 1; i >= 0; --i) {
    T ar = bre[(r0 + i) * ldb + c], ai = bim ? bim[(r0 + i) * ldb + c] : (T)0;
    for (int k = i + 1; k < nb; ++k) {
      const T xr = bre[(r0 + k) * ldb + c], xi = bim ? bim[(r0 + k) * ldb + c] : (T)0;
      const T u_r = su_re[i * nb + k], u_i = su_im[i * nb + k];
      ar -= u_r * xr - u_i * xi;
      ai -= u_r * xi + u_i * xr;
    }
    const T dr = su_re[i * nb + i], di = su_im[i * nb + i];
    const T den = dr * dr + di * di;
    if (!(den > (T)0)) {
      if (c == c0) atomicOr(err, kDevSingular);
      continue;
    }
    const T xr = (ar * dr + ai * di) / den, xi = (ai * dr - ar * di) / den;
    bre[(r0 + i) * ldb + c] = xr;
    if (bim) bim[(r0 + i) * ldb + c] = xi;
  }
}

}  // namespace

template <typename T>
void launch_lu_panel(T* re, T* im, int64_t np, int64_t k0, int nb, int* ipiv, int* err,
                     cudaStream_t s) {
  if (nb > 128) throw Error{FX_ERR_VALUE, "panel width above 128"};
  k_lu_panel<T><<<1, 1024, 0, s>>>(re, im, np, k0, nb, ipiv, err);
  FX_LAUNCH_CHECK();
}

template <typename T>
void launch_row_swaps(T* re, T* im, int64_t ld, int64_t c0, int64_t c1, const int* ipiv,
                      int64_t k0, int nb, cudaStream_t s) {
  if (c1 <= c0) return;
  k_row_swaps<T><<<cdiv(c1 - c0, 256), 256, 0, s>>>(re, im, ld, c0, c1, ipiv, k0, nb);
  FX_LAUNCH_CHECK();
}

template <typename T>
void launch_trsm_lower_unit(const T* lre, const T* lim, int64_t ldl, int64_t r0, int nb, T* bre,
                            T* bim, int64_t ldb, int64_t c0, int64_t cols, cudaStream_t s) {
  if (cols <= 0) return;
  const size_t sm = 2 * sizeof(T) * nb * nb;
  if (sm > 48 * 1024)
    FX_CUDA(cudaFuncSetAttribute(k_trsm_lower_unit<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)sm));
  k_trsm_lower_unit<T><<<cdiv(cols, 128), 128, sm, s>>>(lre, lim, ldl, r0, nb, bre, bim, ldb, c0,
                                                      cols);
  FX_LAUNCH_CHECK();
}

template <typename T>
void launch_trsm_upper(const T* ure, const T* uim, int64_t ldu, int64_t r0, int nb, T* bre,
                       T* bim, int64_t ldb, int64_t c0, int64_t cols, int* err, cudaStream_t s) {
  if (cols <= 0) return;
  const size_t sm = 2 * sizeof(T) * nb * nb;
  if (sm > 48 * 1024)
    FX_CUDA(cudaFuncSetAttribute(k_trsm_upper<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)sm));
  k_trsm_upper<T><<<cdiv(cols, 128), 128, sm, s>>>(ure, uim, ldu, r0, nb, bre, bim, ldb, c0, cols,
                                                 err);
  FX_LAUNCH_CHECK();
}

#define FX_LU_INST(T)                                                                         \
  template void launch_lu_panel<T>(T*, T*, int64_t, int64_t, int, int*, int*, cudaStream_t); \
  template void launch_row_swaps<T>(T*, T*, int64_t, int64_t, int64_t, const int*, int64_t,   \
                                    int, cudaStream_t);                                       \
  template void launch_trsm_lower_unit<T>(const T*, const T*, int64_t, int64_t, int, T*, T*,  \
                                          int64_t, int64_t, int64_t, cudaStream_t);           \
  template void launch_trsm_upper<T>(const T*, const T*, int64_t, int64_t, int, T*, T*,       \
                                     int64_t, int64_t, int64_t, int*, cudaStream_t);

FX_LU_INST(float)
FX_LU_INST(double)

}  // namespace fx
