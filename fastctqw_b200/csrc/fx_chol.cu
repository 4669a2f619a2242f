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

// Blocked form for nb a multiple of 32 (the 128-wide blocks of the grouped solve): far fewer
// CTA-wide barriers than the column loop above (about 25 instead of ~380 for nb = 128).
//   Panels of 32 columns, p = 0 .. nb/32 - 1:
//     warp 0 factors the 32 x 32 diagonal block D (right-looking, lane r owns row r, __syncwarp
//       between the steps) and inverts it (lane c owns column c of X_D = D^-1, forward
//       substitution; X_D goes to xd[p]);
//     the CTA solves the panel below, L_21 = G_21 X_D^T, and updates the trailing lower
//       triangle, G_22 -= L_21 L_21^T.
//   Off-diagonal blocks of X = L^-1 by distance d = q - p from the diagonal:
//     X_qp = -X_qq sum_{m=p..q-1} L_qm X_mp, stored transposed in the strict upper triangle of a.
// Shared memory: a (nb x (nb + 1)), xd (nb/32 blocks of 32 x 33), tmp (nb/32 - 1 blocks of
// 32 x 33): 190 KB for nb = 128 in FP64.
constexpr int kPB = 32;        // panel width
constexpr int kPLD = kPB + 1;  // padded leading dimension of the 32 x 32 buffers
template <typename T>
__device__ __forceinline__ void potrf_inv_block32(T* G, int64_t ld, int64_t k0, int nb, T* Linv, T* LinvT,
                                                  int* err, int* own_err = nullptr) {
  extern __shared__ unsigned char smem_raw[];
  const int sld = nb + 1, P = nb / kPB;
  T* a = reinterpret_cast<T*>(smem_raw);   // nb x sld
  T* xd = a + nb * sld;                     // P x (32 x 33)
  T* tmp = xd + P * kPB * kPLD;             // (P - 1) x (32 x 33)
  __shared__ int s_bad;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nth = blockDim.x;
  if (tid == 0) s_bad = 0;
  for (int idx = tid; idx < nb * nb; idx += nth) {
    const int i = idx / nb, j = idx - i * nb;
    a[i * sld + j] = G[(k0 + i) * ld + k0 + j];
  }
  __syncthreads();
  for (int p = 0; p < P; ++p) {
    const int p0 = p * kPB;
    if (warp == 0) {
      // ---- factor D = a[p0.., p0..] (lower), lane r = row p0 + r
      T* ar = a + (p0 + lane) * sld + p0;
      bool bad = false;
      for (int j = 0; j < kPB; ++j) {
        const T d = a[(p0 + j) * sld + p0 + j];
        if (!(d > (T)0)) {
          bad = true;
          break;
        }
        const T l = sqrt(d);
        __syncwarp();
        if (lane == j) ar[j] = l;
        else if (lane > j) ar[j] = ar[j] / l;
        __syncwarp();
        if (lane > j) {
          const T lrj = ar[j];
          for (int c = j + 1; c <= lane; ++c) ar[c] -= lrj * a[(p0 + c) * sld + p0 + j];
        }
        __syncwarp();
      }
      if (bad) {
        if (lane == 0) {
          atomicOr(err, kDevSingular);
          if (own_err) *own_err = 1;
          s_bad = 1;
        }
      } else {
        // ---- X_D = D^-1 (lower), lane c = column c
        T* x = xd + p * kPB * kPLD;
        const int c = lane;
        for (int i = 0; i < kPB; ++i) {
          if (i < c) {
            x[i * kPLD + c] = (T)0;
            continue;
          }
          const T lii = a[(p0 + i) * sld + p0 + i];
          if (i == c) {
            x[i * kPLD + c] = (T)1 / lii;
            continue;
          }
          T sum = (T)0;
          for (int m = c; m < i; ++m) sum += a[(p0 + i) * sld + p0 + m] * x[m * kPLD + c];
          x[i * kPLD + c] = -sum / lii;
        }
      }
    }
    __syncthreads();
    if (s_bad) return;
    const int rest = nb - p0 - kPB;
    if (rest <= 0) break;
    // ---- panel solve L_21 = G_21 X_D^T: outputs (r, c), r in [p0 + 32, nb), c in [0, 32)
    const T* x = xd + p * kPB * kPLD;
    constexpr int kMaxOut = 4;   // (128 - 32) x 32 / 1024 = 3 per thread at most
    T outv[kMaxOut];
    int cnt = 0;
    for (int idx = tid; idx < rest * kPB; idx += nth, ++cnt) {
      const int r = p0 + kPB + idx / kPB, c = idx % kPB;
      const T* g = a + r * sld + p0;
      T sum = (T)0;
      for (int m = 0; m <= c; ++m) sum += g[m] * x[c * kPLD + m];
      outv[cnt] = sum;
    }
    __syncthreads();
    cnt = 0;
    for (int idx = tid; idx < rest * kPB; idx += nth, ++cnt) {
      const int r = p0 + kPB + idx / kPB, c = idx % kPB;
      a[r * sld + p0 + c] = outv[cnt];
    }
    __syncthreads();
    // ---- trailing update of the lower triangle: a_rc -= sum_m L_rm L_cm, r >= c >= p0 + 32
    for (int idx = tid; idx < rest * rest; idx += nth) {
      const int r = p0 + kPB + idx / rest, c = p0 + kPB + idx % rest;
      if (c > r) continue;
      const T* lr = a + r * sld + p0;
      const T* lc = a + c * sld + p0;
      T sum = (T)0;
#pragma unroll 8
      for (int m = 0; m < kPB; ++m) sum += lr[m] * lc[m];
      a[r * sld + c] -= sum;
    }
    __syncthreads();
  }
  // ---- off-diagonal blocks of X = L^-1, X_qp (q > p) stored transposed: X_ic -> a[c][i]
  auto X_el = [&](int i, int c) -> T {   // X_ic for i >= c
    if (i / kPB == c / kPB) return xd[(i / kPB) * kPB * kPLD + (i % kPB) * kPLD + (c % kPB)];
    return a[c * sld + i];
  };
  for (int d = 1; d < P; ++d) {
    const int nblk = P - d;
    // T_p = sum_{m=p..q-1} L_qm X_mp for the blocks (q = p + d, p)
    for (int idx = tid; idx < nblk * kPB * kPB; idx += nth) {
      const int pb = idx / (kPB * kPB), e = idx % (kPB * kPB), i = e / kPB, c = e % kPB;
      const int q = pb + d, row = q * kPB + i, col = pb * kPB + c;
      T sum = (T)0;
      for (int m = col; m < q * kPB; ++m) sum += a[row * sld + m] * X_el(m, col);
      tmp[pb * kPB * kPLD + i * kPLD + c] = sum;
    }
    __syncthreads();
    // X_qp = -X_qq T_p
    for (int idx = tid; idx < nblk * kPB * kPB; idx += nth) {
      const int pb = idx / (kPB * kPB), e = idx % (kPB * kPB), i = e / kPB, c = e % kPB;
      const int q = pb + d;
      const T* xq = xd + q * kPB * kPLD;
      const T* t = tmp + pb * kPB * kPLD;
      T sum = (T)0;
      for (int m = 0; m <= i; ++m) sum += xq[i * kPLD + m] * t[m * kPLD + c];
      a[(pb * kPB + c) * sld + q * kPB + i] = -sum;
    }
    __syncthreads();
  }
  // ---- write L (zeros above the diagonal), X and X^T
  for (int idx = tid; idx < nb * nb; idx += nth) {
    const int i = idx / nb, j = idx - i * nb;
    G[(k0 + i) * ld + k0 + j] = j <= i ? a[i * sld + j] : (T)0;
    const T xv = j <= i ? X_el(i, j) : (T)0;
    Linv[i * nb + j] = xv;
    LinvT[j * nb + i] = xv;
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
  if (j.nb % kPB == 0)
    potrf_inv_block32<T>((T*)j.G, j.ld, j.k0, j.nb, (T*)j.Linv, (T*)j.LinvT, err, job_err ? job_err + j.tag : nullptr);
  else
    potrf_inv_block<T>((T*)j.G, j.ld, j.k0, j.nb, (T*)j.Linv, (T*)j.LinvT, err, job_err ? job_err + j.tag : nullptr);
}

}  // namespace

void prepare_potrf_inv_grouped() {
  static bool attr = false;
  if (!attr) {
    FX_CUDA(cudaFuncSetAttribute(k_potrf_inv_grouped<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 210 * 1024));
    attr = true;
  }
}

template <typename T>
void launch_potrf_inv_grouped(const GChol* jobs, int njobs, int* err, int* job_err, cudaStream_t s) {
  if (njobs <= 0) return;
  // the larger of the two block kernels' needs (nb = 128): a + xd + tmp of the blocked form
  const size_t sm = sizeof(T) * ((size_t)128 * 129 + (size_t)(4 + 3) * kPB * kPLD);
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
