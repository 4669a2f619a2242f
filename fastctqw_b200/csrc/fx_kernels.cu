// Bandwidth-bound kernels of the expm engine: input statistics and shifts, norms and the
// 1-norm estimator's block products, elementwise combinations, BF16 splitting, transposes,
// the output map and the final U*psi0 product.
//
// All of these are HBM-bound passes over N^2 data.  Rows are read by whole warps (128-byte
// coalesced lines); column reductions use a row-chunked 2-stage sum (partials in a fixed
// order, then an ordered final sum) so that every result is bitwise reproducible.
#include "fx_kernels.cuh"

#include <cuComplex.h>

namespace fx {

namespace {

template <typename Tin>
struct In;
template <>
struct In<float> {
  static __device__ __forceinline__ void get(const float* p, int64_t i, double& re, double& im) {
    re = p[i];
    im = 0.0;
  }
};
template <>
struct In<double> {
  static __device__ __forceinline__ void get(const double* p, int64_t i, double& re, double& im) {
    re = p[i];
    im = 0.0;
  }
};
template <>
struct In<float2> {
  static __device__ __forceinline__ void get(const float2* p, int64_t i, double& re, double& im) {
    float2 v = p[i];
    re = v.x;
    im = v.y;
  }
};
template <>
struct In<double2> {
  static __device__ __forceinline__ void get(const double2* p, int64_t i, double& re, double& im) {
    double2 v = p[i];
    re = v.x;
    im = v.y;
  }
};

template <typename Tin, typename F>
void dispatch_in(const void* X, int dtype, F&& f) {
  switch (dtype) {
    case FX_F32: f((const float*)X); break;
    case FX_F64: f((const double*)X); break;
    case FX_C64: f((const float2*)X); break;
    case FX_C128: f((const double2*)X); break;
    default: throw Error{FX_ERR_TYPE, "unknown dtype"};
  }
}

__device__ __forceinline__ bool finite2(double a, double b) {
  return isfinite(a) && isfinite(b);
}

// ---- row sums, diagonal, Re/Im non-zero and finiteness flags: one warp per row.
template <typename Tin>
__global__ void k_row_stats(const Tin* X, int64_t n, double* rowsum, double* diag, int* flags) {
  const int lane = threadIdx.x & 31;
  const int64_t row = (int64_t)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  if (row >= n) return;
  double sr = 0.0, si = 0.0;
  bool re_nz = false, im_nz = false, bad = false;
  for (int64_t j = lane; j < n; j += 32) {
    double a, b;
    In<Tin>::get(X, row * n + j, a, b);
    sr += a;
    si += b;
    re_nz |= (a != 0.0);
    im_nz |= (b != 0.0);
    bad |= !finite2(a, b);
  }
  // Fixed-order butterfly: same result for the same data.
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    sr += __shfl_xor_sync(0xffffffffu, sr, o);
    si += __shfl_xor_sync(0xffffffffu, si, o);
  }
  unsigned any_re = __ballot_sync(0xffffffffu, re_nz);
  unsigned any_im = __ballot_sync(0xffffffffu, im_nz);
  unsigned any_bad = __ballot_sync(0xffffffffu, bad);
  if (lane == 0) {
    rowsum[2 * row] = sr;
    rowsum[2 * row + 1] = si;
    double a, b;
    In<Tin>::get(X, row * n + row, a, b);
    diag[2 * row] = a;
    diag[2 * row + 1] = b;
    if (any_re) atomicOr(&flags[0], 1);
    if (any_im) atomicOr(&flags[1], 1);
    if (any_bad) atomicOr(&flags[4], 1);
  }
}

// ---- column partial sums over row chunks, then an ordered final sum.
constexpr int kColChunks = 32;

template <typename Tin>
__global__ void k_col_partials_in(const Tin* X, int64_t n, int64_t rows_per_chunk, double* part) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const int64_t r0 = (int64_t)blockIdx.y * rows_per_chunk;
  const int64_t r1 = min(n, r0 + rows_per_chunk);
  double sr = 0.0, si = 0.0;
  for (int64_t i = r0; i < r1; ++i) {
    double a, b;
    In<Tin>::get(X, i * n + j, a, b);
    sr += a;
    si += b;
  }
  part[((int64_t)blockIdx.y * n + j) * 2] = sr;
  part[((int64_t)blockIdx.y * n + j) * 2 + 1] = si;
}

__global__ void k_col_finish2(const double* part, int chunks, int64_t n, double* out) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  double sr = 0.0, si = 0.0;
  for (int c = 0; c < chunks; ++c) {
    sr += part[((int64_t)c * n + j) * 2];
    si += part[((int64_t)c * n + j) * 2 + 1];
  }
  out[2 * j] = sr;
  out[2 * j + 1] = si;
}

__global__ void k_col_finish1(const double* part, int chunks, int64_t n, double* out) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  double s = 0.0;
  for (int c = 0; c < chunks; ++c) s += part[(int64_t)c * n + j];
  out[j] = s;
}

// ---- exact symmetry / skew-Hermitian test on 32x32 tile pairs.
template <typename Tin>
__global__ void k_sym_check(const Tin* X, int64_t n, int* flags) {
  __shared__ double t1r[32][33], t1i[32][33], t2r[32][33], t2i[32][33];
  const int bi = blockIdx.y, bj = blockIdx.x;
  if (bi > bj) return;
  const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
  for (int r = ty; r < 32; r += 8) {
    int64_t i = (int64_t)bi * 32 + r, j = (int64_t)bj * 32 + tx;
    double a = 0, b = 0;
    if (i < n && j < n) In<Tin>::get(X, i * n + j, a, b);
    t1r[r][tx] = a;
    t1i[r][tx] = b;
    i = (int64_t)bj * 32 + r;
    j = (int64_t)bi * 32 + tx;
    a = 0;
    b = 0;
    if (i < n && j < n) In<Tin>::get(X, i * n + j, a, b);
    t2r[r][tx] = a;
    t2i[r][tx] = b;
  }
  __syncthreads();
  bool nsym = false, nskew = false;
  for (int r = ty; r < 32; r += 8) {
    // t1[r][tx] = X[bi*32+r][bj*32+tx];  t2[tx][r] = X[bj*32+tx][bi*32+r]  (its transpose)
    double ar = t1r[r][tx], ai = t1i[r][tx], br = t2r[tx][r], bi2 = t2i[tx][r];
    nsym |= (ar != br) || (ai != bi2);
    nskew |= (ar != -br) || (ai != bi2);   // X_ij == -conj(X_ji)
  }
  if (__syncthreads_or(nsym) && tx == 0 && ty == 0) atomicOr(&flags[2], 1);
  if (__syncthreads_or(nskew) && tx == 0 && ty == 0) atomicOr(&flags[3], 1);
}

template <typename Tin, typename T>
__global__ void k_load_shifted(const Tin* X, int64_t n, int64_t np, double mu_re, double mu_im,
                               double nu_re, double nu_im, T* yre, T* yim) {
  const int64_t total = np * np;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = idx / np, j = idx - (idx / np) * np;
    double a = 0.0, b = 0.0;
    if (i < n && j < n) {
      In<Tin>::get(X, i * n + j, a, b);
      a -= nu_re;
      b -= nu_im;
      if (i == j) {
        a -= mu_re;
        b -= mu_im;
      }
    }
    yre[idx] = (T)a;
    if (yim) yim[idx] = (T)b;
  }
}

// ---- |M| column partials (deterministic), planar complex T.
template <typename T>
__global__ void k_colabs_partials(const T* re, const T* im, int64_t np, int64_t ld,
                                  int64_t rows_per_chunk, double* part) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= np) return;
  const int64_t r0 = (int64_t)blockIdx.y * rows_per_chunk;
  const int64_t r1 = min(np, r0 + rows_per_chunk);
  double s = 0.0;
  for (int64_t i = r0; i < r1; ++i) {
    double a = (double)re[i * ld + j];
    double b = im ? (double)im[i * ld + j] : 0.0;
    s += sqrt(a * a + b * b);
  }
  part[(int64_t)blockIdx.y * np + j] = s;
}

// ---- Y = M X for X: np x 2 complex (column-major, interleaved re/im), warp per row.
template <typename T>
__global__ void k_matvec2(const T* re, const T* im, int64_t np, const double* X, double* Y) {
  const int lane = threadIdx.x & 31;
  const int64_t row = (int64_t)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  if (row >= np) return;
  double y0r = 0, y0i = 0, y1r = 0, y1i = 0;
  for (int64_t j = lane; j < np; j += 32) {
    double a = (double)re[row * np + j];
    double b = im ? (double)im[row * np + j] : 0.0;
    double x0r = X[2 * j], x0i = X[2 * j + 1];
    double x1r = X[2 * np + 2 * j], x1i = X[2 * np + 2 * j + 1];
    y0r += a * x0r - b * x0i;
    y0i += a * x0i + b * x0r;
    y1r += a * x1r - b * x1i;
    y1i += a * x1i + b * x1r;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    y0r += __shfl_xor_sync(0xffffffffu, y0r, o);
    y0i += __shfl_xor_sync(0xffffffffu, y0i, o);
    y1r += __shfl_xor_sync(0xffffffffu, y1r, o);
    y1i += __shfl_xor_sync(0xffffffffu, y1i, o);
  }
  if (lane == 0) {
    Y[2 * row] = y0r;
    Y[2 * row + 1] = y0i;
    Y[2 * np + 2 * row] = y1r;
    Y[2 * np + 2 * row + 1] = y1i;
  }
}

// ---- Z = M^H S partials: Z_j = sum_i conj(M_ij) S_i, row-chunked.
template <typename T>
__global__ void k_matvec2_h_partials(const T* re, const T* im, int64_t np, const double* S,
                                     int64_t rows_per_chunk, double* part) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= np) return;
  const int64_t r0 = (int64_t)blockIdx.y * rows_per_chunk;
  const int64_t r1 = min(np, r0 + rows_per_chunk);
  double z0r = 0, z0i = 0, z1r = 0, z1i = 0;
  for (int64_t i = r0; i < r1; ++i) {
    double a = (double)re[i * np + j];
    double b = im ? -(double)im[i * np + j] : 0.0;  // conj
    double s0r = S[2 * i], s0i = S[2 * i + 1];
    double s1r = S[2 * np + 2 * i], s1i = S[2 * np + 2 * i + 1];
    z0r += a * s0r - b * s0i;
    z0i += a * s0i + b * s0r;
    z1r += a * s1r - b * s1i;
    z1i += a * s1i + b * s1r;
  }
  double* p = part + ((int64_t)blockIdx.y * np + j) * 4;
  p[0] = z0r;
  p[1] = z0i;
  p[2] = z1r;
  p[3] = z1i;
}

__global__ void k_matvec2_h_finish(const double* part, int chunks, int64_t np, double* Z) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= np) return;
  double z0r = 0, z0i = 0, z1r = 0, z1i = 0;
  for (int c = 0; c < chunks; ++c) {
    const double* p = part + ((int64_t)c * np + j) * 4;
    z0r += p[0];
    z0i += p[1];
    z1r += p[2];
    z1i += p[3];
  }
  Z[2 * j] = z0r;
  Z[2 * j + 1] = z0i;
  Z[2 * np + 2 * j] = z1r;
  Z[2 * np + 2 * j + 1] = z1i;
}

template <typename T>
__global__ void k_vec_absmat_partials(const T* re, const T* im, int64_t np, const double* v,
                                      int64_t rows_per_chunk, double* part) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= np) return;
  const int64_t r0 = (int64_t)blockIdx.y * rows_per_chunk;
  const int64_t r1 = min(np, r0 + rows_per_chunk);
  double s = 0.0;
  for (int64_t i = r0; i < r1; ++i) {
    double a = (double)re[i * np + j];
    double b = im ? (double)im[i * np + j] : 0.0;
    s += v[i] * sqrt(a * a + b * b);
  }
  part[(int64_t)blockIdx.y * np + j] = s;
}

template <typename T>
__global__ void k_combo(T* D, const T* M0, double c0, const T* M1, double c1, const T* M2,
                        double c2, const T* M3, double c3, double g, int64_t np) {
  const int64_t total = np * np;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    double v = 0.0;
    if (M0) v += c0 * (double)M0[idx];
    if (M1) v += c1 * (double)M1[idx];
    if (M2) v += c2 * (double)M2[idx];
    if (M3) v += c3 * (double)M3[idx];
    if (g != 0.0 && (idx / np) == (idx % np)) v += g;
    D[idx] = (T)v;
  }
}

template <typename T>
__global__ void k_zero(T* D, int64_t count) {
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < count;
       idx += (int64_t)gridDim.x * blockDim.x)
    D[idx] = (T)0;
}

template <typename T>
__global__ void k_transpose(const T* in, int64_t ld_in, T* out, int64_t ld_out, int64_t rows,
                            int64_t cols) {
  __shared__ T tile[32][33];
  const int64_t r0 = (int64_t)blockIdx.y * 32, c0 = (int64_t)blockIdx.x * 32;
  for (int r = threadIdx.y; r < 32; r += 8) {
    int64_t i = r0 + r, j = c0 + threadIdx.x;
    tile[r][threadIdx.x] = (i < rows && j < cols) ? in[i * ld_in + j] : (T)0;
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += 8) {
    int64_t i = c0 + r, j = r0 + threadIdx.x;  // out row = input column
    if (i < cols && j < rows) out[i * ld_out + j] = tile[threadIdx.x][r];
  }
}

__global__ void k_split(const float* in, int64_t ld_in, __nv_bfloat16* o0, __nv_bfloat16* o1,
                        __nv_bfloat16* o2, __nv_bfloat16* o3, int nparts, int64_t ld_out,
                        int64_t rows, int64_t cols) {
  const int64_t total = rows * cols;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = idx / cols, j = idx - (idx / cols) * cols;
    __nv_bfloat16 p[4];
    split_bf16(in[i * ld_in + j], p, nparts);
    const int64_t o = i * ld_out + j;
    o0[o] = p[0];
    if (nparts > 1) o1[o] = p[1];
    if (nparts > 2) o2[o] = p[2];
    if (nparts > 3) o3[o] = p[3];
  }
}

__global__ void k_split_t(const float* in, int64_t ld_in, __nv_bfloat16* o0, __nv_bfloat16* o1,
                          __nv_bfloat16* o2, __nv_bfloat16* o3, int nparts, int64_t ld_out,
                          int64_t rows, int64_t cols) {
  __shared__ float tile[32][33];
  const int64_t r0 = (int64_t)blockIdx.y * 32, c0 = (int64_t)blockIdx.x * 32;
  for (int r = threadIdx.y; r < 32; r += 8) {
    int64_t i = r0 + r, j = c0 + threadIdx.x;
    tile[r][threadIdx.x] = (i < rows && j < cols) ? in[i * ld_in + j] : 0.f;
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += 8) {
    int64_t i = c0 + r, j = r0 + threadIdx.x;
    if (i < cols && j < rows) {
      __nv_bfloat16 p[4];
      split_bf16(tile[threadIdx.x][r], p, nparts);
      const int64_t o = i * ld_out + j;
      o0[o] = p[0];
      if (nparts > 1) o1[o] = p[1];
      if (nparts > 2) o2[o] = p[2];
      if (nparts > 3) o3[o] = p[3];
    }
  }
}

template <typename Tout>
struct Out;
template <>
struct Out<float> {
  static __device__ __forceinline__ void put(float* p, int64_t i, double re, double) { p[i] = (float)re; }
};
template <>
struct Out<double> {
  static __device__ __forceinline__ void put(double* p, int64_t i, double re, double) { p[i] = re; }
};
template <>
struct Out<float2> {
  static __device__ __forceinline__ void put(float2* p, int64_t i, double re, double im) {
    p[i] = make_float2((float)re, (float)im);
  }
};
template <>
struct Out<double2> {
  static __device__ __forceinline__ void put(double2* p, int64_t i, double re, double im) {
    p[i] = make_double2(re, im);
  }
};

template <typename T, typename Tout>
__global__ void k_output(const T* ere, const T* eim, int64_t n, int64_t np, OutputMap om, Tout* U) {
  const int64_t total = n * n;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = idx / n, j = idx - (idx / n) * n;
    double a = (double)ere[i * np + j] + om.cj_re;
    double b = (eim ? (double)eim[i * np + j] : 0.0) + om.cj_im;
    if (om.ipe && i == j) a += 1.0;
    Out<Tout>::put(U, idx, om.emu_re * a - om.emu_im * b, om.emu_re * b + om.emu_im * a);
  }
}

template <typename Tps>
struct Psi;
template <>
struct Psi<float2> {
  static __device__ __forceinline__ void get(const float2* p, int64_t i, double& a, double& b) {
    a = p[i].x;
    b = p[i].y;
  }
};
template <>
struct Psi<double2> {
  static __device__ __forceinline__ void get(const double2* p, int64_t i, double& a, double& b) {
    a = p[i].x;
    b = p[i].y;
  }
};

// sum of psi0 (for the rank-one term), single block, fixed order.
template <typename Tps>
__global__ void k_psi_sum(const Tps* psi0, int64_t n, double* out) {
  __shared__ double sr[256], si[256];
  double a = 0, b = 0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
    double x, y;
    Psi<Tps>::get(psi0, i, x, y);
    a += x;
    b += y;
  }
  sr[threadIdx.x] = a;
  si[threadIdx.x] = b;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      sr[threadIdx.x] += sr[threadIdx.x + o];
      si[threadIdx.x] += si[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[0] = sr[0];
    out[1] = si[0];
  }
}

template <typename T, typename Tps>
__global__ void k_apply(const T* ere, const T* eim, int64_t n, int64_t np, OutputMap om,
                        const Tps* psi0, Tps* psi, const double* ssum) {
  const int lane = threadIdx.x & 31;
  const int64_t row = (int64_t)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  if (row >= n) return;
  double yr = 0, yi = 0;
  for (int64_t j = lane; j < n; j += 32) {
    double a = (double)ere[row * np + j];
    double b = eim ? (double)eim[row * np + j] : 0.0;
    double x, y;
    Psi<Tps>::get(psi0, j, x, y);
    yr += a * x - b * y;
    yi += a * y + b * x;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    yr += __shfl_xor_sync(0xffffffffu, yr, o);
    yi += __shfl_xor_sync(0xffffffffu, yi, o);
  }
  if (lane == 0) {
    double x, y;
    Psi<Tps>::get(psi0, row, x, y);
    if (om.ipe) {
      yr += x;
      yi += y;
    }
    yr += om.cj_re * ssum[0] - om.cj_im * ssum[1];
    yi += om.cj_re * ssum[1] + om.cj_im * ssum[0];
    Out<Tps>::put(psi, row, om.emu_re * yr - om.emu_im * yi, om.emu_re * yi + om.emu_im * yr);
  }
}

inline unsigned grid_for(int64_t total, int threads = 256) {
  int64_t b = (total + threads - 1) / threads;
  if (b > 148 * 16) b = 148 * 16;
  if (b < 1) b = 1;
  return (unsigned)b;
}

// Scratch for the column reductions (partials), grown on demand, per device context.
struct PartialBuf {
  double* p = nullptr;
  size_t bytes = 0;
  double* get(size_t need) {
    if (need > bytes) {
      if (p) cudaFree(p);
      p = nullptr;
      bytes = 0;
      if (cudaMalloc(&p, need) != cudaSuccess) throw Error{FX_ERR_NOMEM, "partials buffer"};
      bytes = need;
    }
    return p;
  }
};
thread_local PartialBuf g_part;

int64_t chunk_rows(int64_t rows, int chunks) { return (rows + chunks - 1) / chunks; }

}  // namespace

// =============================================================================== API

void launch_input_stats(const void* X, int dtype, int64_t n, InputStats st, cudaStream_t s) {
  dispatch_in<void>(X, dtype, [&](auto p) {
    using Tin = std::remove_const_t<std::remove_pointer_t<decltype(p)>>;
    k_row_stats<Tin><<<cdiv(n, 8), 256, 0, s>>>(p, n, st.rowsum, st.diag, st.flags);
    FX_LAUNCH_CHECK();
    const int64_t rpc = chunk_rows(n, kColChunks);
    double* part = g_part.get(sizeof(double) * 2 * n * kColChunks);
    k_col_partials_in<Tin><<<dim3(cdiv(n, 128), kColChunks), 128, 0, s>>>(p, n, rpc, part);
    FX_LAUNCH_CHECK();
    k_col_finish2<<<cdiv(n, 256), 256, 0, s>>>(part, kColChunks, n, st.colsum);
    FX_LAUNCH_CHECK();
    const unsigned nt = cdiv(n, 32);
    k_sym_check<Tin><<<dim3(nt, nt), dim3(32, 8), 0, s>>>(p, n, st.flags);
    FX_LAUNCH_CHECK();
  });
}

template <typename T>
void launch_load_shifted(const void* X, int dtype, int64_t n, int64_t np, double mu_re,
                         double mu_im, double nu_re, double nu_im, T* yre, T* yim,
                         cudaStream_t s) {
  dispatch_in<void>(X, dtype, [&](auto p) {
    using Tin = std::remove_const_t<std::remove_pointer_t<decltype(p)>>;
    k_load_shifted<Tin, T><<<grid_for(np * np), 256, 0, s>>>(p, n, np, mu_re, mu_im, nu_re,
                                                             nu_im, yre, yim);
    FX_LAUNCH_CHECK();
  });
}

template <typename T>
void launch_col_abs_sums(const T* re, const T* im, int64_t np, int64_t ld, double* colsum,
                         cudaStream_t s) {
  const int64_t rpc = chunk_rows(np, kColChunks);
  double* part = g_part.get(sizeof(double) * np * kColChunks);
  k_colabs_partials<T><<<dim3(cdiv(np, 128), kColChunks), 128, 0, s>>>(re, im, np, ld, rpc, part);
  FX_LAUNCH_CHECK();
  k_col_finish1<<<cdiv(np, 256), 256, 0, s>>>(part, kColChunks, np, colsum);
  FX_LAUNCH_CHECK();
}

template <typename T>
void launch_matvec2(const T* re, const T* im, int64_t np, const double* X, double* Y,
                    cudaStream_t s) {
  k_matvec2<T><<<cdiv(np, 8), 256, 0, s>>>(re, im, np, X, Y);
  FX_LAUNCH_CHECK();
}

template <typename T>
void launch_matvec2_h(const T* re, const T* im, int64_t np, const double* S, double* Z,
                      cudaStream_t s) {
  const int64_t rpc = chunk_rows(np, kColChunks);
  double* part = g_part.get(sizeof(double) * 4 * np * kColChunks);
  k_matvec2_h_partials<T><<<dim3(cdiv(np, 128), kColChunks), 128, 0, s>>>(re, im, np, S, rpc, part);
  FX_LAUNCH_CHECK();
  k_matvec2_h_finish<<<cdiv(np, 256), 256, 0, s>>>(part, kColChunks, np, Z);
  FX_LAUNCH_CHECK();
}

template <typename T>
void launch_vec_absmat(const T* re, const T* im, int64_t np, const double* v, double* w,
                       cudaStream_t s) {
  const int64_t rpc = chunk_rows(np, kColChunks);
  double* part = g_part.get(sizeof(double) * np * kColChunks);
  k_vec_absmat_partials<T><<<dim3(cdiv(np, 128), kColChunks), 128, 0, s>>>(re, im, np, v, rpc, part);
  FX_LAUNCH_CHECK();
  k_col_finish1<<<cdiv(np, 256), 256, 0, s>>>(part, kColChunks, np, w);
  FX_LAUNCH_CHECK();
}

template <typename T>
void launch_combo(T* D, const T* M0, double c0, const T* M1, double c1, const T* M2, double c2,
                  const T* M3, double c3, double g, int64_t np, cudaStream_t s) {
  k_combo<T><<<grid_for(np * np), 256, 0, s>>>(D, M0, c0, M1, c1, M2, c2, M3, c3, g, np);
  FX_LAUNCH_CHECK();
}

template <typename T>
void launch_zero(T* D, int64_t count, cudaStream_t s) {
  k_zero<T><<<grid_for(count), 256, 0, s>>>(D, count);
  FX_LAUNCH_CHECK();
}

template <typename T>
void launch_transpose(const T* in, int64_t ld_in, T* out, int64_t ld_out, int64_t rows,
                      int64_t cols, cudaStream_t s) {
  k_transpose<T><<<dim3(cdiv(cols, 32), cdiv(rows, 32)), dim3(32, 8), 0, s>>>(in, ld_in, out,
                                                                            ld_out, rows, cols);
  FX_LAUNCH_CHECK();
}

void launch_split(const float* in, int64_t ld_in, __nv_bfloat16* const* out, int nparts,
                  int64_t ld_out, int64_t rows, int64_t cols, bool transpose, cudaStream_t s) {
  __nv_bfloat16* o[4] = {out[0], nparts > 1 ? out[1] : nullptr, nparts > 2 ? out[2] : nullptr,
                         nparts > 3 ? out[3] : nullptr};
  if (transpose) {
    k_split_t<<<dim3(cdiv(cols, 32), cdiv(rows, 32)), dim3(32, 8), 0, s>>>(
        in, ld_in, o[0], o[1], o[2], o[3], nparts, ld_out, rows, cols);
  } else {
    k_split<<<grid_for(rows * cols), 256, 0, s>>>(in, ld_in, o[0], o[1], o[2], o[3], nparts,
                                                 ld_out, rows, cols);
  }
  FX_LAUNCH_CHECK();
}

template <typename T>
void launch_output(const T* ere, const T* eim, int64_t n, int64_t np, OutputMap om, void* U,
                   int dtype, cudaStream_t s) {
  const unsigned g = grid_for(n * n);
  switch (dtype) {
    case FX_F32: k_output<T, float><<<g, 256, 0, s>>>(ere, eim, n, np, om, (float*)U); break;
    case FX_F64: k_output<T, double><<<g, 256, 0, s>>>(ere, eim, n, np, om, (double*)U); break;
    case FX_C64: k_output<T, float2><<<g, 256, 0, s>>>(ere, eim, n, np, om, (float2*)U); break;
    case FX_C128: k_output<T, double2><<<g, 256, 0, s>>>(ere, eim, n, np, om, (double2*)U); break;
    default: throw Error{FX_ERR_TYPE, "unknown dtype"};
  }
  FX_LAUNCH_CHECK();
}

template <typename T>
void launch_apply(const T* ere, const T* eim, int64_t n, int64_t np, OutputMap om,
                  const void* psi0, void* psi, int dtype, double* scratch2, cudaStream_t s) {
  if (dtype == FX_C64 || dtype == FX_F32) {
    k_psi_sum<float2><<<1, 256, 0, s>>>((const float2*)psi0, n, scratch2);
    FX_LAUNCH_CHECK();
    k_apply<T, float2><<<cdiv(n, 8), 256, 0, s>>>(ere, eim, n, np, om, (const float2*)psi0,
                                                 (float2*)psi, scratch2);
  } else {
    k_psi_sum<double2><<<1, 256, 0, s>>>((const double2*)psi0, n, scratch2);
    FX_LAUNCH_CHECK();
    k_apply<T, double2><<<cdiv(n, 8), 256, 0, s>>>(ere, eim, n, np, om, (const double2*)psi0,
                                                  (double2*)psi, scratch2);
  }
  FX_LAUNCH_CHECK();
}

#define FX_INST(T)                                                                              \
  template void launch_load_shifted<T>(const void*, int, int64_t, int64_t, double, double,      \
                                       double, double, T*, T*, cudaStream_t);                   \
  template void launch_col_abs_sums<T>(const T*, const T*, int64_t, int64_t, double*,           \
                                       cudaStream_t);                                           \
  template void launch_matvec2<T>(const T*, const T*, int64_t, const double*, double*,          \
                                  cudaStream_t);                                                \
  template void launch_matvec2_h<T>(const T*, const T*, int64_t, const double*, double*,        \
                                    cudaStream_t);                                              \
  template void launch_vec_absmat<T>(const T*, const T*, int64_t, const double*, double*,       \
                                     cudaStream_t);                                             \
  template void launch_combo<T>(T*, const T*, double, const T*, double, const T*, double,       \
                                const T*, double, double, int64_t, cudaStream_t);               \
  template void launch_zero<T>(T*, int64_t, cudaStream_t);                                      \
  template void launch_transpose<T>(const T*, int64_t, T*, int64_t, int64_t, int64_t,           \
                                    cudaStream_t);                                              \
  template void launch_output<T>(const T*, const T*, int64_t, int64_t, OutputMap, void*, int,   \
                                 cudaStream_t);                                                 \
  template void launch_apply<T>(const T*, const T*, int64_t, int64_t, OutputMap, const void*,   \
                                void*, int, double*, cudaStream_t);

FX_INST(float)
FX_INST(double)

}  // namespace fx

namespace fx {
namespace {
// (A + A^T)/2 on 32x32 tile pairs (bi <= bj), in place.
template <typename T>
__global__ void k_symmetrize(T* a, int64_t n, int64_t ld) {
  __shared__ T t1[32][33], t2[32][33];
  const int bi = blockIdx.y, bj = blockIdx.x;
  if (bi > bj) return;
  const int tx = threadIdx.x;
  for (int r = threadIdx.y; r < 32; r += 8) {
    int64_t i = (int64_t)bi * 32 + r, j = (int64_t)bj * 32 + tx;
    t1[r][tx] = (i < n && j < n) ? a[i * ld + j] : (T)0;
    i = (int64_t)bj * 32 + r;
    j = (int64_t)bi * 32 + tx;
    t2[r][tx] = (i < n && j < n) ? a[i * ld + j] : (T)0;
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += 8) {
    // new a[bi*32+r][bj*32+tx] = (t1[r][tx] + t2[tx][r]) / 2 ; and its mirror
    const T v = (t1[r][tx] + t2[tx][r]) * (T)0.5;
    int64_t i = (int64_t)bi * 32 + r, j = (int64_t)bj * 32 + tx;
    if (i < n && j < n) a[i * ld + j] = v;
    const T w = (t2[r][tx] + t1[tx][r]) * (T)0.5;
    i = (int64_t)bj * 32 + r;
    j = (int64_t)bi * 32 + tx;
    if (i < n && j < n) a[i * ld + j] = w;
  }
}
}  // namespace

template <typename T>
void launch_symmetrize(T* a, int64_t n, int64_t ld, cudaStream_t s) {
  const unsigned nt = cdiv(n, 32);
  k_symmetrize<T><<<dim3(nt, nt), dim3(32, 8), 0, s>>>(a, n, ld);
  FX_LAUNCH_CHECK();
}
template void launch_symmetrize<float>(float*, int64_t, int64_t, cudaStream_t);
template void launch_symmetrize<double>(double*, int64_t, int64_t, cudaStream_t);
}  // namespace fx

namespace fx {
namespace {
// Signed row sums (warp per row) and column sums (row-chunked, ordered) of the n x n block.
template <typename T>
__global__ void k_row_sums(const T* a, int64_t n, int64_t ld, double* rs) {
  const int lane = threadIdx.x & 31;
  const int64_t row = (int64_t)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  if (row >= n) return;
  double s = 0.0;
  for (int64_t j = lane; j < n; j += 32) s += (double)a[row * ld + j];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) rs[row] = s;
}
template <typename T>
__global__ void k_col_sum_partials(const T* a, int64_t n, int64_t ld, int64_t rows_per_chunk, double* part) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const int64_t r0 = (int64_t)blockIdx.y * rows_per_chunk;
  const int64_t r1 = min(n, r0 + rows_per_chunk);
  double s = 0.0;
  for (int64_t i = r0; i < r1; ++i) s += (double)a[i * ld + j];
  part[(int64_t)blockIdx.y * n + j] = s;
}
__global__ void k_vec_total(const double* v, int64_t n, double* out) {
  __shared__ double sh[256];
  double s = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) s += v[i];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = sh[0];
}
template <typename T>
__global__ void k_apply_proj(T* a, int64_t n, int64_t ld, const double* rs, const double* cs, const double* tot) {
  const int64_t total = n * n;
  const double inv = 1.0 / (double)n, sig = tot[0] * inv * inv;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = idx / n, j = idx - (idx / n) * n;
    a[i * ld + j] = (T)((double)a[i * ld + j] - rs[i] * inv - cs[j] * inv + sig);
  }
}
}  // namespace

template <typename T>
void launch_project_ones(T* a, int64_t n, int64_t ld, double* scratch, cudaStream_t s) {
  // scratch: rs (n), cs (n), tot (1), partials (32 n)
  double* rs = scratch;
  double* cs = rs + n;
  double* tot = cs + n;
  double* part = tot + 8;
  k_row_sums<T><<<cdiv(n, 8), 256, 0, s>>>(a, n, ld, rs);
  FX_LAUNCH_CHECK();
  const int chunks = 32;
  const int64_t rpc = (n + chunks - 1) / chunks;
  k_col_sum_partials<T><<<dim3(cdiv(n, 128), chunks), 128, 0, s>>>(a, n, ld, rpc, part);
  FX_LAUNCH_CHECK();
  k_col_finish1<<<cdiv(n, 256), 256, 0, s>>>(part, chunks, n, cs);
  FX_LAUNCH_CHECK();
  k_vec_total<<<1, 256, 0, s>>>(rs, n, tot);
  FX_LAUNCH_CHECK();
  unsigned g = (unsigned)std::min<int64_t>((n * n + 255) / 256, 148 * 16);
  k_apply_proj<T><<<g, 256, 0, s>>>(a, n, ld, rs, cs, tot);
  FX_LAUNCH_CHECK();
}
template void launch_project_ones<float>(float*, int64_t, int64_t, double*, cudaStream_t);
template void launch_project_ones<double>(double*, int64_t, int64_t, double*, cudaStream_t);
}  // namespace fx
