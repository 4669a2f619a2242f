// Device-side set-up and read-out around the propagator: the O(N^2) host steps of the
// reference's walk, moved next to the data.
//
//   fx_build_generator   X = -i t H of an undirected graph given as an edge list, with
//                        H = -gamma A or -gamma (D - A) (FastCTQW/Operator.py:49-56), written
//                        straight into the device buffer that the walk reads.  The values are
//                        rounded as the reference's numpy expressions round them in the
//                        walk's dtype, so the matrix equals the host-built one bit for bit.
//   fx_check_hermitian   np.allclose(H, H^H) (FastCTQW/Operator.py:92-103), or the skew-Hermitian
//                        test of a walk's X = -iHt, in one pass over the matrix:
//                        32 x 32 tiles (i, j) and (j, i) read together into shared memory.
//   fx_apply_propagator  psi_out = U psi_in, the GEMV of Ctqw.runWalk (FastCTQW/Ctqw.py:90-94),
//                        for stepping a state through a time grid with one U.
//   fx_probabilities     |psi_i|^2 of all nodes or of listed nodes (FastCTQW/State.py:50-51),
//                        in FP64.
//
// All four are HBM-bound passes; none allocates device memory.  The edge-range and Hermitian
// results come back through one flag word in device memory, so calls of these two entry
// points that overlap on the GPU race on it.
#include <cmath>
#include <mutex>
#include <string>

#include "fx_common.cuh"

namespace fx {
namespace {

__device__ int g_graph_flag;   // 1: an edge endpoint out of range; 2: not Hermitian

std::mutex g_graph_mu;
std::string g_graph_err;

int graph_fail(int code, const std::string& msg) {
  std::lock_guard<std::mutex> lk(g_graph_mu);
  g_graph_err = msg;
  return code;
}

template <typename C>
struct Elem;
template <>
struct Elem<float> {
  static __device__ __forceinline__ double2 load(const float* p, int64_t i) { return make_double2(p[i], 0.0); }
};
template <>
struct Elem<double> {
  static __device__ __forceinline__ double2 load(const double* p, int64_t i) { return make_double2(p[i], 0.0); }
};
template <>
struct Elem<float2> {
  static __device__ __forceinline__ double2 load(const float2* p, int64_t i) {
    const float2 v = p[i];
    return make_double2(v.x, v.y);
  }
  static __device__ __forceinline__ void store(float2* p, int64_t i, double re, double im) {
    p[i] = make_float2((float)re, (float)im);
  }
};
template <>
struct Elem<double2> {
  static __device__ __forceinline__ double2 load(const double2* p, int64_t i) { return p[i]; }
  static __device__ __forceinline__ void store(double2* p, int64_t i, double re, double im) {
    p[i] = make_double2(re, im);
  }
};

__global__ void k_clear_flag() { g_graph_flag = 0; }

// One thread per edge: X[u][v] = X[v][u] = off (writes of one value, so repeated edges are
// harmless); a self-loop puts `self` on the diagonal (adjacency) or nothing (Laplacian).
template <typename C>
__global__ void k_scatter_edges(const int64_t* __restrict__ edges, int64_t m, int64_t n, C off, C self,
                                int lap, C* __restrict__ X) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t u = edges[2 * e], v = edges[2 * e + 1];
    if (u < 0 || u >= n || v < 0 || v >= n) {
      atomicOr(&g_graph_flag, 1);
      continue;
    }
    if (u == v) {
      if (!lap) X[u * n + u] = self;
      continue;
    }
    X[u * n + v] = off;
    X[v * n + u] = off;
  }
}

// Laplacian diagonal, a warp per row: d = the row's off-diagonal nonzeros (its neighbours),
// X[i][i] = i * ((gamma d) t), each product rounded in the element precision R as numpy
// rounds -1j * (-gamma (D - A)) * t for that dtype.
template <typename C, typename R>
__global__ void k_laplacian_diag(int64_t n, R gamma, R t, C* __restrict__ X) {
  const int lane = threadIdx.x & 31;
  const int64_t row = (int64_t)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  if (row >= n) return;
  const C* r = X + row * n;
  long long cnt = 0;
  for (int64_t j = lane; j < n; j += 32) {
    const C v = r[j];
    if (j != row && (v.x != 0 || v.y != 0)) ++cnt;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
  if (lane == 0) {
    const R hd = gamma * (R)cnt;
    C d;
    d.x = (R)0;
    d.y = hd * t;
    X[row * n + row] = d;
  }
}

// np.allclose(H, sH^H), s = +1 (Hermitian) or -1 (skew-Hermitian, as X = -iHt):
// |H_ij - s conj(H_ji)| <= atol + rtol |H_ji| for every i, j (NaN fails).  Block (tj, ti) with
// ti <= tj reads tiles (ti, tj) and (tj, ti) once each.
template <typename T>
__global__ void __launch_bounds__(256) k_check_hermitian(const T* __restrict__ H, int64_t n, double rtol, double atol,
                                                         double sgn) {
  const int ti = blockIdx.y, tj = blockIdx.x;
  if (ti > tj) return;
  __shared__ double2 a[32][33], b[32][33];
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;   // 32 x 8
  for (int r = ty; r < 32; r += 8) {
    const int64_t i = (int64_t)ti * 32 + r, j = (int64_t)tj * 32 + tx;
    a[r][tx] = (i < n && j < n) ? Elem<T>::load(H, i * n + j) : make_double2(0.0, 0.0);
    const int64_t i2 = (int64_t)tj * 32 + r, j2 = (int64_t)ti * 32 + tx;
    b[r][tx] = (i2 < n && j2 < n) ? Elem<T>::load(H, i2 * n + j2) : make_double2(0.0, 0.0);
  }
  __syncthreads();
  bool bad = false;
  for (int r = ty; r < 32; r += 8) {
    const double2 x = a[r][tx];   // H[ti*32 + r][tj*32 + tx]
    const double2 y = b[tx][r];   // H[tj*32 + tx][ti*32 + r]
    const double dr = x.x - sgn * y.x, di = x.y + sgn * y.y;
    if (!(hypot(dr, di) <= atol + rtol * hypot(y.x, y.y))) bad = true;
  }
  if (__any_sync(0xffffffffu, bad) && tx == 0) atomicOr(&g_graph_flag, 2);
}

// y = U x, a warp per row, FP64 accumulation.
template <typename C>
__global__ void k_gemv(const C* __restrict__ U, int64_t n, const C* __restrict__ x, C* __restrict__ y) {
  const int lane = threadIdx.x & 31;
  const int64_t row = (int64_t)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  if (row >= n) return;
  double yr = 0.0, yi = 0.0;
  for (int64_t j = lane; j < n; j += 32) {
    const double2 a = Elem<C>::load(U, row * n + j);
    const double2 v = Elem<C>::load(x, j);
    yr += a.x * v.x - a.y * v.y;
    yi += a.x * v.y + a.y * v.x;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    yr += __shfl_xor_sync(0xffffffffu, yr, o);
    yi += __shfl_xor_sync(0xffffffffu, yi, o);
  }
  if (lane == 0) Elem<C>::store(y, row, yr, yi);
}

template <typename C>
__global__ void k_probabilities(const C* __restrict__ psi, int64_t n, const int64_t* __restrict__ nodes,
                                int64_t count, double* __restrict__ prob) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < count; k += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = nodes ? nodes[k] : k;
    if (i < 0 || i >= n) {
      prob[k] = __longlong_as_double(0x7ff8000000000000ll);   // quiet NaN: no such node
      continue;
    }
    const double2 v = Elem<C>::load(psi, i);
    prob[k] = __dadd_rn(__dmul_rn(v.x, v.x), __dmul_rn(v.y, v.y));   // no contraction: as numpy
  }
}

unsigned grid_for(int64_t items, int per_block) {
  const int64_t b = (items + per_block - 1) / per_block;
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(b, 148 * 32));
}

int read_flag(cudaStream_t s, int* flag) {
  cudaError_t e = cudaMemcpyFromSymbolAsync(flag, g_graph_flag, sizeof(int), 0, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return graph_fail(FX_ERR_CUDA, std::string("flag read-back: ") + cudaGetErrorString(e));
  return FX_OK;
}

int launch_status(const char* what) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return graph_fail(FX_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  return FX_OK;
}

}  // namespace
}  // namespace fx

using namespace fx;

extern "C" {

int fx_build_generator(int64_t n, const int64_t* edges, int64_t m, double gamma, int laplacian, double t,
                       int dtype, void* X, void* stream) {
  if (dtype != FX_C64 && dtype != FX_C128)
    return graph_fail(FX_ERR_TYPE, "fx_build_generator: X is complex64 or complex128");
  if (n <= 0 || m < 0 || !X || (m > 0 && !edges))
    return graph_fail(FX_ERR_VALUE, "fx_build_generator: need n > 0, m >= 0, X and the edge array");
  if (!std::isfinite(gamma) || !std::isfinite(t))
    return graph_fail(FX_ERR_NONFINITE, "fx_build_generator: gamma and t must be finite");
  cudaStream_t s = (cudaStream_t)stream;
  const size_t elem = dtype == FX_C64 ? 8 : 16;
  cudaError_t e = cudaMemsetAsync(X, 0, (size_t)n * (size_t)n * elem, s);
  if (e != cudaSuccess) return graph_fail(FX_ERR_CUDA, std::string("fx_build_generator: ") + cudaGetErrorString(e));
  k_clear_flag<<<1, 1, 0, s>>>();
  const unsigned ge = grid_for(m, 256), gr = grid_for(n * 32, 256);
  if (dtype == FX_C64) {
    // X = -1j * (-gamma A) * t: imaginary part fl(fl(gamma) fl(t)) on the edges (adjacency),
    // its negative (Laplacian off-diagonal)
    const float g = (float)gamma, tt = (float)t, v = g * tt;
    const float2 off = make_float2(0.0f, laplacian ? -v : v), self = make_float2(0.0f, v);
    if (m > 0) k_scatter_edges<float2><<<ge, 256, 0, s>>>(edges, m, n, off, self, laplacian, (float2*)X);
    if (laplacian) k_laplacian_diag<float2, float><<<gr, 256, 0, s>>>(n, g, tt, (float2*)X);
  } else {
    const double v = gamma * t;
    const double2 off = make_double2(0.0, laplacian ? -v : v), self = make_double2(0.0, v);
    if (m > 0) k_scatter_edges<double2><<<ge, 256, 0, s>>>(edges, m, n, off, self, laplacian, (double2*)X);
    if (laplacian) k_laplacian_diag<double2, double><<<gr, 256, 0, s>>>(n, gamma, t, (double2*)X);
  }
  int rc = launch_status("fx_build_generator");
  if (rc) return rc;
  int flag = 0;
  if ((rc = read_flag(s, &flag))) return rc;
  if (flag & 1) return graph_fail(FX_ERR_VALUE, "fx_build_generator: an edge endpoint is outside 0..n-1");
  return FX_OK;
}

int fx_check_hermitian(int64_t n, int dtype, const void* H, double rtol, double atol, int skew,
                       int32_t* hermitian, void* stream) {
  if (n <= 0 || !H || !hermitian) return graph_fail(FX_ERR_VALUE, "fx_check_hermitian: need n > 0, H and the result");
  if (n > (int64_t)65535 * 32) return graph_fail(FX_ERR_VALUE, "fx_check_hermitian: n too large");
  cudaStream_t s = (cudaStream_t)stream;
  k_clear_flag<<<1, 1, 0, s>>>();
  const unsigned nt = (unsigned)((n + 31) / 32);
  const dim3 grid(nt, nt);
  const double sgn = skew ? -1.0 : 1.0;
  switch (dtype) {
    case FX_F32: k_check_hermitian<float><<<grid, 256, 0, s>>>((const float*)H, n, rtol, atol, sgn); break;
    case FX_F64: k_check_hermitian<double><<<grid, 256, 0, s>>>((const double*)H, n, rtol, atol, sgn); break;
    case FX_C64: k_check_hermitian<float2><<<grid, 256, 0, s>>>((const float2*)H, n, rtol, atol, sgn); break;
    case FX_C128: k_check_hermitian<double2><<<grid, 256, 0, s>>>((const double2*)H, n, rtol, atol, sgn); break;
    default: return graph_fail(FX_ERR_TYPE, "fx_check_hermitian: unknown dtype");
  }
  int rc = launch_status("fx_check_hermitian");
  if (rc) return rc;
  int flag = 0;
  if ((rc = read_flag(s, &flag))) return rc;
  *hermitian = (flag & 2) ? 0 : 1;
  return FX_OK;
}

int fx_apply_propagator(int64_t n, int dtype, const void* U, const void* psi_in, void* psi_out, void* stream) {
  if (n <= 0 || !U || !psi_in || !psi_out) return graph_fail(FX_ERR_VALUE, "fx_apply_propagator: need n > 0 and buffers");
  if (psi_in == psi_out) return graph_fail(FX_ERR_VALUE, "fx_apply_propagator: psi_out must not be psi_in");
  cudaStream_t s = (cudaStream_t)stream;
  const unsigned g = (unsigned)((n + 7) / 8);
  if (dtype == FX_C64)
    k_gemv<float2><<<g, 256, 0, s>>>((const float2*)U, n, (const float2*)psi_in, (float2*)psi_out);
  else if (dtype == FX_C128)
    k_gemv<double2><<<g, 256, 0, s>>>((const double2*)U, n, (const double2*)psi_in, (double2*)psi_out);
  else
    return graph_fail(FX_ERR_TYPE, "fx_apply_propagator: U and psi are complex64 or complex128");
  return launch_status("fx_apply_propagator");
}

int fx_probabilities(int64_t n, int dtype, const void* psi, const int64_t* nodes, int64_t count, double* prob,
                     void* stream) {
  if (n <= 0 || !psi || !prob) return graph_fail(FX_ERR_VALUE, "fx_probabilities: need n > 0, psi and prob");
  if (!nodes) count = n;
  if (count <= 0) return FX_OK;
  cudaStream_t s = (cudaStream_t)stream;
  const unsigned g = grid_for(count, 256);
  if (dtype == FX_C64)
    k_probabilities<float2><<<g, 256, 0, s>>>((const float2*)psi, n, nodes, count, prob);
  else if (dtype == FX_C128)
    k_probabilities<double2><<<g, 256, 0, s>>>((const double2*)psi, n, nodes, count, prob);
  else
    return graph_fail(FX_ERR_TYPE, "fx_probabilities: psi is complex64 or complex128");
  return launch_status("fx_probabilities");
}

const char* fx_graph_error(void) {
  std::lock_guard<std::mutex> lk(g_graph_mu);
  return g_graph_err.c_str();
}

}  // extern "C"
