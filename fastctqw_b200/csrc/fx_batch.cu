// Batched walks: many independent expm(X_w) psi0_w of uneven sizes in grouped launches.
//
// The per-walk engine (fx_engine.cu) issues a few hundred launches and several host
// round trips per walk; for hundreds of small and medium walks that is launch- and
// latency-bound.  Here every phase of the pipeline is one grouped launch over all walks that
// take part in it:
//   * grouped int8 Ozaki-slice products (one tile list over all walks' problems, see
//     k_gemm_i8<.., true> in fx_gemm_i8.cu), with the slices of all walks stacked in common
//     slice planes,
//   * grouped elementwise / reduction kernels (this file): grid.y runs over a list of walks,
//   * a device-side block 1-norm estimator (one CTA per walk) so that the selection of (m, s)
//     needs a single host round trip for the whole batch,
//   * the Pade solve for X = i*(real symmetric) as G = Q^H Q = L L^T (blocked Cholesky, one
//     CTA per walk for the diagonal blocks), the explicit inverse X = L^-1 (blocked, backward),
//     and two large triangle-aware products Z = P2 X^T, R^T = Z X (R = G^-1 P2 is symmetric).
// Everything after the selection is recorded once and replayed as one CUDA graph.
//
// Scope: walk generators X = i*(real symmetric) (the walk family X = -iHt with a real
// symmetric H), complex64 or complex128 storage, FP64 masters and 5 int8 slices (the plain
// form of the per-walk engine).  The selection follows the per-walk engine (Al-Mohy & Higham
// 2009, Algorithm 6.1; normal input, so l(A, m) = 0).
#include <algorithm>
#include <array>
#include <cmath>
#include <complex>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "fx_kernels.cuh"

namespace fx {
namespace {

constexpr int kS = 5;          // int8 slices (FP64 masters)
constexpr int kNb = 128;       // Cholesky / inverse block
constexpr int kEstScratch = 8; // doubles per row of a walk in the estimator scratch
// The mixed form's reduced slice counts (and its Newton-Schulz solve) serve walks padded to at
// least this size.  Below it the products are short and their epilogues weigh as much as their
// MMAs, so fewer slices save little, and the blocked Cholesky has few steps (np / 128), which
// run grouped over the batch: smaller walks keep the plain schedule in either form.
constexpr int kMixedMinNp = 4096;
// The mixed form's Pade and solve products run at its reduced slice count only when the
// selection takes at most this many squarings (their errors are amplified 2^s); above it, 5.
constexpr int kMixedMaxPadeS = 10;
// Walks padded to at least this size solve the Pade step by Newton-Schulz (either form).
constexpr int kNewtonMinNp = 4096;
// Walks padded to at least this size, or whose selection takes at least kSquare3MinS squarings,
// square in the three-product form (Re^2, Im^2, (Re+Im)^2, each with the diagonal split) in
// either form.  Large walks: three products instead of four, and at these sizes the products'
// MMAs outweigh their epilogues.  Long chains: the split keeps the iterate's dominant diagonal
// out of the slices, and the 2^(s-k) amplification of squaring k's error needs those bits (on
// walks with 15 to 17 squarings the exact complex square left infidelities near 1e-10, the
// split form 2e-11 and below; on a 3-regular Laplacian walk with 9 squarings 2.6e-9 against
// 2.2e-12, and 3e-11 with 8).
constexpr int kSquare3MinNp = 4096;
constexpr int kSquare3MinS = 8;

struct BWalk {
  int n, np;
  int64_t off;    // element offset of the walk's np x np block in every master arena
  int64_t row0;   // first row of the walk in stacked per-row arrays (sum of np of earlier walks)
};

// ------------------------------------------------------------------ grouped elementwise
struct Planes5 {
  const double* m[5];
};

// Elementwise work over walks of uneven sizes is cut into row chunks of about kChunkElems
// elements (one CTA each, any walk), so that large and small walks load the GPU evenly.
constexpr int kChunkElems = 16384;
struct RChunk {
  int w, r0, r1, pad;   // walk, rows [r0, r1)
};

// D = sum_k c_k M_k + g I on the np x np block of every chunk's walk; coef[(NP + 1) w ..] =
// (c_0..c_{NP-1}, g).  Two elements per thread (np is even); 32-bit indices within the chunk.
template <int NP>
struct PlanesN {
  const double* m[NP];
};
template <int NP>
__global__ void kb_combo(double* D, PlanesN<NP> M, const RChunk* ch, const BWalk* wk, const double* coef) {
  const RChunk q = ch[blockIdx.x];
  const BWalk b = wk[q.w];
  const double* c = coef + (NP + 1) * q.w;
  const uint32_t half = (uint32_t)b.np / 2, total = (uint32_t)(q.r1 - q.r0) * half;
  const double2* src[NP];
  double cc[NP];
#pragma unroll
  for (int k = 0; k < NP; ++k) {   // a zero coefficient skips the term: its plane may be unset
    const bool on = M.m[k] && c[k] != 0.0;
    cc[k] = on ? c[k] : 0.0;
    src[k] = on ? reinterpret_cast<const double2*>(M.m[k] + b.off) : nullptr;
  }
  const double g = c[NP];
  double2* dst = reinterpret_cast<double2*>(D + b.off);
  for (uint32_t t = threadIdx.x; t < total; t += blockDim.x) {
    const uint32_t rr = t / half, c2 = t - rr * half;
    const int64_t r = q.r0 + (int64_t)rr;
    const int64_t e2 = r * half + c2;   // double2 index of (r, 2 c2)
    double vx = 0.0, vy = 0.0;
#pragma unroll
    for (int k = 0; k < NP; ++k)
      if (src[k]) {
        const double2 m = src[k][e2];
        vx += cc[k] * m.x;
        vy += cc[k] * m.y;
      }
    if (2 * (int64_t)c2 == r) vx += g;
    else if (2 * (int64_t)c2 + 1 == r) vy += g;
    dst[e2] = make_double2(vx, vy);
  }
}
using Planes4 = PlanesN<4>;


// Statistics of the interleaved input of each walk, warp per row i < n:
// rowstat[kRS * (row0 + i)] = (Re row sum, Im row sum, Re X_ii, Im X_ii, sum |Re| + |Im|,
// sum |X_ij|^2, number of nonzero off-diagonal entries); flags[w] |= 1 (Re != 0),
// 2 (not symmetric), 4 (non-finite).
constexpr int kRS = 8;
constexpr int kWO = 16;   // per-walk record of kb_walk_reduce
template <typename C>
__global__ void kb_stats(const void* const* X, const int* list, const BWalk* wk, double* rowstat, int* flags) {
  const int w = list[blockIdx.y];
  const BWalk b = wk[w];
  const C* x = (const C*)X[w];
  const int lane = threadIdx.x & 31;
  const int wpb = blockDim.x / 32;
  int f = 0;
  for (int64_t i = (int64_t)blockIdx.x * wpb + threadIdx.x / 32; i < b.n; i += (int64_t)gridDim.x * wpb) {
    double sr = 0, si = 0, sa = 0, sq = 0, nz = 0;
    for (int64_t j = lane; j < b.n; j += 32) {
      const C v = x[i * b.n + j];
      const double vr = (double)v.x, vi = (double)v.y;
      sr += vr;
      si += vi;
      sa += fabs(vr) + fabs(vi);
      sq += vr * vr + vi * vi;
      if (j != i && (vr != 0.0 || vi != 0.0)) nz += 1.0;
      if (vr != 0.0) f |= 1;
      if (!isfinite(vr) || !isfinite(vi)) f |= 4;
      if (j > i) {
        const C u = x[j * b.n + i];
        if (u.x != v.x || u.y != v.y) f |= 2;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      sr += __shfl_xor_sync(0xffffffffu, sr, o);
      si += __shfl_xor_sync(0xffffffffu, si, o);
      sa += __shfl_xor_sync(0xffffffffu, sa, o);
      sq += __shfl_xor_sync(0xffffffffu, sq, o);
      nz += __shfl_xor_sync(0xffffffffu, nz, o);
    }
    if (lane == 0) {
      const C d = x[i * b.n + i];
      double* r = rowstat + kRS * (b.row0 + i);
      r[0] = sr;
      r[1] = si;
      r[2] = (double)d.x;
      r[3] = (double)d.y;
      r[4] = sa;
      r[5] = sq;
      r[6] = nz;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) f |= __shfl_xor_sync(0xffffffffu, f, o);
  if (lane == 0 && f) atomicOr(flags + w, f);
}

// One CTA per walk: the shifts.  mu = trace / n (ordered sum of the diagonal); the rank-one
// shift applies when every row sum equals row 0's within the rounding of a sum,
// 4 n 2^-53 max_i sum_j |X_ij| (the input is exactly symmetric, so the column sums are the
// same numbers); then nu = c0 - mu.  out[kWO w ..] = (mu re, mu im, nu re, nu im, rank1, mu_im,
// nu_im / n, 0, ||X||_F^2, max off-diagonal nonzeros of a row, max absolute row sum); mu_im and
// nu_im / n are the load parameters of kb_load_imag.
__global__ void kb_walk_reduce(const int* list, const BWalk* wk, const double* rowstat, double* out) {
  const int w = list[blockIdx.x];
  const BWalk b = wk[w];
  const double* r = rowstat + kRS * b.row0;
  __shared__ double s_max[256];
  __shared__ double s_dev[256];
  __shared__ double s_nz[256];
  const double c0r = r[0], c0i = r[1];
  double mx = 0.0, dev = 0.0, nz = 0.0;
  for (int i = threadIdx.x; i < b.n; i += blockDim.x) {
    mx = fmax(mx, r[kRS * i + 4]);
    dev = fmax(dev, fmax(fabs(r[kRS * i] - c0r), fabs(r[kRS * i + 1] - c0i)));
    nz = fmax(nz, r[kRS * i + 6]);
  }
  // the trace and ||X||_F^2: per-thread sums over rows i = t mod blockDim in order, then a fixed
  // tree (the same association every run)
  __shared__ double s_tr[256];
  __shared__ double s_ti[256];
  __shared__ double s_fr[256];
  double tr = 0, ti = 0, fro2 = 0;
  for (int i = threadIdx.x; i < b.n; i += blockDim.x) {
    tr += r[kRS * i + 2];
    ti += r[kRS * i + 3];
    fro2 += r[kRS * i + 5];
  }
  s_max[threadIdx.x] = mx;
  s_dev[threadIdx.x] = dev;
  s_nz[threadIdx.x] = nz;
  s_tr[threadIdx.x] = tr;
  s_ti[threadIdx.x] = ti;
  s_fr[threadIdx.x] = fro2;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      s_max[threadIdx.x] = fmax(s_max[threadIdx.x], s_max[threadIdx.x + o]);
      s_dev[threadIdx.x] = fmax(s_dev[threadIdx.x], s_dev[threadIdx.x + o]);
      s_nz[threadIdx.x] = fmax(s_nz[threadIdx.x], s_nz[threadIdx.x + o]);
      s_tr[threadIdx.x] += s_tr[threadIdx.x + o];
      s_ti[threadIdx.x] += s_ti[threadIdx.x + o];
      s_fr[threadIdx.x] += s_fr[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    tr = s_tr[0];
    ti = s_ti[0];
    fro2 = s_fr[0];
    const double n = b.n;
    const double mur = tr / n, mui = ti / n;
    const bool rank1 = b.n > 1 && s_dev[0] <= 4.0 * n * 0x1p-53 * s_max[0];
    const double nur = rank1 ? c0r - mur : 0.0, nui = rank1 ? c0i - mui : 0.0;
    double* o = out + kWO * w;
    o[0] = mur;
    o[1] = mui;
    o[2] = nur;
    o[3] = nui;
    o[4] = rank1 ? 1.0 : 0.0;
    o[5] = mui;
    o[6] = nui / n;
    o[7] = 0.0;
    o[8] = fro2;
    o[9] = s_nz[0];
    o[10] = s_max[0];
  }
}

// Y = Im(X) - mu_im I - nu_im/n J on the n x n block, 0 in the padding (imaginary plane of the
// shifted generator; its real plane is zero for X = i*(real symmetric)).  sh[kWO w + 5, 6] =
// (mu_im, nu_im/n) as written by kb_walk_reduce.
template <typename C>
__global__ void kb_load_imag(const void* const* X, const int* list, const BWalk* wk, const double* sh, double* Y,
                             float* Y32) {
  const int w = list[blockIdx.y];
  const BWalk b = wk[w];
  const C* x = (const C*)X[w];
  const double mu = sh[kWO * w + 5], nun = sh[kWO * w + 6];
  const int64_t n2 = (int64_t)b.np * b.np;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < n2;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = idx / b.np, j = idx - i * b.np;
    double v = 0.0;
    if (i < b.n && j < b.n) v = (double)x[i * b.n + j].y - (i == j ? mu : 0.0) - nun;
    Y[b.off + idx] = v;
    if (Y32) Y32[b.off + idx] = (float)v;
  }
}

// Absolute row sums of a symmetric plane (= column sums), warp per row -> rs[row0 + i].
__global__ void kb_abs_rowsums(const double* P, const int* list, const BWalk* wk, double* rs) {
  const int w = list[blockIdx.y];
  const BWalk b = wk[w];
  const int lane = threadIdx.x & 31, wpb = blockDim.x / 32;
  for (int64_t i = (int64_t)blockIdx.x * wpb + threadIdx.x / 32; i < b.np; i += (int64_t)gridDim.x * wpb) {
    const double* row = P + b.off + i * b.np;
    double s = 0;
    for (int64_t j = lane; j < b.np; j += 32) s += fabs(row[j]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) rs[b.row0 + i] = s;
  }
}
// Signed row sums over the n x n block (the projection along the all-ones vector): a warp per
// row, 16-byte loads four at a time (rows start 16-byte aligned: np is a multiple of 128).
__global__ void kb_rowsums(const double* P, const int* list, const BWalk* wk, double* rs) {
  const int w = list[blockIdx.y];
  const BWalk b = wk[w];
  const int lane = threadIdx.x & 31, wpb = blockDim.x / 32;
  const int64_t half = b.n / 2;
  for (int64_t i = (int64_t)blockIdx.x * wpb + threadIdx.x / 32; i < b.n; i += (int64_t)gridDim.x * wpb) {
    const double* row = P + b.off + i * b.np;
    const double2* r2 = reinterpret_cast<const double2*>(row);
    double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
    int64_t j = lane;
    for (; j + 96 < half; j += 128) {
      const double2 a = r2[j], c = r2[j + 32], d = r2[j + 64], e = r2[j + 96];
      s0 += a.x + a.y;
      s1 += c.x + c.y;
      s2 += d.x + d.y;
      s3 += e.x + e.y;
    }
    for (; j < half; j += 32) {
      const double2 a = r2[j];
      s0 += a.x + a.y;
    }
    if ((b.n & 1) && lane == 0) s1 += row[b.n - 1];
    double s = (s0 + s1) + (s2 + s3);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) rs[b.row0 + i] = s;
  }
}
// Unitarity residual of a symmetric complex iterate U = I + E (diagnostics): with Eh = conj(E),
// U^H U - I = 2 Re E + (Er Er + Ei Ei) + i (Er Ei - Ei Er).  D1 = Er Er + Ei Ei and D2 = Er Ei
// are products over the walk's np x np block (zero padding); every chunk adds its share of
// ||2 Er + D1||_F^2 + ||D2 - D2^T||_F^2 to out[w * kDriftMax + slot[w]].
constexpr int kDriftMax = 64;
__global__ void kb_drift(const double* const* Er, const double* D1, const double* D2, const RChunk* ch,
                         const BWalk* wk, const int* slot, double* out) {
  const RChunk q = ch[blockIdx.x];
  const BWalk b = wk[q.w];
  const double* er = Er[q.w];
  const double* d1 = D1 + b.off;
  const double* d2 = D2 + b.off;
  const int64_t np = b.np, total = (int64_t)(q.r1 - q.r0) * np;
  double acc = 0.0;
  for (int64_t t = threadIdx.x; t < total; t += blockDim.x) {
    const int64_t i = q.r0 + t / np, j = t - (t / np) * np;
    const double v1 = 2.0 * er[i * np + j] + d1[i * np + j];
    const double v2 = d2[i * np + j] - d2[j * np + i];
    acc += v1 * v1 + v2 * v2;
  }
  __shared__ double sh[8];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x / 32] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int k = 0; k < (int)(blockDim.x / 32); ++k) t += sh[k];
    atomicAdd(out + (int64_t)q.w * kDriftMax + slot[q.w], t);
  }
}
// One CTA per walk: out[w * stride + slot] = max (mode 0) or sum (mode 1) of v[row0 .. row0 + len).
__global__ void kb_walk_vec_reduce(const double* v, const int* list, const BWalk* wk, int use_np, int mode,
                                   double* out, int stride, int slot) {
  const int w = list[blockIdx.x];
  const BWalk b = wk[w];
  const int len = use_np ? b.np : b.n;
  __shared__ double sh[256];
  double acc = 0.0;
  for (int i = threadIdx.x; i < len; i += blockDim.x) {
    const double x = v[b.row0 + i];
    acc = mode == 0 ? fmax(acc, x) : acc + x;
  }
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] = mode == 0 ? fmax(sh[threadIdx.x], sh[threadIdx.x + o]) : sh[threadIdx.x] + sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[(int64_t)w * stride + slot] = sh[0];
}
// E <- E - (r_i + r_j)/n + T/n^2 on the n x n block (E symmetric, r its row sums, T = sum r),
// rows [r0, r1) of the chunk's walk.
__global__ void kb_apply_proj(double* E, const RChunk* ch, const BWalk* wk, const double* rs, const double* tot) {
  const RChunk q = ch[blockIdx.x];
  const BWalk b = wk[q.w];
  const double inv = 1.0 / b.n, sig = tot[q.w] * inv * inv;
  const double* r = rs + b.row0;
  const uint32_t n = (uint32_t)b.n, total = (uint32_t)(q.r1 - q.r0) * n;
  for (uint32_t t = threadIdx.x; t < total; t += blockDim.x) {
    const uint32_t ii = t / n, j = t - ii * n;
    const int64_t i = q.r0 + (int64_t)ii;
    double& e = E[b.off + i * b.np + j];
    e = e - r[i] * inv - r[j] * inv + sig;
  }
}

// Two linear combinations of the same planes in one pass, D1 = sum_k c_k M_k (+ g1 on the
// diagonal), D2 = sum_k d_k M_k (+ g2), coef[12 w ..] = (c_0..c_4, g1, d_0..d_4, g2) (a plane whose
// coefficients are both zero is not read), by whole rows: a warp per row (chunks of whole rows,
// 8 warps per CTA), with the signed row sums of D1 and D2 over the n x n block, rs1[row0 + i],
// rs2[row0 + i] (each lane sums its columns in order, then a fixed shuffle tree: the same sums
// every run).
__global__ void kb_combo2_rs(double* D1, double* D2, Planes5 M, const RChunk* ch, const BWalk* wk, const double* coef,
                             double* rs1, double* rs2) {
  const RChunk q = ch[blockIdx.x];
  const BWalk b = wk[q.w];
  const double* c = coef + 12 * q.w;
  const double2* src[5];
  double c1[5], c2[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    const bool on = M.m[k] && (c[k] != 0.0 || c[6 + k] != 0.0);
    c1[k] = on ? c[k] : 0.0;
    c2[k] = on ? c[6 + k] : 0.0;
    src[k] = on ? reinterpret_cast<const double2*>(M.m[k] + b.off) : nullptr;
  }
  const double g1 = c[5], g2 = c[11];
  double2* d1 = reinterpret_cast<double2*>(D1 + b.off);
  double2* d2 = reinterpret_cast<double2*>(D2 + b.off);
  const int lane = threadIdx.x & 31, wpb = blockDim.x / 32;
  const int64_t half = b.np / 2;
  for (int64_t i = q.r0 + threadIdx.x / 32; i < q.r1; i += wpb) {
    double s1 = 0.0, s2 = 0.0;
    for (int64_t c2i = lane; c2i < half; c2i += 32) {
      const int64_t e2 = i * half + c2i;   // double2 index of (i, 2 c2i)
      double ax = 0.0, ay = 0.0, bx = 0.0, by = 0.0;
#pragma unroll
      for (int k = 0; k < 5; ++k)
        if (src[k]) {
          const double2 m = src[k][e2];
          ax += c1[k] * m.x;
          ay += c1[k] * m.y;
          bx += c2[k] * m.x;
          by += c2[k] * m.y;
        }
      if (2 * c2i == i) {
        ax += g1;
        bx += g2;
      } else if (2 * c2i + 1 == i) {
        ay += g1;
        by += g2;
      }
      d1[e2] = make_double2(ax, ay);
      d2[e2] = make_double2(bx, by);
      if (2 * c2i < b.n) {
        s1 += ax;
        s2 += bx;
      }
      if (2 * c2i + 1 < b.n) {
        s1 += ay;
        s2 += by;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      s1 += __shfl_xor_sync(0xffffffffu, s1, o);
      s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    }
    if (lane == 0 && i < b.n) {
      rs1[b.row0 + i] = s1;
      rs2[b.row0 + i] = s2;
    }
  }
}
// The projection of both planes, E <- E - (r_i + r_j)/n + T/n^2 on the n x n block, over the
// chunk's rows of the np x np block; with V, also V = E1 + E2 on the whole np x np block.
__global__ void kb_apply_proj2(double* E1, double* E2, double* V, const RChunk* ch, const BWalk* wk, const double* rs1,
                               const double* rs2, const double* tot1, const double* tot2) {
  const RChunk q = ch[blockIdx.x];
  const BWalk b = wk[q.w];
  const double inv = 1.0 / b.n, sig1 = tot1[q.w] * inv * inv, sig2 = tot2[q.w] * inv * inv;
  const double* r1 = rs1 + b.row0;
  const double* r2 = rs2 + b.row0;
  const uint32_t np = (uint32_t)b.np, total = (uint32_t)(q.r1 - q.r0) * np;
  for (uint32_t t = threadIdx.x; t < total; t += blockDim.x) {
    const uint32_t ii = t / np, j = t - ii * np;
    const int64_t i = q.r0 + (int64_t)ii;
    const int64_t e = b.off + i * b.np + j;
    double x = E1[e], y = E2[e];
    if (i < b.n && j < (uint32_t)b.n) {
      x = x - r1[i] * inv - r1[j] * inv + sig1;
      y = y - r2[i] * inv - r2[j] * inv + sig2;
      E1[e] = x;
      E2[e] = y;
    }
    if (V) V[e] = x + y;
  }
}

// Out-of-place transpose of every listed walk's np x np block (32 x 32 tiles).
__global__ void kb_transpose(const double* in, double* out, const int* list, const BWalk* wk, int tiles_max) {
  const int w = list[blockIdx.z];
  const BWalk b = wk[w];
  const int nt = b.np / 32;
  __shared__ double tile[32][33];
  for (int t = blockIdx.x; t < nt * nt; t += gridDim.x) {
    const int64_t r0 = (int64_t)(t / nt) * 32, c0 = (int64_t)(t % nt) * 32;
    for (int r = threadIdx.y; r < 32; r += 8) tile[r][threadIdx.x] = in[b.off + (r0 + r) * b.np + c0 + threadIdx.x];
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += 8) out[b.off + (c0 + r) * b.np + r0 + threadIdx.x] = tile[threadIdx.x][r];
    __syncthreads();
  }
  (void)tiles_max;
}
// A <- (A + A^T)/2 in place for every listed walk (32 x 32 tile pairs, upper tiles drive).
__global__ void kb_symmetrize(double* A, const int* list, const BWalk* wk) {
  const int w = list[blockIdx.z];
  const BWalk b = wk[w];
  const int nt = b.np / 32;
  __shared__ double t1[32][33], t2[32][33];
  for (int t = blockIdx.x; t < nt * nt; t += gridDim.x) {
    const int bi = t / nt, bj = t % nt;
    if (bi > bj) continue;   // uniform per block
    double* a = A + b.off;
    for (int r = threadIdx.y; r < 32; r += 8) {
      t1[r][threadIdx.x] = a[((int64_t)bi * 32 + r) * b.np + bj * 32 + threadIdx.x];
      t2[r][threadIdx.x] = a[((int64_t)bj * 32 + r) * b.np + bi * 32 + threadIdx.x];
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += 8) {
      a[((int64_t)bi * 32 + r) * b.np + bj * 32 + threadIdx.x] = (t1[r][threadIdx.x] + t2[threadIdx.x][r]) * 0.5;
      a[((int64_t)bj * 32 + r) * b.np + bi * 32 + threadIdx.x] = (t2[r][threadIdx.x] + t1[threadIdx.x][r]) * 0.5;
    }
    __syncthreads();
  }
}
// Zero the chunk's rows of its walk's block, then copy the diagonal 128 x 128 blocks of L^-1
// (stored per walk as np x 128, block j at rows [128 j, 128 j + 128)) into X.
__global__ void kb_init_inverse(double* X, const double* Linv, const RChunk* ch, const BWalk* wk, const int64_t* loff) {
  const RChunk q = ch[blockIdx.x];
  const BWalk b = wk[q.w];
  const uint32_t np = (uint32_t)b.np, total = (uint32_t)(q.r1 - q.r0) * np;
  for (uint32_t t = threadIdx.x; t < total; t += blockDim.x) {
    const uint32_t ii = t / np, j = t - ii * np;
    const int64_t i = q.r0 + (int64_t)ii;
    const int64_t bi = i / kNb;
    double v = 0.0;
    if (bi == (int64_t)(j / kNb)) v = Linv[loff[q.w] + i * kNb + (j - bi * kNb)];
    X[b.off + i * b.np + j] = v;
  }
}

// psi = e^mu (E psi0 + psi0 + cj (1^T psi0) 1), warp per row; om[w] = (emu re, im, cj re, im);
// E planes per walk (the squaring chain leaves E in one of two arena pairs).
template <typename C>
__global__ void kb_apply(const double* const* Ere, const double* const* Eim, const void* const* psi0,
                         void* const* psi, const int* list, const BWalk* wk, const double* om, const double* psum) {
  const int w = list[blockIdx.y];
  const BWalk b = wk[w];
  const C* p0 = (const C*)psi0[w];
  C* p1 = (C*)psi[w];
  if (!p0 || !p1) return;
  const double* er = Ere[w] + b.off;
  const double* ei = Eim[w] + b.off;
  const int lane = threadIdx.x & 31, wpb = blockDim.x / 32;
  const double* o = om + 4 * w;
  // pairs of columns per lane: 16-byte loads of E's FP64 planes (rows start 16-byte aligned,
  // np even) and of two psi0 entries when psi0 allows it; column n of a row is padding (zero off
  // the diagonal block) and its psi0 entry is taken as 0
  const bool vec = sizeof(C) == 8 && (reinterpret_cast<uintptr_t>(p0) & 15) == 0;
  for (int64_t i = (int64_t)blockIdx.x * wpb + threadIdx.x / 32; i < b.n; i += (int64_t)gridDim.x * wpb) {
    double yr = 0, yi = 0;
    const double2* ra = reinterpret_cast<const double2*>(er + i * b.np);
    const double2* rc = reinterpret_cast<const double2*>(ei + i * b.np);
#pragma unroll 4
    for (int64_t j = 2 * lane; j < b.n; j += 64) {
      const double2 a = ra[j >> 1], c = rc[j >> 1];
      double x0, y0, x1 = 0.0, y1 = 0.0;
      if (vec && j + 1 < b.n) {
        const float4 q = *reinterpret_cast<const float4*>(p0 + j);
        x0 = q.x;
        y0 = q.y;
        x1 = q.z;
        y1 = q.w;
      } else {
        x0 = (double)p0[j].x;
        y0 = (double)p0[j].y;
        if (j + 1 < b.n) {
          x1 = (double)p0[j + 1].x;
          y1 = (double)p0[j + 1].y;
        }
      }
      yr += a.x * x0 - c.x * y0;
      yi += a.x * y0 + c.x * x0;
      yr += a.y * x1 - c.y * y1;
      yi += a.y * y1 + c.y * x1;
    }
#pragma unroll
    for (int k = 16; k > 0; k >>= 1) {
      yr += __shfl_xor_sync(0xffffffffu, yr, k);
      yi += __shfl_xor_sync(0xffffffffu, yi, k);
    }
    if (lane == 0) {
      yr += (double)p0[i].x;
      yi += (double)p0[i].y;
      const double sr = psum[2 * w], si = psum[2 * w + 1];
      yr += o[2] * sr - o[3] * si;
      yi += o[2] * si + o[3] * sr;
      C out;
      out.x = (decltype(out.x))(o[0] * yr - o[1] * yi);
      out.y = (decltype(out.y))(o[0] * yi + o[1] * yr);
      p1[i] = out;
    }
  }
}
// nrm[2 w .. 2 w + 1] = (||psi0_w||^2, ||psi_w||^2): the unitarity residual of the result on the
// walk's own state (one CTA per walk).
template <typename C>
__global__ void kb_psi_norms(const void* const* psi0, void* const* psi, const int* list, const BWalk* wk,
                             double* nrm) {
  const int w = list[blockIdx.x];
  const C* a = (const C*)psi0[w];
  const C* b = (const C*)psi[w];
  __shared__ double sa[256], sb[256];
  double xa = 0, xb = 0;
  if (a && b)
    for (int j = threadIdx.x; j < wk[w].n; j += blockDim.x) {
      xa += (double)a[j].x * a[j].x + (double)a[j].y * a[j].y;
      xb += (double)b[j].x * b[j].x + (double)b[j].y * b[j].y;
    }
  sa[threadIdx.x] = xa;
  sb[threadIdx.x] = xb;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      sa[threadIdx.x] += sa[threadIdx.x + o];
      sb[threadIdx.x] += sb[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    nrm[2 * w] = sa[0];
    nrm[2 * w + 1] = sb[0];
  }
}

// psum[w] = sum_j psi0_w[j] (ordered, one thread).
template <typename C>
__global__ void kb_psi_sum(const void* const* psi0, const int* list, const BWalk* wk, double* psum) {
  const int w = list[blockIdx.x];
  const C* p = (const C*)psi0[w];
  if (!p) return;
  // per-thread sums over j = t mod blockDim in order, then a fixed tree (blockDim = 256)
  __shared__ double s_r[256];
  __shared__ double s_i[256];
  double sr = 0, si = 0;
  for (int j = threadIdx.x; j < wk[w].n; j += blockDim.x) {
    sr += (double)p[j].x;
    si += (double)p[j].y;
  }
  s_r[threadIdx.x] = sr;
  s_i[threadIdx.x] = si;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      s_r[threadIdx.x] += s_r[threadIdx.x + o];
      s_i[threadIdx.x] += s_i[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    psum[2 * w] = s_r[0];
    psum[2 * w + 1] = s_i[0];
  }
}

// ------------------------------------------------------------------ block 1-norm estimator
// Deterministic Higham-Tisseur estimate (t = 2) of ||M0 M1||_1 for real symmetric M0, M1 (so
// M^H = M) of every listed walk: start columns 1/n and a fixed +-1/n pattern, at most 5
// iterations, sign vectors, and the two largest unvisited entries of |Z| (ties to the lower
// index) as the next unit columns -- the iteration of the oracle's normest1.  The products
// are grid-wide grouped mat-vecs; the decisions run in one CTA per walk; a per-walk `done`
// flag in device memory makes the fixed launch sequence (5 rounds) graph-capturable.
// Per walk, scr holds kEstScratch vectors of np doubles: X0 X1 T0 T1 Y0 Y1 H VIS, and est
// holds 4 doubles: (estimate, best index, done, unused).
__device__ __forceinline__ double probe_sign_d(int64_t i) {
  const uint32_t h = (uint32_t)((uint64_t)i * 0x9E3779B1ull);
  return (h >> 31) & 1 ? -1.0 : 1.0;
}
__device__ __forceinline__ double* est_vec(double* scr, const BWalk& b, int k) {
  return scr + (int64_t)kEstScratch * b.row0 + (int64_t)k * b.np;
}
enum { kEX0, kEX1, kET0, kET1, kEY0, kEY1, kEH, kEVIS };

__global__ void kb_est_init(const int* list, const BWalk* wk, double* scr, double* est) {
  const int w = list[blockIdx.x];
  const BWalk b = wk[w];
  double* X0 = est_vec(scr, b, kEX0);
  double* X1 = est_vec(scr, b, kEX1);
  double* VIS = est_vec(scr, b, kEVIS);
  for (int i = threadIdx.x; i < b.np; i += blockDim.x) {
    X0[i] = i < b.n ? 1.0 / b.n : 0.0;
    X1[i] = (i < b.n && b.n > 1) ? probe_sign_d(i) / b.n : 0.0;
    VIS[i] = 0.0;
  }
  if (threadIdx.x == 0) {
    est[4 * w] = 0.0;
    est[4 * w + 1] = 0.0;
    est[4 * w + 2] = 0.0;
  }
}
// (out0, out1) = M (in0, in1) on the chunk's rows of its walk, unless that walk is done; warp
// per row.
__global__ void kb_est_matvec(const double* M, const RChunk* ch, const BWalk* wk, double* scr, const double* est,
                              int in0, int out0) {
  const RChunk q = ch[blockIdx.x];
  const int w = q.w;
  if (est[4 * w + 2] != 0.0) return;
  const BWalk b = wk[w];
  const double* x0 = est_vec(scr, b, in0);
  const double* x1 = est_vec(scr, b, in0 + 1);
  double* y0 = est_vec(scr, b, out0);
  double* y1 = est_vec(scr, b, out0 + 1);
  const double* A = M + b.off;
  const int lane = threadIdx.x & 31, wpb = blockDim.x / 32;
  // 16-byte loads (np and every row start are even), two steps per iteration in flight
  const int64_t h = b.np / 2;
  const double2* u0 = reinterpret_cast<const double2*>(x0);
  const double2* u1 = reinterpret_cast<const double2*>(x1);
  for (int64_t i = q.r0 + threadIdx.x / 32; i < q.r1; i += wpb) {
    const double2* row = reinterpret_cast<const double2*>(A + i * b.np);
    double a = 0, c = 0;
#pragma unroll 2
    for (int64_t j = lane; j < h; j += 32) {
      const double2 m = row[j], p = u0[j], r = u1[j];
      a += m.x * p.x;
      a += m.y * p.y;
      c += m.x * r.x;
      c += m.y * r.y;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_xor_sync(0xffffffffu, a, o);
      c += __shfl_xor_sync(0xffffffffu, c, o);
    }
    if (lane == 0) {
      y0[i] = a;
      y1[i] = c;
    }
  }
}
// The same pair of mat-vecs from an FP32 copy of M (the Lanczos steps: half the bytes of the
// FP64 plane; the rounding moves the spectrum by ~1e-7 of its radius, far inside the margins
// the estimate is used with).  16-byte loads of four values, FP64 accumulation.
__global__ void kb_est_matvec32(const float* M, const RChunk* ch, const BWalk* wk, double* scr, const double* est,
                                int in0, int out0) {
  const RChunk q = ch[blockIdx.x];
  const int w = q.w;
  if (est[4 * w + 2] != 0.0) return;
  const BWalk b = wk[w];
  const double* x0 = est_vec(scr, b, in0);
  const double* x1 = est_vec(scr, b, in0 + 1);
  double* y0 = est_vec(scr, b, out0);
  double* y1 = est_vec(scr, b, out0 + 1);
  const float* A = M + b.off;
  const int lane = threadIdx.x & 31, wpb = blockDim.x / 32;
  const int64_t h = b.np / 4;   // np is a multiple of 128: rows start 16-byte aligned
  const double2* u0 = reinterpret_cast<const double2*>(x0);
  const double2* u1 = reinterpret_cast<const double2*>(x1);
  for (int64_t i = q.r0 + threadIdx.x / 32; i < q.r1; i += wpb) {
    const float4* row = reinterpret_cast<const float4*>(A + i * b.np);
    double a = 0, c = 0;
#pragma unroll 2
    for (int64_t j = lane; j < h; j += 32) {
      const float4 m = row[j];
      const double2 p0 = u0[2 * j], p1 = u0[2 * j + 1], r0 = u1[2 * j], r1 = u1[2 * j + 1];
      a += (double)m.x * p0.x;
      a += (double)m.y * p0.y;
      a += (double)m.z * p1.x;
      a += (double)m.w * p1.y;
      c += (double)m.x * r0.x;
      c += (double)m.y * r0.y;
      c += (double)m.z * r1.x;
      c += (double)m.w * r1.y;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_xor_sync(0xffffffffu, a, o);
      c += __shfl_xor_sync(0xffffffffu, c, o);
    }
    if (lane == 0) {
      y0[i] = a;
      y1[i] = c;
    }
  }
}

// ---- Lanczos estimate of the spectral radius of every walk's real symmetric generator B
// (the imaginary plane of the shifted Y): two independent runs of kLanSteps steps from
// pseudo-random sign vectors, sharing kb_est_matvec (X0, X1 -> T0, T1), without
// reorthogonalisation (the extreme Ritz values, all this needs, stay inside the spectrum).
// Per walk and run, lan holds (alpha_j, beta_j) for j < kLanSteps; Y0 / Y1 keep v_{j-1}.
constexpr int kLanSteps = 30;
__device__ double block_reduce(double v, double* sh, bool take_max);
__device__ __forceinline__ double probe_sign_d2(int64_t i) {
  const uint32_t h = (uint32_t)((uint64_t)(i + 977) * 0x85EBCA6Bull) ^ 0x27D4EB2Fu;
  return ((h * 0xC2B2AE35u) >> 31) & 1 ? -1.0 : 1.0;
}
__global__ void kb_lan_init(const int* list, const BWalk* wk, double* scr, double* est) {
  const int w = list[blockIdx.x];
  const BWalk b = wk[w];
  double* X0 = est_vec(scr, b, kEX0);
  double* X1 = est_vec(scr, b, kEX1);
  double* Y0 = est_vec(scr, b, kEY0);
  double* Y1 = est_vec(scr, b, kEY1);
  const double inv = 1.0 / sqrt((double)b.n);
  for (int i = threadIdx.x; i < b.np; i += blockDim.x) {
    X0[i] = i < b.n ? probe_sign_d(i) * inv : 0.0;
    X1[i] = i < b.n ? probe_sign_d2(i) * inv : 0.0;
    Y0[i] = 0.0;
    Y1[i] = 0.0;
  }
  if (threadIdx.x == 0) est[4 * w + 2] = 0.0;   // kb_est_matvec skips walks marked done
}
// After T_r = B X_r: alpha = T.v, w = T - alpha v - beta_prev v_prev, beta = |w|, v_prev <- v,
// v <- w / beta (v <- 0 once the Krylov space is exhausted).
// One block per (walk, run): blockIdx.x = 2 * (index in list) + run; blockDim a power of two up
// to 1024.
__global__ void kb_lan_step(const int* list, const BWalk* wk, double* scr, double* lan, int j) {
  const int w = list[blockIdx.x >> 1], r = blockIdx.x & 1;
  const BWalk b = wk[w];
  __shared__ double sh[1024];
  double* v = est_vec(scr, b, kEX0 + r);
  const double* t = est_vec(scr, b, kET0 + r);
  double* vp = est_vec(scr, b, kEY0 + r);
  double* rec = lan + ((int64_t)w * 2 + r) * 2 * kLanSteps;
  const double bprev = j > 0 ? rec[2 * (j - 1) + 1] : 0.0;
  double a = 0.0;
  for (int i = threadIdx.x; i < b.n; i += blockDim.x) a += t[i] * v[i];
  a = block_reduce(a, sh, false);
  double nn = 0.0;
  for (int i = threadIdx.x; i < b.n; i += blockDim.x) {
    const double x = t[i] - a * v[i] - bprev * vp[i];
    nn += x * x;
  }
  const double beta = sqrt(block_reduce(nn, sh, false));
  const double scale = beta > 1e-300 ? 1.0 / beta : 0.0;
  for (int i = threadIdx.x; i < b.n; i += blockDim.x) {
    const double x = t[i] - a * v[i] - bprev * vp[i];
    vp[i] = v[i];
    v[i] = x * scale;
  }
  if (threadIdx.x == 0) {
    rec[2 * j] = a;
    rec[2 * j + 1] = beta;
  }
}
__device__ double block_reduce(double v, double* sh, bool take_max) {
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] = take_max ? fmax(sh[threadIdx.x], sh[threadIdx.x + o]) : sh[threadIdx.x] + sh[threadIdx.x + o];
    __syncthreads();
  }
  const double r = sh[0];
  __syncthreads();
  return r;
}
// argmax of val over i < n with skip[i] == 0 and i != excl (ties to the lower index); -1 if none.
__device__ int block_argmax(const double* val, const double* skip, int n, int excl, double* shv, int* shi) {
  double best = -1.0;
  int bi = -1;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    if (skip[i] != 0.0 || i == excl) continue;
    const double v = val[i];
    if (bi < 0 || v > best) {
      best = v;
      bi = i;
    }
  }
  shv[threadIdx.x] = best;
  shi[threadIdx.x] = bi;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      const int j = threadIdx.x + o;
      const int ia = shi[threadIdx.x], ib = shi[j];
      const double va = shv[threadIdx.x], vb = shv[j];
      bool take_b = false;
      if (ib >= 0) {
        if (ia < 0) take_b = true;
        else if (vb > va) take_b = true;
        else if (vb == va && ib < ia) take_b = true;
      }
      if (take_b) {
        shv[threadIdx.x] = vb;
        shi[threadIdx.x] = ib;
      }
    }
    __syncthreads();
  }
  const int r = shi[0];
  __syncthreads();
  return r;
}
// After Y = M0 M1 X: the estimate of round k; stop, or S = sign(Y) -> X.
__global__ void kb_est_step1(const int* list, const BWalk* wk, double* scr, double* est, int k) {
  const int w = list[blockIdx.x];
  if (est[4 * w + 2] != 0.0) return;
  const BWalk b = wk[w];
  __shared__ double sh[256];
  const double* Y0 = est_vec(scr, b, kEY0);
  const double* Y1 = est_vec(scr, b, kEY1);
  double* X0 = est_vec(scr, b, kEX0);
  double* X1 = est_vec(scr, b, kEX1);
  const int t = b.n > 1 ? 2 : 1;
  const double old = est[4 * w];   // read before any thread can write it below
  double c0 = 0, c1 = 0;
  for (int i = threadIdx.x; i < b.n; i += blockDim.x) {
    c0 += fabs(Y0[i]);
    c1 += fabs(Y1[i]);
  }
  c0 = block_reduce(c0, sh, false);
  c1 = block_reduce(c1, sh, false);
  const double e = (t == 2 && c1 > c0) ? c1 : c0;
  if ((k >= 2 && e <= old) || k == 5) {
    if (threadIdx.x == 0) {
      if (!(k >= 2 && e <= old)) est[4 * w] = e;
      est[4 * w + 2] = 1.0;
    }
    return;
  }
  for (int i = threadIdx.x; i < b.np; i += blockDim.x) {
    X0[i] = i < b.n ? (Y0[i] != 0.0 ? (Y0[i] > 0 ? 1.0 : -1.0) : 1.0) : 0.0;
    X1[i] = (i < b.n && t == 2) ? (Y1[i] != 0.0 ? (Y1[i] > 0 ? 1.0 : -1.0) : 1.0) : 0.0;
  }
  if (threadIdx.x == 0) est[4 * w] = e;
}
// After Z = M1 M0 S (in Y): stop, or the next two unit columns.
__global__ void kb_est_step2(const int* list, const BWalk* wk, double* scr, double* est, int k) {
  const int w = list[blockIdx.x];
  if (est[4 * w + 2] != 0.0) return;
  const BWalk b = wk[w];
  __shared__ double shv[256];
  __shared__ int shi[256];
  const double* Y0 = est_vec(scr, b, kEY0);
  const double* Y1 = est_vec(scr, b, kEY1);
  double* X0 = est_vec(scr, b, kEX0);
  double* X1 = est_vec(scr, b, kEX1);
  double* H = est_vec(scr, b, kEH);
  double* VIS = est_vec(scr, b, kEVIS);
  const int t = b.n > 1 ? 2 : 1;
  double hm = 0.0;
  for (int i = threadIdx.x; i < b.np; i += blockDim.x) {
    const double h = i < b.n ? (t == 2 ? fmax(fabs(Y0[i]), fabs(Y1[i])) : fabs(Y0[i])) : 0.0;
    H[i] = h;
    hm = fmax(hm, h);
  }
  hm = block_reduce(hm, shv, true);   // also orders the H writes before the reads below
  const int best = (int)est[4 * w + 1];   // written (by thread 0) only after the last barrier
  if (k >= 2 && hm <= H[best]) {
    if (threadIdx.x == 0) est[4 * w + 2] = 1.0;
    return;
  }
  const int p0 = block_argmax(H, VIS, b.n, -1, shv, shi);
  const int p1 = t == 2 ? block_argmax(H, VIS, b.n, p0, shv, shi) : -1;
  if (p0 < 0 || (t == 2 && p1 < 0)) {
    if (threadIdx.x == 0) est[4 * w + 2] = 1.0;
    return;
  }
  for (int i = threadIdx.x; i < b.np; i += blockDim.x) {
    X0[i] = i == p0 ? 1.0 : 0.0;
    X1[i] = (t == 2 && i == p1) ? 1.0 : 0.0;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    VIS[p0] = 1.0;
    if (p1 >= 0) VIS[p1] = 1.0;
    est[4 * w + 1] = p0;
  }
}
__global__ void kb_est_final(const int* list, int nlist, const double* est, double* out, int stride, int slot) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nlist) return;
  const int w = list[i];
  out[(int64_t)w * stride + slot] = est[4 * w];
}

// U = e^mu (I + E + cj J) on the n x n block, written to the walk's interleaved output.
template <typename C>
__global__ void kb_output(const double* const* Ere, const double* const* Eim, void* const* U, const int* list,
                          const BWalk* wk, const double* om) {
  const int w = list[blockIdx.y];
  C* u = (C*)U[w];
  if (!u) return;
  const BWalk b = wk[w];
  const double* er = Ere[w] + b.off;
  const double* ei = Eim[w] + b.off;
  const double* o = om + 4 * w;
  const int64_t n2 = (int64_t)b.n * b.n;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < n2;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = idx / b.n, j = idx - i * b.n;
    double a = er[i * b.np + j] + o[2] + (i == j ? 1.0 : 0.0);
    double c = ei[i * b.np + j] + o[3];
    C v;
    v.x = (decltype(v.x))(o[0] * a - o[1] * c);
    v.y = (decltype(v.y))(o[0] * c + o[1] * a);
    u[idx] = v;
  }
}

unsigned grid_x_for(int64_t max_elems, int nlist) {
  // enough CTAs per walk to cover the largest block with ~8 elements per thread, and enough
  // in total to fill the GPU a few times over
  int64_t per = (max_elems + 2047) / 2048;
  int64_t want = std::max<int64_t>(1, (148 * 16 + nlist - 1) / std::max(1, nlist));
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(per, std::max<int64_t>(want, 1)));
}

// Al-Mohy & Higham (2009), Table 3.1 (theta_13 = 4.25 of their Algorithm 6.1).
const double kTheta3 = 1.495585217958292e-2, kTheta5 = 2.539398330063230e-1,
             kTheta7 = 9.504178996162932e-1, kTheta9 = 2.097847961257068e0, kTheta13 = 4.25;
double factorial(int k) {
  double f = 1;
  for (int i = 2; i <= k; ++i) f *= i;
  return f;
}
std::vector<double> pade_coeffs(int m) {
  std::vector<double> b(m + 1);
  for (int j = 0; j <= m; ++j) b[j] = factorial(2 * m - j) / (factorial(j) * factorial(m - j));
  return b;
}
int pade_products(int m) { return m == 3 ? 2 : m == 5 ? 3 : m == 7 ? 4 : m == 9 ? 5 : 6; }

// ---- certified truncation bound for normal generators Y = i B (B real symmetric).
// The [m/m] Pade approximant maps the imaginary axis onto the unit circle, r_m(ix) =
// p_m(ix) / conj(p_m(ix)), so its only error at an eigenvalue i lambda is the phase
// phi_m(x) = 2 arg p_m(ix) - x, x = lambda / 2^s, and after s squarings 2^s phi_m(x).  |phi_m| is
// increasing in |x| until the phase wraps (|phi| = pi near x = 10, 14.4, 18.7, 23, 31.4 for
// m = 3..13); below half that point the error over every |lambda| <= rho is at most
// 2^s |phi_m(rho / 2^s)|.  rho_up = min(||Y||_1, d4, d6) bounds the spectral radius (exact
// norms of powers), so the bound holds for every eigenvalue.
const int kDegrees[5] = {3, 5, 7, 9, 13};
double pade_phase_error(int m, double x) {
  const std::vector<double> b = pade_coeffs(m);
  const std::complex<double> z(0.0, x);
  std::complex<double> acc(0.0, 0.0);
  for (int j = m; j >= 0; --j) acc = acc * z + b[j];
  return std::remainder(2.0 * std::atan2(acc.imag(), acc.real()) - x, 2.0 * M_PI);
}
double pade_x_limit(int m) { return m == 3 ? 5.0 : m == 5 ? 7.2 : m == 7 ? 9.3 : m == 9 ? 11.4 : 15.6; }
bool certified(int m, int s, double rho_up, double tol) {
  const double x = std::ldexp(rho_up, -s);
  if (x > pade_x_limit(m)) return false;
  return std::ldexp(std::fabs(pade_phase_error(m, x)), s) <= tol;
}
// Cheapest (m, s) (products pi_m + s; ties to the larger m) that the bound certifies.
void certified_choice(double rho_up, double tol, int* m_out, int* s_out) {
  int bm = 13, bs = 0, best = 1 << 30;
  for (int m : kDegrees) {
    int s = 0;
    while (s < 200 && !certified(m, s, rho_up, tol)) ++s;
    const int cost = pade_products(m) + s;
    if (cost <= best) {
      best = cost;
      bm = m;
      bs = s;
    }
  }
  *m_out = bm;
  *s_out = bs;
}
// Phase tolerance of the certified and learned selections: 1e-6 per eigenvalue keeps the
// infidelity of any state below 1e-12 and the relative error of U below 1e-6.
constexpr double kPhaseTol = 1e-6;
// Spectral radius from the Lanczos coefficients of one run (alpha_j, beta_j interleaved, k
// steps): the extreme eigenvalues of the k x k tridiagonal, by Sturm-sequence bisection inside
// Gershgorin bounds.  Ritz values lie inside the spectrum, so this never exceeds the radius.
double tridiag_radius(const double* ab, int k) {
  // a run whose Krylov space ran out has beta = 0: the tridiagonal ends there
  int kk = k;
  for (int j = 0; j + 1 < k; ++j)
    if (!(ab[2 * j + 1] > 0.0)) {
      kk = j + 1;
      break;
    }
  double lo = 1e300, hi = -1e300;
  for (int i = 0; i < kk; ++i) {
    const double off = (i > 0 ? std::fabs(ab[2 * (i - 1) + 1]) : 0.0) + (i + 1 < kk ? std::fabs(ab[2 * i + 1]) : 0.0);
    lo = std::min(lo, ab[2 * i] - off);
    hi = std::max(hi, ab[2 * i] + off);
  }
  if (!(lo <= hi)) return 0.0;
  auto below = [&](double x) {   // eigenvalues < x
    int cnt = 0;
    double q = 1.0;
    for (int i = 0; i < kk; ++i) {
      const double b2 = i > 0 ? ab[2 * (i - 1) + 1] * ab[2 * (i - 1) + 1] : 0.0;
      q = ab[2 * i] - x - (i > 0 ? b2 / q : 0.0);
      if (q == 0.0) q = -1e-300;
      if (q < 0.0) ++cnt;
    }
    return cnt;
  };
  auto kth = [&](int want) {   // the smallest x with below(x) >= want
    double a = lo, b = hi;
    for (int it = 0; it < 200 && b - a > 1e-14 * std::max(std::fabs(a), std::fabs(b)); ++it) {
      const double m = 0.5 * (a + b);
      if (below(m) >= want) b = m;
      else a = m;
    }
    return 0.5 * (a + b);
  };
  return std::max(std::fabs(kth(1)), std::fabs(kth(kk)));
}
// Relative margin on the Lanczos estimate in the estimated selection (selector 3) and in the
// gate of the learned selection.
constexpr double kLanMargin = 0.10;
// Phase tolerance of the learned selection's gate: a phase error phi at the spectrum's edges
// gives an infidelity of at most sin^2(phi) for any state, so 1e-5 keeps it below 1e-10.
constexpr double kGateTol = 1e-5;

}  // namespace

// ---- Chebyshev-Bessel polynomial stage for walk generators Y = i B (FX_OPT_APPROX = 1).
// On [-1, 1], e^{iaz} = J_0(a) + 2 sum_{k>=1} i^k J_k(a) T_k(z) (Jacobi-Anger; Tal-Ezer &
// Kosloff 1984).  With rho >= the spectral radius of B, Z = B / rho and a = rho / 2^s, the
// polynomial truncated after degree D approximates e^{iB/2^s} to 2 sum_{k>D} |J_k(a)| on the
// whole spectrum, and the s squarings multiply that by at most 2^s.  No Pade solve: every step
// is a product of two commuting real symmetric matrices (polynomials in B).
//
// Evaluation: even part sum_j e_j T_j(C) with C = T_2(Z) = 2Z^2 - I (T_2j(Z) = T_j(C)); odd part
// Z sum_j b_j T_j(C), its coefficients moved from T_2k+1(Z) onto Z T_j(C) =
// (T_2j+1(Z) + T_2j-1(Z)) / 2; each part written as sum_g T_g(G) r_g(C) with G = T_m(C) and
// deg r_g < m (baby steps T_1..T_m of C; T_g(T_m) = T_gm) and summed by Clenshaw's recurrence in
// G.  The plan (s, D, m) is the cheapest in matrix products, kChebSquareProducts per squaring.
constexpr int kChebMaxBaby = 5;          // baby steps T_1..T_5 of C (arenas)
constexpr int kChebSquareProducts = 3;   // cost of one squaring in the plan
constexpr double kChebMaxA = 1024.0;     // larger a would need hundreds of products: skipped
// Margin on the Lanczos estimate where the selection uses it: outside [-1, 1] the truncated
// series grows like cosh(D acosh|z|), so the interval must hold the whole spectrum.
constexpr double kChebLanMargin = 0.25;
// Error bound of the polynomial after the squarings: the phase tolerance of the selections
// (1e-6) for complex64 walks; for complex128 walks a bound far below the int8 products' own
// rounding (35-bit slices), so that the truncation never adds to it.
constexpr double kChebTolC128 = 1e-12;

// J_0(a) .. J_kmax(a), a >= 0, by Miller's backward recurrence J_{k-1} = (2k / a) J_k - J_{k+1}
// from far above max(kmax, a), normalised by J_0 + 2 sum_{k>=1} J_2k = 1 (Abramowitz & Stegun
// 9.1.27, 9.1.46).
std::vector<double> bessel_j(double a, int kmax) {
  std::vector<double> out((size_t)kmax + 1, 0.0);
  if (a == 0.0) {
    out[0] = 1.0;
    return out;
  }
  int top = std::max(kmax, (int)a) + 20 + (int)std::sqrt(40.0 * std::max((double)kmax, a));
  top += top & 1;
  std::vector<double> v((size_t)top + 1, 0.0);
  double jp = 0.0, j = 1e-300;
  v[top] = j;
  for (int k = top; k > 0; --k) {
    const double jm = (2.0 * k / a) * j - jp;
    jp = j;
    j = jm;
    v[k - 1] = j;
    if (std::fabs(j) > 1e250) {
      for (int i = k - 1; i <= top; ++i) v[i] *= 1e-250;
      jp *= 1e-250;
      j *= 1e-250;
    }
  }
  double norm = 0.0;
  for (int k = 2; k <= top; k += 2) norm += v[k];
  norm = v[0] + 2.0 * norm;
  for (int k = 0; k <= kmax; ++k) out[k] = v[k] / norm;
  return out;
}
// Smallest D with 2 sum_{k>D} |J_k(a)| <= tol.
int cheb_degree(double a, double tol) {
  const int kmax = (int)a + 80 + (int)(8.0 * std::pow(std::max(a, 1.0), 1.0 / 3.0));
  const std::vector<double> J = bessel_j(a, kmax);
  std::vector<double> tail((size_t)kmax + 2, 0.0);
  for (int k = kmax; k >= 0; --k) tail[k] = tail[k + 1] + std::fabs(J[k]);
  for (int d = 0; d < kmax; ++d)
    if (2.0 * tail[d + 1] <= tol) return d;
  return kmax;
}
// Degrees in C of the even part and of the odd part's cofactor (-1: none).
void cheb_parts(int D, int* je, int* jo) {
  *je = D / 2;
  *jo = D >= 1 ? (D - 1) / 2 : -1;
}
// Highest baby step T_k(C) the plan computes: G = T_m when a chain has a giant step, else the
// parts' own degree (their sums are then linear combinations of T_0..T_top).
int cheb_baby_top(int D, int m) {
  int je, jo;
  cheb_parts(D, &je, &jo);
  if (D <= 1) return 0;
  if (je / m >= 1 || (jo >= 0 && jo / m >= 1)) return m;
  return std::max(je, jo);
}
// Products of the polynomial stage: baby steps T_2..T_top, the two Clenshaw chains (floor(j / m)
// products each) and the product by Z of the odd chain (none when its degree is 0).
int cheb_plan_cost(int D, int m) {
  int je, jo;
  cheb_parts(D, &je, &jo);
  if (D <= 1) return 0;
  return std::max(cheb_baby_top(D, m) - 1, 0) + je / m + (jo >= 1 ? jo / m + 1 : 0);
}
struct ChebPlan {
  int s = 0, degree = 0, baby = 1, cost = 0;
  double a = 0.0;
  bool ok = false;   // false: rho / 2^60 above kChebMaxA (no plan)
};
// The cheapest (s, D, m) for the spectral bound rho at error tol after the squarings (ties to
// the smaller s and the smaller m).
ChebPlan cheb_plan(double rho, double tol) {
  ChebPlan best;
  bool have = false;
  for (int s = 0; s <= 60; ++s) {
    const double a = std::ldexp(rho, -s);
    if (a > kChebMaxA) continue;
    const int D = cheb_degree(a, std::ldexp(tol, -s));
    int bc = 0, bm = 1;
    for (int m = 1; m <= kChebMaxBaby; ++m) {
      const int c = cheb_plan_cost(D, m);
      if (m == 1 || c < bc) {
        bc = c;
        bm = m;
      }
    }
    const int tot = bc + kChebSquareProducts * s;
    if (!have || tot < best.cost) {
      best.s = s;
      best.degree = D;
      best.baby = bm;
      best.cost = tot;
      best.a = a;
      best.ok = have = true;
    }
    if (a < 1e-3) break;
  }
  return best;
}
// Coefficients of the plan's two parts: e_j of sum_j e_j T_j(C) (even) and b_j of
// Z sum_j b_j T_j(C) (odd): b_jo = 2 o_jo, b_k = 2 o_k - b_{k+1}, b_0 = o_0 - b_1 / 2, with
// o_k = 2 (-1)^k J_2k+1(a) the coefficient of T_2k+1(Z).
void cheb_split(double a, int D, std::vector<double>* e, std::vector<double>* b) {
  const std::vector<double> J = bessel_j(a, std::max(D, 1));
  int je, jo;
  cheb_parts(D, &je, &jo);
  e->assign((size_t)je + 1, 0.0);
  (*e)[0] = J[0];
  for (int j = 1; j <= je; ++j) (*e)[j] = 2.0 * ((j & 1) ? -1.0 : 1.0) * J[2 * j];
  b->clear();
  if (jo < 0) return;
  std::vector<double> o((size_t)jo + 1), bb((size_t)jo + 2, 0.0);
  for (int k = 0; k <= jo; ++k) o[k] = 2.0 * ((k & 1) ? -1.0 : 1.0) * J[2 * k + 1];
  for (int k = jo; k >= 1; --k) bb[k] = 2.0 * o[k] - bb[k + 1];
  bb[0] = o[0] - 0.5 * bb[1];
  b->assign(bb.begin(), bb.begin() + jo + 1);
}
// r[g][j] (j < m) with sum_k x_k T_k(C) = sum_g T_g(T_m(C)) sum_j r[g][j] T_j(C): from the top
// degree down, r[g][j] = 2 x_k and x_{gm-j} -= x_k for g, j >= 1 (T_gm T_j = (T_gm+j + T_gm-j) / 2),
// else r[g][j] = x_k.
std::vector<std::array<double, kChebMaxBaby>> cheb_blocks(std::vector<double> x, int m) {
  const int L = ((int)x.size() - 1) / m;
  std::vector<std::array<double, kChebMaxBaby>> r((size_t)L + 1);
  for (auto& row : r) row.fill(0.0);
  for (int k = (int)x.size() - 1; k >= 0; --k) {
    const int g = k / m, j = k % m;
    if (g == 0 || j == 0) {
      r[g][j] = x[k];
    } else {
      r[g][j] = 2.0 * x[k];
      x[g * m - j] -= x[k];
    }
  }
  return r;
}

namespace {

// Process-wide weights of the learned selector (device copy; fx_selector_set_weights).
std::mutex g_sel_mu;
float* g_sel_weights = nullptr;
int g_sel_device = -1;

struct DevArena {
  void* p = nullptr;
  size_t bytes = 0;
  void alloc(size_t b) {
    release();
    if (b == 0) return;
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
  ~DevArena() { release(); }
};

// Host staging of the small device descriptors of a launch sequence, uploaded in one copy.
struct Staging {
  std::vector<unsigned char> buf;
  template <typename T>
  size_t put(const T* data, size_t count) {
    size_t off = (buf.size() + 255) & ~(size_t)255;
    buf.resize(off + sizeof(T) * count);
    if (count) std::memcpy(buf.data() + off, data, sizeof(T) * count);
    return off;
  }
  template <typename T>
  size_t put(const std::vector<T>& v) {
    return put(v.data(), v.size());
  }
};

}  // namespace

// ================================================================== batch pipeline
class BatchPipeline {
 public:
  BatchPipeline(const std::vector<int64_t>& ns, int dtype) : dtype_(dtype) {
    const int W = (int)ns.size();
    walks_.resize(W);
    int64_t off = 0, row = 0;
    maxnp_ = kNb;
    for (int w = 0; w < W; ++w) {
      const int64_t n = ns[w];
      if (n <= 0 || n > 32768) throw Error{FX_ERR_VALUE, "batched walk sizes must be 1..32768"};
      const int64_t np = pad_n(n);
      walks_[w] = BWalk{(int)n, (int)np, off, row};
      off += np * np;
      row += np;
      maxnp_ = std::max<int64_t>(maxnp_, np);
    }
    elems_ = off;
    rows_ = row;
    pitch_ = maxnp_;
    for (int a = 0; a < kBaseArenas; ++a) arena_[a].alloc(sizeof(double) * (size_t)std::max<int64_t>(elems_, 1));
    // int8 slice planes: A re (2 rows per walk row: the two planes of a complex left factor
    // side by side), A im, A -im, B re; 5 slices each.
    a_rows_ = 2 * rows_;
    const size_t sl = (size_t)pitch_ * (size_t)(a_rows_ + 3 * rows_) * kS;
    slices_.alloc(sl);
    exps_.alloc(sizeof(int) * (size_t)(a_rows_ + rows_ + 64));
    diag_.alloc(sizeof(double) * (size_t)(a_rows_ + rows_ + 64));
    linv_.alloc(sizeof(double) * (size_t)rows_ * kNb * 2);
    lanc_.alloc(sizeof(double) * (size_t)W * 4 * kLanSteps);
    // small: rowstat (kRS per row), estimator vectors (kEstScratch per row), row sums (1 per
    // row), per-walk records (8 + 8 + 4 + 8 + W ints)
    small_.alloc(sizeof(double) * (size_t)(rows_ * (kRS + kEstScratch + 2) + (kWO + 8 + 4 + 8 + 8) * W + 64));
    err_.alloc(sizeof(int) * 8);
    d_walks_.alloc(sizeof(BWalk) * W);
    FX_CUDA(cudaMemcpy(d_walks_.p, walks_.data(), sizeof(BWalk) * W, cudaMemcpyHostToDevice));
    ptrs_.alloc(sizeof(void*) * 4 * W);
    sel_m_.assign(W, 13);
    sel_s_.assign(W, 0);
    cheb_deg_.assign(W, -1);
    cheb_baby_.assign(W, 1);
    cheb_rho_.assign(W, 0.0);
    rank1_.assign(W, 0);
    mu_.assign(W, {0, 0});
    nu_.assign(W, {0, 0});
    norms_.assign(8 * W, 0.0);
    record_phase1();
  }
  ~BatchPipeline() {
    if (graph1_) cudaGraphExecDestroy(graph1_);
    if (graph2_) cudaGraphExecDestroy(graph2_);
    for (cudaEvent_t e : ev_pool_) cudaEventDestroy(e);
    for (cudaEvent_t e : phase_ev_) cudaEventDestroy(e);
  }

  int count() const { return (int)walks_.size(); }
  int64_t n_of(int w) const { return walks_[w].n; }
  void selection(int w, int* m, int* s) const {
    *m = sel_m_[w];
    *s = sel_s_[w];
  }
  int launches() const { return launches_; }
  double flops() const { return flops_; }
  void set_graph(bool g) { use_graph_ = g; }
  void set_timeout(unsigned ms) { timeout_ms_ = ms; }
  void set_profile(bool p) { profile_ = p; }
  // 0 plain (Al-Mohy & Higham), 1 certified bound, 2 learned (gated by the bound), 3 estimated.
  // Phase 1 runs the Lanczos estimate only where a selection or the form needs it.
  // Phase 1 runs the 1-norm estimates of A^8 and A^10 only where the Al-Mohy & Higham
  // selection itself is made (plain and certified selections, analyze-only runs); the
  // estimated and learned selections take the plain choice, their fallback, from the bounds
  // ||A^8|| <= ||A^4||^2 and ||A^10|| <= ||A^4|| ||A^6|| (a choice with as many squarings or
  // more).
  void set_selector(int k) {
    const int before = phase1_needs();
    selector_ = k;
    if (phase1_needs() != before) rerecord_phase1();
  }
  bool needs_lanczos() const { return selector_ >= 2 || form_ == 1 || analyze_only_; }
  bool needs_estimates() const { return selector_ <= 1 || analyze_only_; }
  // A^4 and A^6 are products of phase 1 for the exact norms d4, d6 (the Al-Mohy & Higham
  // selection, the rigorous spectral bound, the Pade stage's operands).  When every walk takes
  // the Chebyshev polynomial on the Lanczos bound (estimated or learned selection, nothing
  // forced), they serve only as the cap min(||Y||_1, d4, d6) of that bound, and phase 1 computes
  // A2 alone: the cap is then min(||Y||_1, ||A2||_1^(1/2)) (||A^4|| <= ||A2||^2 and
  // ||A^6|| <= ||A2||^3 stand in for the exact norms), still a rigorous bound.
  bool needs_powers46() const {
    bool forced = force_m_ > 0 || force_s_ >= 0;
    for (int m : pw_m_) forced = forced || m > 0;
    return !(approx_ == 1 && selector_ >= 2 && !analyze_only_ && !forced);
  }
  int phase1_needs() const {
    return (needs_lanczos() ? 1 : 0) | (needs_estimates() ? 2 : 0) | (needs_powers46() ? 4 : 0);
  }
  void rerecord_phase1() {
    if (graph1_) cudaGraphExecDestroy(graph1_);
    graph1_ = nullptr;
    st1_ = Staging();
    r1_ = Rec();
    desc1_.release();
    record_phase1();
    key2_.clear();
  }
  // Stop after the selection (statistics, norms, estimates, features; no exponential).
  void set_analyze_only(bool a) {
    const int before = phase1_needs();
    analyze_only_ = a;
    if (phase1_needs() != before) rerecord_phase1();
  }
  // Phase-2 schedule: tune it at the next run, or set it.
  void set_autotune(bool a) { autotune_ = a; }
  void set_schedule(int group, int order) {
    tile_group_ = group;
    tile_order_ = order;
    key2_.clear();
  }
  void schedule(int* group, int* order) const {
    *group = tile_group_;
    *order = tile_order_;
  }
  const std::vector<std::array<double, 3>>& tuned() const { return tuned_; }
  // Diagonal split, a mask: 1 the real products (V^2, W^2, VW, and every product of the mixed
  // form); 2 the complex products P2 L^-T and Z L^-1; 4 the plain form's powers and Pade
  // products; 8 the plain form's squarings as three split products (as the mixed form's).
  // Default 7; changing it re-records both phases.
  void set_diag_split(int v) {
    if (v == split_) return;
    split_ = v;
    rerecord_phase1();
  }
  int selector() const { return selector_; }
  // Spectral-radius estimates of walk w in the last run: Lanczos (a lower estimate) and the
  // rigorous upper bound min(||Y||_1, d4, d6).
  void spectral(int w, double* rho_lanczos, double* rho_up) const {
    *rho_lanczos = rho_lan_.empty() ? 0.0 : rho_lan_[w];
    *rho_up = rho_up_.empty() ? 0.0 : rho_up_[w];
  }
  // Diagnostics of the failure path: product launch k (k >= 0) of every run leaves the loads of
  // its first K step out, so that its bounded waits run out; runs are then replayed eagerly.
  void set_inject_stall(int k) { inject_ = k; }
  // Precision form of the squarings: 0 plain (every squaring the exact complex square, 4 real
  // products at 5 slices); 1 mixed (each squaring as the two real products (Er + Ei)(Er - Ei)
  // and 2 Er Ei, 5 slices except the last n4 + n3 squarings: n4 at 4 slices, then n3 at 3).
  void set_form(int form, int n4, int n3, int pade_slices = kS, int newton_slices = kS) {
    if (newton_slices != newton_S_) {   // read when phase 2 is recorded
      newton_S_ = newton_slices;
      key2_.clear();
    }
    if (form == form_ && n4 == sq_n4_ && n3 == sq_n3_ && pade_slices == pade_S_) return;
    const bool rerecord = form != form_ || (form == 1 && pade_slices != pade_S_);
    form_ = form;
    sq_n4_ = n4;
    sq_n3_ = n3;
    pade_S_ = pade_slices;
    key2_.clear();
    // phase 1's powers take the form's slice count and diagonal split
    if (rerecord) rerecord_phase1();
  }
  int pade_slices() const { return pade_S_; }
  // Solve of the walk-generator Pade step: 0 Newton-Schulz for walks padded to 4096 or more and
  // Cholesky otherwise, 1 Cholesky, 2 Newton-Schulz.
  void set_solve(int mode) {
    if (mode == solve_mode_) return;
    solve_mode_ = mode;
    key2_.clear();
  }
  // Approximant of the walk generators' exponential before the squarings: 0 Pade with its
  // solve, 1 the Chebyshev-Bessel polynomial (products only) with its own (s, degree) plan.
  void set_approx(int a) {
    if (a == approx_) return;
    const int before = phase1_needs();
    approx_ = a;
    key2_.clear();
    if (phase1_needs() != before) rerecord_phase1();
  }
  int approx() const { return approx_; }
  int form() const { return form_; }
  // Diagnostics: the unitarity residual ||U_k^H U_k - I||_F / sqrt(n) of the iterate after every
  // squaring k = 0..s (k = 0: the Pade result), from two extra 5-slice products per squaring.
  void set_drift(bool d) {
    if (d == drift_) return;
    drift_ = d;
    key2_.clear();
  }
  // Residuals of walk w in the last run with drift on (s + 1 values; empty otherwise).
  std::vector<double> drift_curve(int w) const {
    std::vector<double> out;
    if (!drift_ || drift_host_.empty()) return out;
    const int cnt = std::min(sel_s_[w], kDriftMax - 1) + 1;
    for (int k = 0; k < cnt; ++k)
      out.push_back(std::sqrt(std::max(0.0, drift_host_[(size_t)w * kDriftMax + k])) / std::sqrt((double)walks_[w].n));
    return out;
  }
  void details(int w, double* feat, int* pm, int* ps, int* cm, int* cs, int* outcome) const {
    for (int k = 0; k < 8; ++k) feat[k] = features_.empty() ? 0.0 : features_[8 * w + k];
    *pm = plain_m_.empty() ? 0 : plain_m_[w];
    *ps = plain_s_.empty() ? 0 : plain_s_[w];
    *cm = cert_m_.empty() ? 0 : cert_m_[w];
    *cs = cert_s_.empty() ? 0 : cert_s_[w];
    *outcome = outcome_.empty() ? 0 : outcome_[w];
  }
  // Per walk: ||Y||_1, d4, d6, d8, d10 and the shift flags of the last run.
  void walk_stats(int w, fx_stats* st) const {
    st->m = sel_m_[w];
    st->s = sel_s_[w];
    st->structured = 1;
    st->rank1_shift = rank1_[w];
    st->symmetric = 1;
    st->solver = cheb_deg_[w] >= 0 ? 3 : uses_newton(w) ? 2 : 1;
    st->degree = cheb_deg_[w] >= 0 ? cheb_deg_[w] : 0;
    st->norm1 = norms_[8 * w];
    st->d[0] = std::pow(norms_[8 * w + 1], 0.25);
    st->d[1] = std::pow(norms_[8 * w + 2], 1.0 / 6);
    st->d[2] = std::pow(norms_[8 * w + 3], 0.125);
    st->d[3] = std::pow(norms_[8 * w + 4], 0.1);
    st->d[4] = -1.0;
    st->prod_ms = prod_ms_;
    st->prod_ops = prod_ops_;
    st->prod_flops = prod_flops_;
    st->prod_launches = prod_launches_;
  }
  int gemm_launches() const { return gemm_launches_; }
  // Skip-tile argument of the next product launch (the injected stall hits tile 0 of launch k).
  int next_skip() { return (inject_ >= 0 && prod_index_++ == inject_) ? 0 : -1; }

  // psi_w = expm(X_w) psi0_w and/or U_w = expm(X_w); any of dpsi0 / dpsi / dU may be null (a
  // null table, or a null entry, skips that output for that walk).
  void run(const void* const* dX, const void* const* dpsi0, void* const* dpsi, void* const* dU, cudaStream_t s) {
    const int W = count();
    stream_ = s;
    launches_ = 0;
    gemm_launches_ = 0;
    prod_index_ = 0;
    prof_reset();
    phase_mark(0);
    std::vector<const void*> tab(4 * W, nullptr);
    for (int w = 0; w < W; ++w) {
      tab[w] = dX[w];
      tab[W + w] = dpsi0 ? dpsi0[w] : nullptr;
      tab[2 * W + w] = dpsi ? dpsi[w] : nullptr;
      tab[3 * W + w] = dU ? dU[w] : nullptr;
    }
    FX_CUDA(cudaMemcpyAsync(ptrs_.p, tab.data(), sizeof(void*) * 4 * W, cudaMemcpyHostToDevice, s));
    FX_CUDA(cudaMemsetAsync(err_.p, 0, sizeof(int) * 8, s));
    FX_CUDA(cudaMemsetAsync(flags(), 0, sizeof(int) * W, s));

    // ---- phase 1: statistics and shifts, powers, exact norms, estimates (one host round trip)
    run_recorded(desc1_, st1_, r1_, graph1_, use_graph_ && !profile_ && inject_ < 0);
    phase_mark(1);
    std::vector<double>& h_wo = walkrec_;
    h_wo.assign(kWO * W, 0.0);
    std::vector<int> h_flags(W);
    FX_CUDA(cudaMemcpyAsync(h_wo.data(), walkout(), sizeof(double) * kWO * W, cudaMemcpyDeviceToHost, s));
    FX_CUDA(cudaMemcpyAsync(h_flags.data(), flags(), sizeof(int) * W, cudaMemcpyDeviceToHost, s));
    FX_CUDA(cudaMemcpyAsync(norms_.data(), norms(), sizeof(double) * 8 * W, cudaMemcpyDeviceToHost, s));
    lan_host_.assign((size_t)W * 4 * kLanSteps, 0.0);
    const bool lan = lan_recorded_;
    if (lan)
      FX_CUDA(cudaMemcpyAsync(lan_host_.data(), lanc_.p, sizeof(double) * lan_host_.size(), cudaMemcpyDeviceToHost, s));
    FX_CUDA(cudaStreamSynchronize(s));
    check_err();
    rho_lan_.assign(W, 0.0);
    rho_up_.assign(W, 0.0);
    for (int w = 0; w < W && lan; ++w) {
      const double* base = lan_host_.data() + (size_t)w * 4 * kLanSteps;
      rho_lan_[w] = std::max(tridiag_radius(base, kLanSteps), tridiag_radius(base + 2 * kLanSteps, kLanSteps));
    }
    for (int w = 0; w < W && !p46_recorded_; ++w) {   // bounds in place of ||A^4||, ||A^6||
      double* nw = norms_.data() + 8 * w;
      nw[1] = nw[5] * nw[5];
      nw[2] = nw[5] * nw[5] * nw[5];
    }
    for (int w = 0; w < W && !est_recorded_; ++w) {   // bounds in place of the estimates
      double* nw = norms_.data() + 8 * w;
      nw[3] = nw[1] * nw[1];
      nw[4] = nw[1] * nw[2];
    }
    for (int w = 0; w < W; ++w) {
      if (h_flags[w] & 4) throw Error{FX_ERR_NONFINITE, "input " + std::to_string(w) + " contains NaN or Inf"};
      if (h_flags[w] & 3)
        throw Error{FX_ERR_VALUE, "batched walks need generators X = i*(real symmetric); input " +
                                      std::to_string(w) + " is not"};
      mu_[w] = std::complex<double>(h_wo[kWO * w], h_wo[kWO * w + 1]);
      nu_[w] = std::complex<double>(h_wo[kWO * w + 2], h_wo[kWO * w + 3]);
      rank1_[w] = h_wo[kWO * w + 4] != 0.0;
    }

    // ---- selection (m, s) per walk: Al-Mohy & Higham (2009) Alg. 6.1, normal input (l = 0),
    // then optionally the certified or the learned selection (both gated by the certified
    // truncation bound; the plain choice is the fallback).
    flops_ = 0;
    plain_m_.assign(W, 13);
    plain_s_.assign(W, 0);
    cert_m_.assign(W, 13);
    cert_s_.assign(W, 0);
    outcome_.assign(W, 0);
    features_.assign(8 * W, 0.0);
    for (int w = 0; w < W; ++w) {
      const double* nw = norms_.data() + 8 * w;
      const double anorm = nw[0], d4 = std::pow(nw[1], 0.25), d6 = std::pow(nw[2], 1.0 / 6);
      if (!std::isfinite(anorm) || !std::isfinite(d4) || !std::isfinite(d6))
        throw Error{FX_ERR_NONFINITE, "non-finite norm in walk " + std::to_string(w)};
      int m = 13, sq = 0;
      if (std::max(d4, d6) < kTheta3) {
        m = 3;
      } else if (std::max(d4, d6) < kTheta5) {
        m = 5;
      } else {
        const double d8 = std::pow(nw[3], 0.125);
        const double eta3 = std::max(d6, d8);
        if (eta3 < kTheta7) {
          m = 7;
        } else if (eta3 < kTheta9) {
          m = 9;
        } else {
          const double d10 = std::pow(nw[4], 0.1);
          const double eta5 = std::min(eta3, std::max(d8, d10));
          sq = eta5 == 0.0 ? 0 : std::max((int)std::ceil(std::log2(eta5 / kTheta13)), 0);
        }
      }
      if (m != 13) sq = 0;
      plain_m_[w] = m;
      plain_s_[w] = sq;
      const double rho_up = std::min(anorm, std::min(d4, d6));
      rho_up_[w] = rho_up;
      certified_choice(rho_up, kPhaseTol, &cert_m_[w], &cert_s_[w]);
      // features of the learned selection
      const double n = walks_[w].n;
      const double* rec = walkrec_.data() + kWO * w;
      double* f = features_.data() + 8 * w;
      f[0] = std::log2(n);
      f[1] = std::log2(anorm + 1e-300);
      f[2] = std::log2(std::sqrt(rec[8] / n) + 1e-300);
      f[3] = std::log2(1.0 + rec[9]);
      f[4] = std::log2(rho_lan_[w] + 1e-300);
      f[5] = rank1_[w] ? 1.0 : 0.0;
      f[6] = std::log2(d4 + 1e-300);
      f[7] = std::log2(d6 + 1e-300);
    }
    std::vector<float> prop;
    // the network proposes Pade (m, s): not needed when every walk takes the polynomial
    if (selector_ == 2 && needs_powers46()) prop = infer_proposals();
    for (int w = 0; w < W; ++w) {
      int m = plain_m_[w], sq = plain_s_[w];
      const double* nw = norms_.data() + 8 * w;
      const double rho_up = std::min(nw[0], std::min(std::pow(nw[1], 0.25), std::pow(nw[2], 1.0 / 6)));
      if (selector_ == 1 && pade_products(cert_m_[w]) + cert_s_[w] < pade_products(m) + sq) {
        m = cert_m_[w];
        sq = cert_s_[w];
        outcome_[w] = 1;
      } else if (selector_ == 3 || selector_ == 2) {
        // the phase bound at the Lanczos estimate of the spectral radius, with a margin (never
        // above the rigorous bound rho_up)
        const double rho_est = std::min(rho_up, rho_lan_[w] * (1.0 + kLanMargin));
        int em = 13, es = 0;
        certified_choice(rho_est, kPhaseTol, &em, &es);
        if (pade_products(em) + es < pade_products(m) + sq) {
          m = em;
          sq = es;
          outcome_[w] = 3;
        }
        if (selector_ == 2 && !prop.empty()) {
          // the learned proposal replaces the estimated choice when it is cheaper still and
          // passes the gate: the same phase bound at the phase error that keeps the
          // infidelity of every state below 1e-10
          const float* o = prop.data() + 6 * w;
          int c = 0;
          for (int k = 1; k < 5; ++k)
            if (o[k] > o[c]) c = k;
          const int pm = kDegrees[c];
          const int ps = std::max(0, (int)std::lround(o[5]));
          if (pade_products(pm) + ps < pade_products(m) + sq) {
            if (certified(pm, ps, rho_est, kGateTol)) {
              m = pm;
              sq = ps;
              outcome_[w] = 2;
            } else if (outcome_[w] != 3) {
              outcome_[w] = -1;   // rejected by the bound, and no estimated choice: plain (m, s)
            }
          }
        }
      }
      if (force_m_ > 0) m = force_m_;
      if (force_s_ >= 0 && m == 13) sq = force_s_;
      if (m != 13 && force_s_ < 0 && outcome_[w] <= 0) sq = 0;
      const bool pw = !pw_m_.empty() && pw_m_[w] > 0;
      if (pw) {   // per-walk forced (m, s): measured sweeps
        m = pw_m_[w];
        sq = std::max(0, pw_s_[w]);
        outcome_[w] = 4;
      }
      const double N3 = (double)walks_[w].n * walks_[w].n * walks_[w].n;
      cheb_deg_[w] = -1;
      if (approx_ == 1 && !pw && force_m_ <= 0 && force_s_ < 0) {
        // the polynomial on the rigorous bound, or (estimated and learned selections) on the
        // Lanczos estimate with its margin when that is smaller
        const double rho_c = selector_ >= 2 && rho_lan_[w] > 0.0
                                 ? std::min(rho_up, rho_lan_[w] * (1.0 + kChebLanMargin))
                                 : rho_up;
        const ChebPlan cp = cheb_plan(rho_c, dtype_ == FX_C128 ? kChebTolC128 : kPhaseTol);
        if (!cp.ok) throw Error{FX_ERR_VALUE, "walk " + std::to_string(w) + ": no Chebyshev plan for a spectral bound this large"};
        m = 0;
        sq = cp.s;
        cheb_deg_[w] = cp.degree;
        cheb_baby_[w] = cp.baby;
        cheb_rho_[w] = rho_c;
        outcome_[w] = 5;
        sel_m_[w] = m;
        sel_s_[w] = sq;
        // as for the Pade stage, every product counts as one generic complex GEMM
        flops_ += 8.0 * N3 * (cp.cost - kChebSquareProducts * cp.s + sq) + 8.0 * N3;
        continue;
      }
      sel_m_[w] = m;
      sel_s_[w] = sq;
      flops_ += 8.0 * N3 * (pade_products(m) + sq) + (8.0 / 3.0) * N3 + 8.0 * N3;
    }
    if (analyze_only_) return;

    // ---- phase 2, then the a-posteriori checks of the non-plain selections: a walk whose
    // Pade denominator fails to factor, or whose state loses its norm, is redone alone with the
    // plain (m, s) in a pipeline of its own (its outputs are overwritten; the other walks keep
    // theirs).  A failure under the plain choice is an error.
    if (autotune_) {
      autotune_phase2(tab);
      autotune_ = false;
    }
    FX_CUDA(cudaMemsetAsync(walk_err(), 0, sizeof(int) * W, s));
    phase_mark(2);
    run_phase2(tab);
    phase_mark(3);
    std::vector<int> werr(W), own(W, 0);
    int herr = 0;
    FX_CUDA(cudaMemcpyAsync(werr.data(), walk_err(), sizeof(int) * W, cudaMemcpyDeviceToHost, s));
    FX_CUDA(cudaMemcpyAsync(&herr, err_.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    FX_CUDA(cudaStreamSynchronize(s));
    // a wait that ran out leaves every later result meaningless: report it before anything else
    if (herr & kDevTimeout) throw Error{FX_ERR_TIMEOUT, "a device-side wait timed out"};
    bool any = false;
    for (int w = 0; w < W; ++w) {
      if (!werr[w]) continue;
      if (outcome_[w] <= 0) throw Error{FX_ERR_SINGULAR, "Pade denominator is not positive definite (walk " + std::to_string(w) + ")"};
      own[w] = 1;
      any = true;
    }
    any = verify_states(tab, own) || any;
    any = sample_compare(tab, own) || any;
    if (any) {
      if (herr & kDevTimeout) throw Error{FX_ERR_TIMEOUT, "a device-side wait timed out"};
      FX_CUDA(cudaMemsetAsync(err_.p, 0, sizeof(int) * 8, s));
      std::vector<int> redo;
      for (int w = 0; w < W; ++w)
        if (own[w]) redo.push_back(w);
      std::vector<int64_t> ns;
      std::vector<const void*> x, p0;
      std::vector<void*> p1, u;
      for (int w : redo) {
        ns.push_back(walks_[w].n);
        x.push_back(tab[w]);
        p0.push_back(tab[W + w]);
        p1.push_back((void*)tab[2 * W + w]);
        u.push_back((void*)tab[3 * W + w]);
      }
      BatchPipeline sub(ns, dtype_);
      sub.set_timeout(timeout_ms_);
      sub.run(x.data(), p0.data(), p1.data(), u.data(), s);
      launches_ += sub.launches();
      for (size_t i = 0; i < redo.size(); ++i) {
        const int w = redo[i];
        outcome_[w] = -2;
        sub.selection((int)i, &sel_m_[w], &sel_s_[w]);
      }
    }
    phase_mark(4);
    FX_CUDA(cudaStreamSynchronize(s));
    check_err();
    prof_collect();
    if (profile_) {   // the run's timeline (not part of the product totals)
      for (int k = 0; k < 4; ++k) {
        float t = 0;
        FX_CUDA(cudaEventElapsedTime(&t, phase_ev_[k], phase_ev_[k + 1]));
        prod_list_.push_back(ProdRecord{kTagPhase1 + k, (double)t, 0.0, 0.0});
      }
    }
    if (drift_ && drift_buf_.p) {
      drift_host_.assign((size_t)W * kDriftMax, 0.0);
      FX_CUDA(cudaMemcpy(drift_host_.data(), drift_buf_.p, sizeof(double) * drift_host_.size(), cudaMemcpyDeviceToHost));
    }
  }

  // Phase 2: Pade, solve, squarings, outputs.  The recorded launch sequence (and its CUDA graph)
  // depends only on the sizes, (m, s), the shifts and which outputs are wanted; it is rebuilt
  // only when one of those changed since the last run.
  void run_phase2(const std::vector<const void*>& tab) {
    const int W = count();
    std::vector<double> key;
    for (int w = 0; w < W; ++w) {
      key.insert(key.end(), {(double)sel_m_[w], (double)sel_s_[w], (double)rank1_[w], mu_[w].real(),
                             mu_[w].imag(), nu_[w].real(), nu_[w].imag(), tab[W + w] ? 1.0 : 0.0,
                             tab[2 * W + w] ? 1.0 : 0.0, tab[3 * W + w] ? 1.0 : 0.0});
      // the Newton-Schulz solve takes its step count and scaling from these
      key.insert(key.end(), {rho_up_[w], rho_lan_[w], (double)cheb_deg_[w], cheb_rho_[w]});
    }
    if (key != key2_ || profile_) {
      st2_ = Staging();
      r2_ = Rec();
      if (graph2_) {
        cudaGraphExecDestroy(graph2_);
        graph2_ = nullptr;
      }
      record_rest(st2_, r2_);
      desc2_.alloc(std::max<size_t>(st2_.buf.size(), 256));
      FX_CUDA(cudaMemcpyAsync(desc2_.p, st2_.buf.data(), st2_.buf.size(), cudaMemcpyHostToDevice, stream_));
      key2_ = profile_ ? std::vector<double>() : key;
    }
    run_recorded(desc2_, st2_, r2_, graph2_, use_graph_ && !profile_ && inject_ < 0, false);
  }

  // A-posteriori unitarity check of the walks that did not take the plain (m, s): ||psi|| must
  // equal ||psi0|| to 1e-3 (U is unitary in exact arithmetic whatever (m, s)).  The bound is
  // loose on purpose: it catches arithmetic breakdowns of a proposal, not the norm drift that
  // the plain choice shares (up to ~2e-4 after 13 squarings for walks dominated by one
  // eigenvalue, where the int8 slices hold that mode's off-diagonal entries to ~1e-8).  Returns
  // true when a walk failed.
  // Sampled comparison with the plain method: up to sample_walks_ of the walks that ran a
  // non-plain (m, s) (the smallest, so that the check stays cheap; ties to the lower index) are
  // run again with the plain (m, s) in a side pipeline, and the two states compared.  An
  // infidelity above kSampleInfid marks every non-plain walk of the batch for the plain redo.
  // Walks are dropped from the sample (largest first) while it costs more than a tenth of the
  // batch by N^3, but one walk is always sampled; only a batch of one walk (a single structured
  // walk, which would be computed twice) skips the comparison (sample_count_ = -1).
  bool sample_compare(const std::vector<const void*>& tab, std::vector<int>& own) {
    constexpr double kSampleInfid = 1e-10;
    const int W = count();
    sample_count_ = 0;
    sample_max_infid_ = 0.0;
    std::vector<int> cand;
    for (int w = 0; w < W; ++w)
      if (outcome_[w] > 0 && !own[w] && tab[W + w] && tab[2 * W + w] &&
          (sel_m_[w] != plain_m_[w] || sel_s_[w] != plain_s_[w]))
        cand.push_back(w);
    if (cand.empty() || sample_walks_ <= 0) return false;
    if (W == 1) {
      sample_count_ = -1;
      return false;
    }
    std::stable_sort(cand.begin(), cand.end(), [&](int a, int b) { return walks_[a].n < walks_[b].n; });
    if ((int)cand.size() > sample_walks_) cand.resize(sample_walks_);
    double all_n3 = 0.0, cand_n3 = 0.0;
    for (int w = 0; w < W; ++w) all_n3 += std::pow((double)walks_[w].n, 3);
    for (int w : cand) cand_n3 += std::pow((double)walks_[w].n, 3);
    while (cand.size() > 1 && cand_n3 > 0.1 * all_n3) {
      cand_n3 -= std::pow((double)walks_[cand.back()].n, 3);
      cand.pop_back();
    }
    std::vector<int64_t> ns;
    for (int w : cand) ns.push_back(walks_[w].n);
    if (!sample_pipe_ || ns != sample_ns_) {
      sample_pipe_.reset(new BatchPipeline(ns, dtype_));
      sample_ns_ = ns;
    }
    sample_pipe_->set_timeout(timeout_ms_);
    const size_t elem = dtype_ == FX_C64 ? 8 : 16;
    size_t total = 0;
    for (int64_t n : ns) total += (size_t)n * elem;
    if (sample_io_.bytes < total) sample_io_.alloc(total);
    std::vector<const void*> x, p0;
    std::vector<void*> p1, u(cand.size(), nullptr);
    size_t off = 0;
    for (int w : cand) {
      x.push_back(tab[w]);
      p0.push_back(tab[W + w]);
      p1.push_back((unsigned char*)sample_io_.p + off);
      off += (size_t)walks_[w].n * elem;
    }
    sample_pipe_->run(x.data(), p0.data(), p1.data(), u.data(), stream_);
    launches_ += sample_pipe_->launches();
    // both states to the host, compared in FP64
    std::vector<unsigned char> a(total), b(total);
    off = 0;
    for (size_t i = 0; i < cand.size(); ++i) {
      const size_t bytes = (size_t)walks_[cand[i]].n * elem;
      FX_CUDA(cudaMemcpyAsync(a.data() + off, tab[2 * W + cand[i]], bytes, cudaMemcpyDeviceToHost, stream_));
      FX_CUDA(cudaMemcpyAsync(b.data() + off, p1[i], bytes, cudaMemcpyDeviceToHost, stream_));
      off += bytes;
    }
    FX_CUDA(cudaStreamSynchronize(stream_));
    off = 0;
    for (size_t i = 0; i < cand.size(); ++i) {
      const int64_t n = walks_[cand[i]].n;
      std::complex<double> ov(0.0, 0.0);
      double na = 0.0, nb = 0.0;
      for (int64_t k = 0; k < n; ++k) {
        std::complex<double> va, vb;
        if (dtype_ == FX_C64) {
          const float* fa = (const float*)(a.data() + off);
          const float* fb = (const float*)(b.data() + off);
          va = {fa[2 * k], fa[2 * k + 1]};
          vb = {fb[2 * k], fb[2 * k + 1]};
        } else {
          const double* da = (const double*)(a.data() + off);
          const double* db = (const double*)(b.data() + off);
          va = {da[2 * k], da[2 * k + 1]};
          vb = {db[2 * k], db[2 * k + 1]};
        }
        ov += std::conj(vb) * va;
        na += std::norm(va);
        nb += std::norm(vb);
      }
      const double inf = (na > 0 && nb > 0) ? 1.0 - std::norm(ov) / (na * nb) : 1.0;
      sample_max_infid_ = std::max(sample_max_infid_, inf);
      off += (size_t)n * elem;
    }
    sample_count_ = (int)cand.size();
    if (!(sample_max_infid_ <= kSampleInfid)) {
      for (int w = 0; w < W; ++w)
        if (outcome_[w] > 0) own[w] = 1;
      return true;
    }
    return false;
  }
  void set_sample_walks(int k) { sample_walks_ = k; }
  void sample_check(int* count, double* max_infid) const {
    *count = sample_count_;
    *max_infid = sample_max_infid_;
  }

  bool verify_states(const std::vector<const void*>& tab, std::vector<int>& own) {
    const int W = count();
    std::vector<int> list;
    for (int w = 0; w < W; ++w)
      if (outcome_[w] > 0 && tab[W + w] && tab[2 * W + w]) list.push_back(w);
    if (list.empty()) return false;
    const size_t need = sizeof(double) * 2 * W + sizeof(int) * list.size() + 64;
    if (ver_io_.bytes < need) ver_io_.alloc(need);
    double* nrm = (double*)ver_io_.p;
    int* dl = (int*)(nrm + 2 * W);
    FX_CUDA(cudaMemcpyAsync(dl, list.data(), sizeof(int) * list.size(), cudaMemcpyHostToDevice, stream_));
    if (dtype_ == FX_C64)
      kb_psi_norms<float2><<<(unsigned)list.size(), 256, 0, stream_>>>(dP0(), dP1(), dl, (const BWalk*)d_walks_.p, nrm);
    else
      kb_psi_norms<double2><<<(unsigned)list.size(), 256, 0, stream_>>>(dP0(), dP1(), dl, (const BWalk*)d_walks_.p, nrm);
    FX_LAUNCH_CHECK();
    ++launches_;
    std::vector<double> h(2 * W);
    FX_CUDA(cudaMemcpyAsync(h.data(), nrm, sizeof(double) * 2 * W, cudaMemcpyDeviceToHost, stream_));
    FX_CUDA(cudaStreamSynchronize(stream_));
    bool bad = false;
    for (int w : list) {
      const double a = std::sqrt(h[2 * w]), b = std::sqrt(h[2 * w + 1]);
      if (!(std::fabs(b - a) <= 1e-3 * a)) own[w] = 1, bad = true;
    }
    return bad;
  }

 private:
  // kX1, kX2: the Chebyshev stage's baby steps T_4, T_5 of C, allocated at the first plan that
  // needs them; the others from the start
  enum { kY, kA2, kA4, kA6, kT1, kT2, kW, kV, kX1, kX2, kArenas };
  static constexpr int kBaseArenas = kX1;
  struct Rec {
    std::vector<std::function<void()>> ops;
    int launches = 0, gemms = 0;
  };

  int dtype_;
  std::vector<BWalk> walks_;
  int64_t elems_ = 0, rows_ = 0, maxnp_ = 0, pitch_ = 0, a_rows_ = 0;
  DevArena arena_[kArenas];
  DevArena slices_, exps_, diag_, linv_, small_, err_, d_walks_, ptrs_, desc1_, desc2_;
  Staging st1_, st2_;
  Rec r1_, r2_;
  std::vector<double> key2_;
  std::vector<int> sel_m_, sel_s_, rank1_;
  std::vector<std::complex<double>> mu_, nu_;
  std::vector<double> norms_;
  std::vector<double> walkrec_;
  std::vector<int> plain_m_, plain_s_, cert_m_, cert_s_, outcome_;
  std::vector<double> features_;
  int selector_ = 0;
  std::vector<cudaEvent_t> phase_ev_;   // profile mode: the run's timeline events
  bool lan_recorded_ = false;   // phase 1 as recorded runs the Lanczos estimate
  bool est_recorded_ = true;    // phase 1 as recorded runs the 1-norm estimates of A^8, A^10
  bool p46_recorded_ = true;    // phase 1 as recorded computes A^4 and A^6
  bool analyze_only_ = false;
  int split_ = 7;
  int tile_group_ = 8, tile_order_ = 0;   // phase-2 schedule of the grouped products
  int sample_walks_ = 2, sample_count_ = 0;   // sampled comparison with the plain method
  double sample_max_infid_ = 0.0;
  std::unique_ptr<BatchPipeline> sample_pipe_;
  std::vector<int64_t> sample_ns_;
  DevArena sample_io_;
  bool autotune_ = false;
  std::vector<std::array<double, 3>> tuned_;   // (group, order, ms) of the last tuning
  DevArena sel_io_, ver_io_;
  cudaStream_t stream_ = nullptr;
  unsigned timeout_ms_ = 2000;
  bool use_graph_ = true, profile_ = false;
  int force_m_ = -1, force_s_ = -1;
  std::vector<int> pw_m_, pw_s_;   // per-walk forced (m, s) (diagnostics and measured sweeps)
  int inject_ = -1, prod_index_ = 0;   // stall injection (diagnostics), product launches so far
  int form_ = 0, sq_n4_ = 0, sq_n3_ = 0;   // squaring form and slice schedule
  int pade_S_ = kS;                        // mixed form: slices of the Pade and solve products
  int newton_S_ = kS;                      // mixed form: slices of the early Newton-Schulz steps
  int solve_mode_ = 0;                     // 0 by form and size, 1 Cholesky, 2 Newton-Schulz
  int approx_ = 0;                         // 0 Pade, 1 Chebyshev-Bessel polynomial
  bool nvtx_open_ = false;                 // a phase's NVTX range is open
  std::vector<int> cheb_deg_, cheb_baby_;  // per walk: the polynomial's degree (-1: Pade), m
  std::vector<double> cheb_rho_;           // per walk: the spectral bound of the polynomial
  int gS_ = kS;                            // slices of the grouped products being recorded
  DevArena lanc_;                          // Lanczos coefficients (W x 2 runs x kLanSteps x 2)
  std::vector<double> lan_host_, rho_lan_, rho_up_;
  bool drift_ = false;                     // per-squaring unitarity residual (diagnostics)
  DevArena drift_buf_;
  std::vector<double> drift_host_;
  int launches_ = 0, gemm_launches_ = 0;
  double flops_ = 0;
  cudaGraphExec_t graph1_ = nullptr, graph2_ = nullptr;
  unsigned char* desc_base_ = nullptr;
  // product-launch timing (profile mode)
  std::vector<cudaEvent_t> ev_pool_;
  struct ProdWork {
    double ops, flops;
    int tag;
  };
  std::vector<ProdWork> ev_work_;
  double prod_ms_ = 0, prod_ops_ = 0, prod_flops_ = 0;
  int prod_launches_ = 0;
  int tag_ = kTagPowers;                  // stage of the products being recorded
  std::vector<ProdRecord> prod_list_;    // per product launch of the last profiled run

 public:
  const std::vector<ProdRecord>& prod_list() const { return prod_list_; }

 private:

 public:
  void force(int m, int s) {
    const int before = phase1_needs();
    force_m_ = m;
    force_s_ = s;
    if (phase1_needs() != before) rerecord_phase1();
  }
  // Per-walk (m, s) for the next runs (m <= 0: that walk's own selection); empty clears.
  void force_each(const int* m, const int* s) {
    const int W = count();
    const int before = phase1_needs();
    if (!m) {
      pw_m_.clear();
      pw_s_.clear();
    } else {
      pw_m_.assign(m, m + W);
      pw_s_.assign(s, s + W);
    }
    if (phase1_needs() != before) rerecord_phase1();
  }

 private:
  double* A(int a) const { return (double*)arena_[a].p; }
  // layout of small_
  double* rowstat() const { return (double*)small_.p; }
  double* est_scr() const { return rowstat() + kRS * rows_; }
  double* rsum() const { return est_scr() + kEstScratch * rows_; }
  double* rsum2() const { return rsum() + rows_; }   // the imaginary plane's row sums
  double* walkout() const { return rsum2() + rows_; }
  double* norms() const { return walkout() + kWO * count(); }
  double* estst() const { return norms() + 8 * count(); }
  double* misc() const { return estst() + 4 * count(); }   // 8 per walk: psum, projection totals
  int* flags() const { return (int*)(misc() + 8 * count()); }
  int* walk_err() const { return flags() + count(); }   // per walk: Cholesky of G failed
  const void* const* dX() const { return (const void* const*)ptrs_.p; }
  const void* const* dP0() const { return dX() + count(); }
  void* const* dP1() const { return (void* const*)(dX() + 2 * count()); }
  void* const* dUo() const { return (void* const*)(dX() + 3 * count()); }

  int8_t* slice_plane(int which, int q) const {
    // which: 0 A re (a_rows_), 1 A im, 2 A -im, 3 B re (rows_ each)
    const size_t plane_a = (size_t)pitch_ * a_rows_, plane_r = (size_t)pitch_ * rows_;
    int8_t* base = (int8_t*)slices_.p;
    if (which == 0) return base + q * plane_a;
    return base + kS * plane_a + (size_t)((which - 1) * kS + q) * plane_r;
  }
  int* aexp() const { return (int*)exps_.p; }
  int* bexp() const { return (int*)exps_.p + a_rows_ + 32; }
  double* adiag() const { return (double*)diag_.p; }
  double* bdiag() const { return (double*)diag_.p + a_rows_ + 32; }
  double* linv(int w) const { return (double*)linv_.p + (size_t)walks_[w].row0 * kNb; }
  double* linvT(int w) const { return (double*)linv_.p + (size_t)rows_ * kNb + (size_t)walks_[w].row0 * kNb; }
  template <typename T>
  T* dev(size_t off) const {
    return (T*)(desc_base_ + off);
  }

  void check_err() {
    int h = 0;
    FX_CUDA(cudaMemcpy(&h, err_.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (h & kDevTimeout) throw Error{FX_ERR_TIMEOUT, "a device-side wait timed out"};
    if (h & kDevSingular) throw Error{FX_ERR_SINGULAR, "Pade denominator is not positive definite"};
  }

  // MLP proposals for every walk (6 floats each: 5 logits, s), from the process-wide weights.
  std::vector<float> infer_proposals() {
    const int W = count();
    float* wts = nullptr;
    {
      std::lock_guard<std::mutex> lk(g_sel_mu);
      int dev = -1;
      FX_CUDA(cudaGetDevice(&dev));
      if (!g_sel_weights || g_sel_device != dev)
        throw Error{FX_ERR_VALUE, "learned selection needs weights on this device (fx_selector_set_weights)"};
      wts = g_sel_weights;
    }
    if (sel_io_.bytes < sizeof(float) * 14 * (size_t)W) sel_io_.alloc(sizeof(float) * 14 * (size_t)W);
    std::vector<float> fx(8 * W), out(6 * W);
    for (int i = 0; i < 8 * W; ++i) fx[i] = (float)features_[i];
    float* dfx = (float*)sel_io_.p;
    float* dout = dfx + 8 * W;
    FX_CUDA(cudaMemcpyAsync(dfx, fx.data(), sizeof(float) * 8 * W, cudaMemcpyHostToDevice, stream_));
    launch_mlp_infer(wts, dfx, W, dout, stream_);
    ++launches_;
    FX_CUDA(cudaMemcpyAsync(out.data(), dout, sizeof(float) * 6 * W, cudaMemcpyDeviceToHost, stream_));
    FX_CUDA(cudaStreamSynchronize(stream_));
    return out;
  }

  // Profile mode: event k of the run's timeline (0 start, 1 after phase 1, 2 before phase 2,
  // 3 after phase 2, 4 end).
  // Phase boundaries of a run: an NVTX range per phase (phase 1, selection and recording,
  // phase 2, the a-posteriori checks) and, in profile mode, a CUDA event at each boundary.
  void phase_mark(int k) {
    static const char* kNames[4] = {"fx batch: phase 1 (statistics, powers, norms, Lanczos)",
                                    "fx batch: selection and phase-2 recording",
                                    "fx batch: phase 2 (approximant, squarings, outputs)",
                                    "fx batch: a-posteriori checks"};
    if (nvtx_open_) nvtxRangePop();
    nvtx_open_ = k < 4;
    if (nvtx_open_) nvtxRangePushA(kNames[k]);
    if (!profile_) return;
    while ((int)phase_ev_.size() < 5) {
      cudaEvent_t e;
      FX_CUDA(cudaEventCreate(&e));
      phase_ev_.push_back(e);
    }
    FX_CUDA(cudaEventRecord(phase_ev_[k], stream_));
  }
  void prof_reset() {
    ev_work_.clear();
    prod_list_.clear();
    prod_ms_ = prod_ops_ = prod_flops_ = 0;
    prod_launches_ = 0;
  }
  // Events around a product launch (profile mode, eager replay only).
  size_t prof_begin() {
    if (!profile_) return 0;
    const size_t i = ev_work_.size();
    while (ev_pool_.size() < 2 * (i + 1)) {
      cudaEvent_t e;
      FX_CUDA(cudaEventCreate(&e));
      ev_pool_.push_back(e);
    }
    FX_CUDA(cudaEventRecord(ev_pool_[2 * i], stream_));
    return i;
  }
  void prof_end(size_t i, double ops, double fl, int tag) {
    if (!profile_) return;
    FX_CUDA(cudaEventRecord(ev_pool_[2 * i + 1], stream_));
    ev_work_.push_back({ops, fl, tag});
  }
  void prof_collect() {
    if (!profile_) return;
    for (size_t i = 0; i < ev_work_.size(); ++i) {
      float t = 0;
      FX_CUDA(cudaEventElapsedTime(&t, ev_pool_[2 * i], ev_pool_[2 * i + 1]));
      prod_ms_ += t;
      prod_ops_ += ev_work_[i].ops;
      prod_flops_ += ev_work_[i].flops;
      prod_list_.push_back(ProdRecord{ev_work_[i].tag, (double)t, ev_work_[i].ops, ev_work_[i].flops});
    }
    prod_launches_ = (int)ev_work_.size();
  }

  // Replay a recorded launch sequence: eagerly, or through its (cached) CUDA graph.
  void run_recorded(DevArena& desc, Staging& st, Rec& r, cudaGraphExec_t& gexec, bool graph, bool upload = true) {
    if (upload && desc.bytes == 0) {
      desc.alloc(std::max<size_t>(st.buf.size(), 256));
      FX_CUDA(cudaMemcpy(desc.p, st.buf.data(), st.buf.size(), cudaMemcpyHostToDevice));
    }
    desc_base_ = (unsigned char*)desc.p;
    launches_ += r.launches;
    gemm_launches_ += r.gemms;
    if (!graph) {
      for (auto& op : r.ops) op();
      return;
    }
    if (!gexec) {
      warm_attributes();
      cudaGraph_t g = nullptr;
      FX_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
      try {
        for (auto& op : r.ops) op();
      } catch (...) {
        cudaStreamEndCapture(stream_, &g);
        if (g) cudaGraphDestroy(g);
        throw;
      }
      FX_CUDA(cudaStreamEndCapture(stream_, &g));
      const cudaError_t e = cudaGraphInstantiate(&gexec, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) {
        gexec = nullptr;
        throw Error{FX_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e)};
      }
    }
    FX_CUDA(cudaGraphLaunch(gexec, stream_));
  }
  // Kernel attributes (dynamic shared memory) are set outside any stream capture.
  void warm_attributes() {
    prepare_gemm_i8_grouped(3);
    prepare_gemm_i8_grouped(4);
    prepare_gemm_i8_grouped(kS);
    prepare_potrf_inv_grouped();
  }

  // Phase 1, recorded once: statistics and shifts, Y, A2 = Y^2, A4, A6, exact norms of Y, A4,
  // A6 and the estimates of ||A4 A4||_1 and ||A4 A6||_1.
  void record_phase1() {
    const int W = count();
    Staging& st = st1_;
    Rec& r = r1_;
    std::vector<int> all(W);
    for (int w = 0; w < W; ++w) all[w] = w;
    const size_t o_all = st.put(all);
    const dim3 g_rows(grid_x_for(maxnp_ * 32, W), W), g_el(grid_x_for(maxnp_ * maxnp_, W), W);
    const int dt = dtype_;
    const bool lan = needs_lanczos();
    r.ops.push_back([=]() {
      const BWalk* wk = (const BWalk*)d_walks_.p;
      if (dt == FX_C64)
        kb_stats<float2><<<g_rows, 256, 0, stream_>>>(dX(), dev<int>(o_all), wk, rowstat(), flags());
      else
        kb_stats<double2><<<g_rows, 256, 0, stream_>>>(dX(), dev<int>(o_all), wk, rowstat(), flags());
      FX_LAUNCH_CHECK();
      kb_walk_reduce<<<W, 256, 0, stream_>>>(dev<int>(o_all), wk, rowstat(), walkout());
      FX_LAUNCH_CHECK();
      // with the Lanczos estimate recorded, an FP32 copy of Y for its mat-vecs (arena T1, free
      // until phase 2)
      float* y32 = lan ? (float*)A(kT1) : nullptr;
      if (dt == FX_C64)
        kb_load_imag<float2><<<g_el, 256, 0, stream_>>>(dX(), dev<int>(o_all), wk, walkout(), A(kY), y32);
      else
        kb_load_imag<double2><<<g_el, 256, 0, stream_>>>(dX(), dev<int>(o_all), wk, walkout(), A(kY), y32);
      FX_LAUNCH_CHECK();
    });
    r.launches += 3;
    tag_ = kTagPowers;
    // the mixed form's slice count, with the diagonals split off (the shifted generator's rows
    // are dominated by their diagonal, and its powers' even more)
    const bool psplit = form_ == 1 || (split_ & 4);
    p46_recorded_ = needs_powers46();
    const bool p46 = p46_recorded_;
    by_slices(all, [&](int w) { return reduced(w) ? pade_S_ : kS; }, [&](const std::vector<int>& l) {
      product(st, r, l, kY, kY, -1.0, -1, 0.0, 0.0, kA2, true, nullptr, nullptr, psplit);
      if (!p46) return;
      product(st, r, l, kA2, kA2, 1.0, -1, 0.0, 0.0, kA4, true, nullptr, nullptr, psplit);
      product(st, r, l, kA4, kA2, 1.0, -1, 0.0, 0.0, kA6, true, nullptr, nullptr, psplit);
    });
    // exact 1-norms of Y, A4, A6 into norms slots 0, 1, 2 (or of Y and A2 into slots 0 and 5)
    const int arenas[3] = {kY, p46 ? kA4 : kA2, kA6}, slots[3] = {0, p46 ? 1 : 5, 2};
    const int nnorm = p46 ? 3 : 2;
    r.ops.push_back([=]() {
      const BWalk* wk = (const BWalk*)d_walks_.p;
      for (int k = 0; k < nnorm; ++k) {
        kb_abs_rowsums<<<g_rows, 256, 0, stream_>>>(A(arenas[k]), dev<int>(o_all), wk, rsum());
        FX_LAUNCH_CHECK();
        kb_walk_vec_reduce<<<W, 256, 0, stream_>>>(rsum(), dev<int>(o_all), wk, 1, 0, norms(), 8, slots[k]);
        FX_LAUNCH_CHECK();
      }
    });
    r.launches += 2 * nnorm;
    est_recorded_ = needs_estimates();
    if (est_recorded_) {
      estimate(st, r, all, kA4, kA4, 3);
      estimate(st, r, all, kA4, kA6, 4);
    }
    lan_recorded_ = needs_lanczos();
    if (lan_recorded_) lanczos(st, r, all);
  }

  // Lanczos runs on B = Im Y (arena Y) of the listed walks into lanc_ (kLanSteps steps).
  void lanczos(Staging& st, Rec& r, const std::vector<int>& list) {
    const size_t o_l = st.put(list);
    const int nl = (int)list.size();
    std::vector<RChunk> ch;
    for (int w : list) {
      const int np = walks_[w].np, R = std::max(8, (kChunkElems / np) & ~7);
      for (int r0 = 0; r0 < np; r0 += R) ch.push_back(RChunk{w, r0, std::min(np, r0 + R), 0});
    }
    const size_t o_ch = st.put(ch);
    const unsigned g_rows = (unsigned)ch.size();
    r.ops.push_back([=]() {
      const BWalk* wk = (const BWalk*)d_walks_.p;
      const int* l = dev<int>(o_l);
      kb_lan_init<<<nl, 256, 0, stream_>>>(l, wk, est_scr(), estst());
      FX_LAUNCH_CHECK();
      for (int j = 0; j < kLanSteps; ++j) {
        kb_est_matvec32<<<g_rows, 256, 0, stream_>>>((const float*)A(kT1), dev<RChunk>(o_ch), wk, est_scr(),
                                                    estst(), kEX0, kET0);
        kb_lan_step<<<2 * nl, 1024, 0, stream_>>>(l, wk, est_scr(), (double*)lanc_.p, j);
      }
      FX_LAUNCH_CHECK();
    });
    r.launches += 1 + 2 * kLanSteps;
  }

  // Block 1-norm estimate of ||M0 M1||_1 for the listed walks into norms()[8 w + slot].
  void estimate(Staging& st, Rec& r, const std::vector<int>& list, int m0, int m1, int slot) {
    const size_t o_l = st.put(list);
    const int nl = (int)list.size();
    std::vector<RChunk> ch;   // rows per chunk: a multiple of the 8 warps of a CTA
    for (int w : list) {
      const int np = walks_[w].np, R = std::max(8, (kChunkElems / np) & ~7);
      for (int r0 = 0; r0 < np; r0 += R) ch.push_back(RChunk{w, r0, std::min(np, r0 + R), 0});
    }
    const size_t o_ch = st.put(ch);
    const unsigned g_rows = (unsigned)ch.size();
    r.ops.push_back([=]() {
      const BWalk* wk = (const BWalk*)d_walks_.p;
      const int* l = dev<int>(o_l);
      kb_est_init<<<nl, 256, 0, stream_>>>(l, wk, est_scr(), estst());
      FX_LAUNCH_CHECK();
      for (int k = 1; k <= 5; ++k) {
        kb_est_matvec<<<g_rows, 256, 0, stream_>>>(A(m1), dev<RChunk>(o_ch), wk, est_scr(), estst(), kEX0, kET0);
        kb_est_matvec<<<g_rows, 256, 0, stream_>>>(A(m0), dev<RChunk>(o_ch), wk, est_scr(), estst(), kET0, kEY0);
        kb_est_step1<<<nl, 256, 0, stream_>>>(l, wk, est_scr(), estst(), k);
        FX_LAUNCH_CHECK();
        if (k == 5) break;
        kb_est_matvec<<<g_rows, 256, 0, stream_>>>(A(m0), dev<RChunk>(o_ch), wk, est_scr(), estst(), kEX0, kET0);
        kb_est_matvec<<<g_rows, 256, 0, stream_>>>(A(m1), dev<RChunk>(o_ch), wk, est_scr(), estst(), kET0, kEY0);
        kb_est_step2<<<nl, 256, 0, stream_>>>(l, wk, est_scr(), estst(), k);
        FX_LAUNCH_CHECK();
      }
      kb_est_final<<<(nl + 255) / 256, 256, 0, stream_>>>(l, nl, estst(), norms(), 8, slot);
      FX_LAUNCH_CHECK();
    });
    r.launches += 1 + 5 * 3 + 4 * 3 + 1;
  }

  // ---- recorded grouped operations --------------------------------------------------
  // Tile order of one problem: G x G blocks of tiles (G = tile_group_, 8 unless tuned),
  // row-major inside a block and over the blocks.  The ~148 tiles in flight then cover a few
  // blocks, so every A row panel and Bt column panel of a K step is fetched from HBM once and
  // served to up to G CTAs from L2 (a row-major order would stream a distinct Bt panel for every
  // CTA).
  template <typename F>
  void for_tiles(int tm, int tn, F&& f) const {
    const int G = tile_group_;
    for (int bm = 0; bm < tm; bm += G)
      for (int bn = 0; bn < tn; bn += G)
        for (int mb = bm; mb < std::min(tm, bm + G); ++mb)
          for (int nb = bn; nb < std::min(tn, bn + G); ++nb) f(mb, nb);
  }
  // Launch order of a grouped product's tiles (tile_order_): 0, the longest K ranges first (the
  // persistent CTAs then finish close together); 1, problems by decreasing K with the tiles of a
  // problem kept together in their blocked order (the CTAs working at the same time share its
  // panels in L2).
  void order_tiles(std::vector<GTile>& tiles, const std::vector<GProblem>& pr) const {
    if (tile_order_ == 0)
      std::stable_sort(tiles.begin(), tiles.end(),
                       [](const GTile& x, const GTile& y) { return (x.kb1 - x.kb0) > (y.kb1 - y.kb0); });
    else
      std::stable_sort(tiles.begin(), tiles.end(),
                       [&](const GTile& x, const GTile& y) { return pr[x.prob].K > pr[y.prob].K; });
  }

  // Autotuning of the phase-2 schedule (tile_group_, tile_order_): every candidate is recorded,
  // replayed once to warm up and once timed on this batch, and the fastest is kept.  Phase 2
  // overwrites the powers that phase 1 left in the arenas, so phase 1 is replayed before every
  // phase-2 run (and once more before the real one); only phase 2 is timed.  The schedule
  // changes only the order in which tiles run, never a tile's arithmetic, so the results do not
  // depend on it.
  void autotune_phase2(const std::vector<const void*>& tab) {
    static const int cand[][2] = {{8, 0}, {8, 1}, {4, 0}, {16, 0}, {16, 1}};
    tuned_.clear();
    double best = 1e300;
    int bg = tile_group_, bo = tile_order_;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    FX_CUDA(cudaEventCreate(&e0));
    FX_CUDA(cudaEventCreate(&e1));
    try {
      for (const auto& c : cand) {
        tile_group_ = c[0];
        tile_order_ = c[1];
        key2_.clear();
        replay_phase1();
        run_phase2(tab);
        replay_phase1();
        FX_CUDA(cudaEventRecord(e0, stream_));
        run_phase2(tab);
        FX_CUDA(cudaEventRecord(e1, stream_));
        FX_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        FX_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        tuned_.push_back({(double)c[0], (double)c[1], (double)ms});
        if (ms < best) {
          best = ms;
          bg = c[0];
          bo = c[1];
        }
      }
    } catch (...) {
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    tile_group_ = bg;
    tile_order_ = bo;
    key2_.clear();
    replay_phase1();
  }
  void replay_phase1() { run_recorded(desc1_, st1_, r1_, graph1_, use_graph_ && !profile_); }

  // Real multiply-adds x 2 that the listed tiles compute (tile-level: 128 x BN x 64 per K step
  // and term); the int8 MMA operations issued are S(S+1)/2 times that.
  static double tile_ops(const std::vector<GTile>& tiles, int nterms, int S = kS) {
    double steps = 0;
    for (const GTile& t : tiles) steps += t.kb1 - t.kb0;
    return steps * 2.0 * 128.0 * i8_tile_bn(S) * 64.0 * nterms;
  }
  // Real product D_w = alpha_w A_w B_w + beta_w C_w + gamma_w I on np x np blocks of the listed
  // walks (arenas; B symmetric so Bt = B); c_arena < 0: no C.
  // split: take the diagonals out of the int8 slices (operands close to a multiple of I).
  // b_cached (a_cached): walks whose B (A) slices, exponents and split-off diagonals from an
  // earlier product of the same operand, slice count and split are still in the B (A) planes:
  // not sliced again.
  void product(Staging& st, Rec& r, const std::vector<int>& list, int a, int b, double alpha, int c_arena,
               double beta, double gamma, int d_arena, bool sym, const std::vector<double>* alpha_w = nullptr,
               const std::vector<double>* gamma_w = nullptr, bool split = false,
               const std::vector<char>* b_cached = nullptr, const std::vector<char>* a_cached = nullptr) {
    std::vector<GSlab> sa, sb;
    std::vector<GProblem> pr;
    const bool same = a == b;
    split = split && (split_ & 1);
    for (int w : list) {
      const BWalk& bw = walks_[w];
      const int dg = split ? 0 : kNoDiag;
      if (!(a_cached && (*a_cached)[w] && !same))
        sa.push_back(GSlab{A(a) + bw.off, nullptr, bw.np, bw.np, bw.np, (int)bw.row0, dg});
      if (!same && !(b_cached && (*b_cached)[w]))
        sb.push_back(GSlab{A(b) + bw.off, nullptr, bw.np, bw.np, bw.np, (int)bw.row0, dg});
      GProblem p{};
      p.a_row0 = p.b_row0 = (int)bw.row0;
      p.M = p.N = p.K = bw.np;
      p.sym = sym ? 1 : 0;
      p.alpha = alpha_w ? (*alpha_w)[w] : alpha;
      p.beta = c_arena >= 0 ? beta : 0.0;
      p.gamma = gamma_w ? (*gamma_w)[w] : gamma;
      p.C = c_arena >= 0 ? A(c_arena) + bw.off : nullptr;
      p.ldc = bw.np;
      p.D = A(d_arena) + bw.off;
      p.ldd = bw.np;
      if (split) {   // A and B symmetric (polynomials in Y): Bt = B, A read by columns
        p.split = 2;
        p.Am = A(a) + bw.off;
        p.Btm = A(b) + bw.off;
        p.ldam = p.ldbm = bw.np;
      }
      pr.push_back(p);
    }
    grouped(st, r, sa, same ? nullptr : &sb, pr, same, 0, split);
  }

  // Generic grouped product over explicit slabs and problems (one real term; A slabs into
  // the A re planes, B slabs into the B re planes, or B = A when `same`).  tri: 0 none;
  // 1: Bt rows are lower-triangular rows (Bt[c][k] = 0 for k > c); 2: Bt[c][k] = 0 for k < c;
  // 3: A[r][k] = 0 for k > r.
  // split: the slabs leave their diagonals out of the slices (GSlab::diag0) and the problems
  // add the diagonal terms in FP64 (GProblem::split).  A diagonal much larger than the rest of
  // its row (V ~ b_0 I, G, L^-1, the Pade numerator) would otherwise set the row's exponent
  // and cost the off-diagonal entries as many bits as the ratio.
  void grouped(Staging& st, Rec& r, const std::vector<GSlab>& sa, const std::vector<GSlab>* sb,
               const std::vector<GProblem>& pr, bool same, int tri, bool split = false) {
    if (pr.empty()) return;
    const int S = gS_;
    const int bn = i8_tile_bn(S);
    std::vector<GTile> tiles;
    for (int i = 0; i < (int)pr.size(); ++i) {
      const GProblem& p = pr[i];
      const int tm = (p.M + 127) / 128, tn = (p.N + bn - 1) / bn, kbs = p.K / 64;
      for_tiles(tm, tn, [&](int mb, int nb) {
        if (p.sym && !((long long)nb * bn + bn - 1 >= (long long)mb * 128)) return;
        int kb0 = 0, kb1 = kbs;
        if (tri == 1) kb1 = std::min(kbs, (nb * bn + bn + 63) / 64);
        if (tri == 2) kb0 = std::min(kbs, (nb * bn) / 64);
        if (tri == 3) kb1 = std::min(kbs, (mb * 128 + 128 + 63) / 64);
        tiles.push_back(GTile{i, mb, nb, kb0, kb1, 0});
      });
    }
    order_tiles(tiles, pr);
    std::vector<GSlab> a_sorted = sa, b_sorted = sb ? *sb : std::vector<GSlab>();
    auto by_row = [](const GSlab& x, const GSlab& y) { return x.row0 < y.row0; };
    std::sort(a_sorted.begin(), a_sorted.end(), by_row);
    std::sort(b_sorted.begin(), b_sorted.end(), by_row);
    const size_t o_sa = st.put(a_sorted), o_sb = st.put(b_sorted), o_pr = st.put(pr), o_t = st.put(tiles);
    const int nsa = (int)a_sorted.size(), nsb = (int)b_sorted.size(), nt = (int)tiles.size();
    const double ops = tile_ops(tiles, 1, S);
    int64_t a_span = 0, b_span = 0;
    const std::vector<int> pla = slice_plan(a_sorted), plb = slice_plan(b_sorted);
    const size_t o_pla = st.put(pla), o_plb = st.put(plb);
    const int bla = pla.back(), blb = plb.back();
    for (const GSlab& g : a_sorted) a_span = std::max<int64_t>(a_span, (int64_t)g.row0 + g.rows);
    for (const GSlab& g : b_sorted) b_span = std::max<int64_t>(b_span, (int64_t)g.row0 + g.rows);
    r.launches += same ? 2 : 3;
    r.gemms += 1;
    const int tag = tag_;
    r.ops.push_back([=]() {
      I8Slices outa{}, outb{};
      for (int q = 0; q < S; ++q) {
        outa.re[q] = slice_plane(0, q);
        outb.re[q] = slice_plane(3, q);
      }
      outa.exp = aexp();
      outb.exp = bexp();
      outa.dg = split ? adiag() : nullptr;
      outb.dg = split ? bdiag() : nullptr;
      outa.ld = outb.ld = pitch_;
      launch_slice_rows_grouped<double>(S, dev<GSlab>(o_sa), nsa, a_span, outa, false, stream_,
                                        SlicePlan{dev<int>(o_pla), bla});
      I8Term t{};
      for (int q = 0; q < S; ++q) t.a[q] = outa.re[q];
      if (!same) {
        launch_slice_rows_grouped<double>(S, dev<GSlab>(o_sb), nsb, b_span, outb, false, stream_,
                                          SlicePlan{dev<int>(o_plb), blb});
        for (int q = 0; q < S; ++q) t.b[q] = outb.re[q];
      } else {
        for (int q = 0; q < S; ++q) t.b[q] = outa.re[q];
      }
      const size_t pi = prof_begin();
      launch_gemm_i8_grouped<double>(S, &t, 1, pitch_, a_rows_, same ? a_rows_ : rows_, aexp(),
                                     same ? aexp() : bexp(), dev<GProblem>(o_pr), dev<GTile>(o_t), nt,
                                     (int*)err_.p, timeout_ms_, stream_, split ? adiag() : nullptr,
                                     split ? (same ? adiag() : bdiag()) : nullptr, next_skip());
      prof_end(pi, ops * S * (S + 1) / 2, ops, tag);
    });
  }

  // Row chunks of the listed walks' n x n (use_n) or np x np blocks, about kChunkElems each.
  std::vector<RChunk> row_chunks(const std::vector<int>& list, bool use_n) const {
    std::vector<RChunk> ch;
    for (int w : list) {
      const int rows = use_n ? walks_[w].n : walks_[w].np, cols = rows;
      const int R = std::max(1, kChunkElems / std::max(1, cols));
      for (int r0 = 0; r0 < rows; r0 += R) ch.push_back(RChunk{w, r0, std::min(rows, r0 + R), 0});
    }
    return ch;
  }

  void combo(Staging& st, Rec& r, const std::vector<int>& list, int d_arena, const int m_arena[4],
             const std::vector<std::array<double, 5>>& coef) {
    if (list.empty()) return;
    std::vector<double> c(5 * count(), 0.0);
    for (int w : list)
      for (int k = 0; k < 5; ++k) c[5 * w + k] = coef[w][k];
    const std::vector<RChunk> ch = row_chunks(list, false);
    const size_t o_ch = st.put(ch), o_c = st.put(c);
    Planes4 M{};
    for (int k = 0; k < 4; ++k) M.m[k] = m_arena[k] >= 0 ? A(m_arena[k]) : nullptr;
    double* D = A(d_arena);
    const unsigned nch = (unsigned)ch.size();
    r.launches += 1;
    r.ops.push_back([=]() {
      kb_combo<4><<<nch, 256, 0, stream_>>>(D, M, dev<RChunk>(o_ch), (const BWalk*)d_walks_.p, dev<double>(o_c));
      FX_LAUNCH_CHECK();
    });
  }

  // D = sum_k c_k M_k + g I over five arenas (kb_combo<5>); coef[w] = (c_0..c_4, g).
  void combo5(Staging& st, Rec& r, const std::vector<int>& list, int d_arena, const int m_arena[5],
              const std::vector<std::array<double, 6>>& coef) {
    if (list.empty()) return;
    std::vector<double> c(6 * count(), 0.0);
    for (int w : list)
      for (int k = 0; k < 6; ++k) c[6 * w + k] = coef[w][k];
    const std::vector<RChunk> ch = row_chunks(list, false);
    const size_t o_ch = st.put(ch), o_c = st.put(c);
    PlanesN<5> M{};
    for (int k = 0; k < 5; ++k) M.m[k] = m_arena[k] >= 0 ? A(m_arena[k]) : nullptr;
    double* D = A(d_arena);
    const unsigned nch = (unsigned)ch.size();
    r.launches += 1;
    r.ops.push_back([=]() {
      kb_combo<5><<<nch, 256, 0, stream_>>>(D, M, dev<RChunk>(o_ch), (const BWalk*)d_walks_.p, dev<double>(o_c));
      FX_LAUNCH_CHECK();
    });
  }



  void transpose(Staging& st, Rec& r, const std::vector<int>& list, int in, int out) {
    if (list.empty()) return;
    const size_t o_l = st.put(list);
    const int nl = (int)list.size();
    const double* src = A(in);
    double* dst = A(out);
    const unsigned gx = (unsigned)std::min(1024, std::max(8, 148 * 8 / nl));
    r.launches += 1;
    r.ops.push_back([=]() {
      kb_transpose<<<dim3(gx, 1, nl), dim3(32, 8), 0, stream_>>>(src, dst, dev<int>(o_l), (const BWalk*)d_walks_.p, 0);
      FX_LAUNCH_CHECK();
    });
  }

  void symmetrize(Staging& st, Rec& r, const std::vector<int>& list, int a) {
    if (list.empty()) return;
    const size_t o_l = st.put(list);
    const int nl = (int)list.size();
    double* p = A(a);
    const unsigned gx = (unsigned)std::min(1024, std::max(8, 148 * 8 / nl));
    r.launches += 1;
    r.ops.push_back([=]() {
      kb_symmetrize<<<dim3(gx, 1, nl), dim3(32, 8), 0, stream_>>>(p, dev<int>(o_l), (const BWalk*)d_walks_.p);
      FX_LAUNCH_CHECK();
    });
  }

  // Exact projection E 1 = 0 = 1^T E of the symmetric iterates of rank-one-shifted walks.
  void project(Staging& st, Rec& r, const std::vector<int>& list, int a) {
    if (list.empty()) return;
    const size_t o_l = st.put(list);
    const int nl = (int)list.size();
    double* p = A(a);
    double* rs = rsum();
    double* tot = misc();   // W doubles
    const std::vector<RChunk> ch = row_chunks(list, true);
    const size_t o_ch = st.put(ch);
    const unsigned nch = (unsigned)ch.size();
    const dim3 g_rows(grid_x_for(maxnp_ * 32, nl), nl);
    r.ops.push_back([=]() {
      const BWalk* wk = (const BWalk*)d_walks_.p;
      kb_rowsums<<<g_rows, 256, 0, stream_>>>(p, dev<int>(o_l), wk, rs);
      FX_LAUNCH_CHECK();
      kb_walk_vec_reduce<<<nl, 256, 0, stream_>>>(rs, dev<int>(o_l), wk, 0, 1, tot, 1, 0);
      FX_LAUNCH_CHECK();
      kb_apply_proj<<<nch, 256, 0, stream_>>>(p, dev<RChunk>(o_ch), wk, rs, tot);
      FX_LAUNCH_CHECK();
    });
    r.launches += 3;
  }

  // combo2 by whole rows (kb_combo2_rs) with the signed row sums of both outputs over the n x n
  // block into rsum() and rsum2(), for the projection that follows a three-product squaring.
  void combo2_rs(Staging& st, Rec& r, const std::vector<int>& list, int d1, int d2, const int m_arena[5],
                 const std::vector<std::array<double, 12>>& coef) {
    if (list.empty()) return;
    std::vector<double> c(12 * count(), 0.0);
    for (int w : list)
      for (int k = 0; k < 12; ++k) c[12 * w + k] = coef[w][k];
    std::vector<RChunk> ch;   // rows per chunk: a multiple of the 8 warps of a CTA
    for (int w : list) {
      const int np = walks_[w].np, R = std::max(8, (kChunkElems / np) & ~7);
      for (int r0 = 0; r0 < np; r0 += R) ch.push_back(RChunk{w, r0, std::min(np, r0 + R), 0});
    }
    const size_t o_ch = st.put(ch), o_c = st.put(c);
    Planes5 M{};
    for (int k = 0; k < 5; ++k) M.m[k] = m_arena[k] >= 0 ? A(m_arena[k]) : nullptr;
    double* D1 = A(d1);
    double* D2 = A(d2);
    const unsigned nch = (unsigned)ch.size();
    r.launches += 1;
    r.ops.push_back([=]() {
      kb_combo2_rs<<<nch, 256, 0, stream_>>>(D1, D2, M, dev<RChunk>(o_ch), (const BWalk*)d_walks_.p, dev<double>(o_c),
                                             rsum(), rsum2());
      FX_LAUNCH_CHECK();
    });
  }

  // Exact projection E 1 = 0 = 1^T E of both planes of the listed walks' iterates, from the row
  // sums their squaring's combination wrote (combo2_rs), in one pass; walks with vready[w] also
  // get Er + Ei in arena V for their next squaring (the same sums combo would form).
  void project_fused(Staging& st, Rec& r, const std::vector<int>& list, const std::vector<int>& er,
                     const std::vector<int>& ei, const std::vector<char>& vready) {
    if (list.empty()) return;
    const int W = count();
    double* tot = misc();        // W doubles: the real plane's total
    double* tot2 = misc() + W;   // W doubles: the imaginary plane's total
    for (int pa : {kA4, kT1}) {
      for (int withv = 0; withv < 2; ++withv) {
        std::vector<int> l;
        for (int w : list)
          if (er[w] == pa && (int)vready[w] == withv) l.push_back(w);
        if (l.empty()) continue;
        const size_t o_l = st.put(l);
        const int nl = (int)l.size();
        double* E1 = A(er[l[0]]);
        double* E2 = A(ei[l[0]]);
        double* V = withv ? A(kV) : nullptr;
        const std::vector<RChunk> ch = row_chunks(l, false);
        const size_t o_ch = st.put(ch);
        const unsigned nch = (unsigned)ch.size();
        r.ops.push_back([=]() {
          const BWalk* wk = (const BWalk*)d_walks_.p;
          kb_walk_vec_reduce<<<nl, 256, 0, stream_>>>(rsum(), dev<int>(o_l), wk, 0, 1, tot, 1, 0);
          FX_LAUNCH_CHECK();
          kb_walk_vec_reduce<<<nl, 256, 0, stream_>>>(rsum2(), dev<int>(o_l), wk, 0, 1, tot2, 1, 0);
          FX_LAUNCH_CHECK();
          kb_apply_proj2<<<nch, 256, 0, stream_>>>(E1, E2, V, dev<RChunk>(o_ch), wk, rsum(), rsum2(), tot, tot2);
          FX_LAUNCH_CHECK();
        });
        r.launches += 3;
        (void)W;
      }
    }
  }

  // Everything after the selection.
  void record_rest(Staging& st, Rec& r) {
    const int W = count();
    // all: every walk; pd: the walks of the Pade stage and its solve (below it leaves E = R - I
    // in A4 / A2); cw: the walks of the Chebyshev polynomial stage (which leaves E there too)
    std::vector<int> all, pd, cw, m13, m9, mlt13, rank1;
    for (int w = 0; w < W; ++w) {
      all.push_back(w);
      if (rank1_[w]) rank1.push_back(w);
      if (cheb_deg_[w] >= 0) {
        cw.push_back(w);
        continue;
      }
      pd.push_back(w);
      if (sel_m_[w] == 13) m13.push_back(w);
      else mlt13.push_back(w);
      if (sel_m_[w] == 9) m9.push_back(w);
    }
    // ---- Pade numerator / denominator (powers scaled by 2^-s folded into the coefficients)
    std::vector<std::array<double, 5>> cf(W), cg(W);
    std::vector<double> al(W, 1.0), ga(W, 0.0);
    auto cs = [&](int w, int p) { return std::ldexp(1.0, -p * sel_s_[w]); };
    // the Pade and solve products: 5 slices, or the mixed form's count (pade_slices_of); the
    // (dominant) diagonals of the Pade products' operands are taken out of their slices
    const bool psplit = form_ == 1 || (split_ & 4);
    const auto ps = [&](int w) { return pade_slices_of(w); };
    // m = 9: A8 = A4 A4 -> T2
    tag_ = kTagPade;
    by_slices(m9, ps, [&](const std::vector<int>& l) {
      product(st, r, l, kA4, kA4, 1.0, -1, 0.0, 0.0, kT2, true, nullptr, nullptr, psplit);
    });
    // m = 13: T1 = b13 A6 + b11 A4 + b9 A2 (scaled), T2 = A6 T1 (scaled)
    for (int w : m13) {
      const auto b = pade_coeffs(13);
      cf[w] = {b[13] * cs(w, 6), b[11] * cs(w, 4), b[9] * cs(w, 2), 0.0, 0.0};
      al[w] = cs(w, 6);
    }
    const int m_642[4] = {kA6, kA4, kA2, -1};
    combo(st, r, m13, kT1, m_642, cf);
    by_slices(m13, ps, [&](const std::vector<int>& l) {
      product(st, r, l, kA6, kT1, 1.0, -1, 0.0, 0.0, kT2, true, &al, nullptr, psplit);
    });
    // odd part: T1 = [T2] + b7 A6 + b5 A4 + b3 A2 + b1 I  (T2 = W1 for m = 13, A8 for m = 9)
    const int m_t2642[4] = {kT2, kA6, kA4, kA2};
    for (int w : pd) {
      const int m = sel_m_[w];
      const auto b = pade_coeffs(m);
      // powers of the scaled generator Y / 2^s: A_k -> 2^(-k s) A_k (s = 0 for the plain
      // choice of m < 13; the certified and learned choices may scale any degree)
      if (m == 13) cf[w] = {1.0, b[7] * cs(w, 6), b[5] * cs(w, 4), b[3] * cs(w, 2), b[1]};
      else if (m == 9) cf[w] = {b[9] * cs(w, 8), b[7] * cs(w, 6), b[5] * cs(w, 4), b[3] * cs(w, 2), b[1]};
      else if (m == 7) cf[w] = {0.0, b[7] * cs(w, 6), b[5] * cs(w, 4), b[3] * cs(w, 2), b[1]};
      else if (m == 5) cf[w] = {0.0, 0.0, b[5] * cs(w, 4), b[3] * cs(w, 2), b[1]};
      else cf[w] = {0.0, 0.0, 0.0, b[3] * cs(w, 2), b[1]};
      al[w] = cs(w, 1);
    }
    combo(st, r, pd, kT1, m_t2642, cf);
    // U = i W with W = c Yim T1
    by_slices(pd, ps, [&](const std::vector<int>& l) {
      product(st, r, l, kY, kT1, 1.0, -1, 0.0, 0.0, kW, true, &al, nullptr, psplit);
    });
    // even part.  m = 13: T1 = b12 A6 + b10 A4 + b8 A2, T2 = b6 A6 + b4 A4 + b2 A2,
    // V = A6 T1 + T2 + b0 I.  m < 13: V = [b8 A8] + b6 A6 + b4 A4 + b2 A2 + b0 I.
    for (int w : m13) {
      const auto b = pade_coeffs(13);
      cf[w] = {b[12] * cs(w, 6), b[10] * cs(w, 4), b[8] * cs(w, 2), 0.0, 0.0};
      cg[w] = {b[6] * cs(w, 6), b[4] * cs(w, 4), b[2] * cs(w, 2), 0.0, 0.0};
      al[w] = cs(w, 6);
      ga[w] = b[0];
    }
    combo(st, r, m13, kT1, m_642, cf);
    combo(st, r, m13, kT2, m_642, cg);
    for (int w : mlt13) {
      const int m = sel_m_[w];
      const auto b = pade_coeffs(m);
      if (m == 9) cf[w] = {b[8] * cs(w, 8), b[6] * cs(w, 6), b[4] * cs(w, 4), b[2] * cs(w, 2), b[0]};
      else if (m == 7) cf[w] = {0.0, b[6] * cs(w, 6), b[4] * cs(w, 4), b[2] * cs(w, 2), b[0]};
      else if (m == 5) cf[w] = {0.0, 0.0, b[4] * cs(w, 4), b[2] * cs(w, 2), b[0]};
      else cf[w] = {0.0, 0.0, 0.0, b[2] * cs(w, 2), b[0]};
    }
    combo(st, r, mlt13, kV, m_t2642, cf);
    by_slices(m13, ps, [&](const std::vector<int>& l) {
      product(st, r, l, kA6, kT1, 1.0, kT2, 1.0, 0.0, kV, true, &al, &ga, psplit);
    });

    // ---- solve: G = V^2 + W^2 = L L^T, P2 = (V + iW)^2, R = G^-1 P2
    // V ~ b_0 I once scaled: these products and the complex ones below split the diagonals off
    tag_ = kTagSolve;
    by_slices(pd, ps, [&](const std::vector<int>& l) {
      product(st, r, l, kV, kV, 1.0, -1, 0.0, 0.0, kT1, true, nullptr, nullptr, true);    // VV
      product(st, r, l, kW, kW, 1.0, -1, 0.0, 0.0, kT2, true, nullptr, nullptr, true);    // WW
      product(st, r, l, kV, kW, 1.0, -1, 0.0, 0.0, kA2, true, nullptr, nullptr, true);    // VW
    });
    const int m_12[4] = {kT1, kT2, -1, -1};
    const int m_a2[4] = {kA2, -1, -1, -1};
    for (int w = 0; w < W; ++w) cf[w] = {1.0, 1.0, 0.0, 0.0, 0.0};
    combo(st, r, pd, kA4, m_12, cf);                              // G -> A4
    for (int w = 0; w < W; ++w) cf[w] = {1.0, -1.0, 0.0, 0.0, 0.0};
    combo(st, r, pd, kA6, m_12, cf);                              // P2 re -> A6
    for (int w = 0; w < W; ++w) cf[w] = {2.0, 0.0, 0.0, 0.0, 0.0};
    combo(st, r, pd, kY, m_a2, cf);                               // P2 im -> Y
    // large walks solve by Newton-Schulz (their Cholesky would be a long chain of dependent
    // block steps); smaller walks, whose few steps run grouped over the batch, keep the
    // Cholesky solve
    std::vector<int> ns_list, ch_list;
    for (int w : pd) (uses_newton(w) ? ns_list : ch_list).push_back(w);
    by_slices(ns_list, ps, [&](const std::vector<int>& l) { newton_solve(st, r, l); });   // R re -> A4, im -> A2
    by_slices(ch_list, ps, [&](const std::vector<int>& l) {
      tag_ = kTagCholesky;
      cholesky(st, r, kA4, l);
      transpose(st, r, l, kA4, kT1);                              // L^T -> T1
      tag_ = kTagInverse;
      inverse(st, r, kT1, kT2, kW, kA2, l);                       // X = L^-1 -> T2, X^T -> W (scratch A2)
      // Z = P2 X^T (re -> V, im -> T1); R^T = Z X (re -> A4, im -> A2)
      tag_ = kTagTriangular;
      complex_by_real(st, r, l, kA6, kY, kT2, kV, kT1, 1, true);    // P2 symmetric
      complex_by_real(st, r, l, kV, kT1, kW, kA4, kA2, 2, false);
      symmetrize(st, r, l, kA4);
      symmetrize(st, r, l, kA2);
    });


    // ---- squarings in I + E form: E = R - I, E <- 2E + E^2
    for (int w = 0; w < W; ++w) cf[w] = {1.0, 0.0, 0.0, 0.0, -1.0};
    const int m_a4[4] = {kA4, -1, -1, -1};
    combo(st, r, pd, kA4, m_a4, cf);
    // the Chebyshev walks: E = p(Z) - I straight into A4 / A2
    chebyshev(st, r, cw);
    std::vector<int> er(W, kA4), ei(W, kA2), tr(W, kT1), ti(W, kT2);
    project_pair(st, r, rank1, er, ei);
    int smax = 0;
    for (int w = 0; w < W; ++w) smax = std::max(smax, sel_s_[w]);
    if (drift_) {
      if (!drift_buf_.p) drift_buf_.alloc(sizeof(double) * (size_t)W * kDriftMax);
      const size_t bytes = drift_buf_.bytes;
      r.ops.push_back([=]() { FX_CUDA(cudaMemsetAsync(drift_buf_.p, 0, bytes, stream_)); });
    }
    tag_ = kTagSquare;
    std::vector<char> vready(W, 0);   // walks whose Er + Ei (arena V) the projection formed
    for (int k = 0; k < smax; ++k) {
      std::vector<int> act;
      for (int w = 0; w < W; ++w)
        if (sel_s_[w] > k) act.push_back(w);
      if (drift_) drift(st, r, act, er, ei, std::vector<int>(W, std::min(k, kDriftMax - 1)));
      std::vector<int> act3, act4;
      for (int w : act) (use_square3(w) ? act3 : act4).push_back(w);
      if (!act3.empty()) square3(st, r, act3, er, ei, tr, ti, k, vready);
      if (!act4.empty()) square(st, r, act4, er, ei, tr, ti);
      for (int w : act) {
        std::swap(er[w], tr[w]);
        std::swap(ei[w], ti[w]);
      }
      // the projection of rank-one walks: after a three-product squaring with the row sums its
      // combination took, both planes in one pass that also forms the next squaring's Er + Ei
      // (not with the drift diagnostics, whose products use that arena in between)
      std::vector<int> pj3, pj4;
      std::fill(vready.begin(), vready.end(), 0);
      for (int w : act) {
        if (!rank1_[w]) continue;
        (use_square3(w) ? pj3 : pj4).push_back(w);
        if (use_square3(w) && !drift_ && sel_s_[w] > k + 1) vready[w] = 1;
      }
      project_fused(st, r, pj3, er, ei, vready);
      project_pair(st, r, pj4, er, ei);
    }
    if (drift_) {
      std::vector<int> last(W);
      for (int w = 0; w < W; ++w) last[w] = std::min(sel_s_[w], kDriftMax - 1);
      drift(st, r, all, er, ei, last);
    }

    // ---- outputs: psi = e^mu (E psi0 + psi0 + cj (1^T psi0) 1) and U = e^mu (I + E + cj J)
    std::vector<const double*> pre(W), pim(W);
    std::vector<double> om(4 * W);
    for (int w = 0; w < W; ++w) {
      pre[w] = A(er[w]);
      pim[w] = A(ei[w]);
      const std::complex<double> e = std::exp(mu_[w]);
      om[4 * w] = e.real();
      om[4 * w + 1] = e.imag();
      if (rank1_[w]) {
        const std::complex<double> cj = (std::exp(nu_[w]) - 1.0) / (double)walks_[w].n;
        om[4 * w + 2] = cj.real();
        om[4 * w + 3] = cj.imag();
      }
    }
    const size_t o_pre = st.put(pre), o_pim = st.put(pim), o_om = st.put(om), o_all = st.put(all);
    double* psum = misc() + 2 * W;
    const dim3 g_rows(grid_x_for(maxnp_ * 32, W), W);
    const dim3 g_el(grid_x_for(maxnp_ * maxnp_, W), W);
    const int dt = dtype_;
    r.launches += 3;
    r.ops.push_back([=]() {
      const BWalk* wk = (const BWalk*)d_walks_.p;
      const int* l = dev<int>(o_all);
      const double* const* er_ = dev<const double*>(o_pre);
      const double* const* ei_ = dev<const double*>(o_pim);
      if (dt == FX_C64) {
        kb_psi_sum<float2><<<W, 256, 0, stream_>>>(dP0(), l, wk, psum);
        FX_LAUNCH_CHECK();
        kb_apply<float2><<<g_rows, 256, 0, stream_>>>(er_, ei_, dP0(), dP1(), l, wk, dev<double>(o_om), psum);
        FX_LAUNCH_CHECK();
        kb_output<float2><<<g_el, 256, 0, stream_>>>(er_, ei_, dUo(), l, wk, dev<double>(o_om));
      } else {
        kb_psi_sum<double2><<<W, 256, 0, stream_>>>(dP0(), l, wk, psum);
        FX_LAUNCH_CHECK();
        kb_apply<double2><<<g_rows, 256, 0, stream_>>>(er_, ei_, dP0(), dP1(), l, wk, dev<double>(o_om), psum);
        FX_LAUNCH_CHECK();
        kb_output<double2><<<g_el, 256, 0, stream_>>>(er_, ei_, dUo(), l, wk, dev<double>(o_om));
      }
      FX_LAUNCH_CHECK();
    });
  }

  void project_pair(Staging& st, Rec& r, const std::vector<int>& list, const std::vector<int>& er,
                    const std::vector<int>& ei) {
    // group the walks by the arena their iterate lives in
    for (int pa : {kA4, kT1}) {
      std::vector<int> l1;
      for (int w : list)
        if (er[w] == pa) l1.push_back(w);
      project(st, r, l1, pa);
    }
    for (int pa : {kA2, kT2}) {
      std::vector<int> l2;
      for (int w : list)
        if (ei[w] == pa) l2.push_back(w);
      project(st, r, l2, pa);
    }
  }

  // One squaring E <- 2E + E^2 of the listed walks (E symmetric complex, planes er/ei; result in
  // tr/ti).  Walks whose iterates sit in different arena pairs go in separate launches.
  void square(Staging& st, Rec& r, const std::vector<int>& act, const std::vector<int>& er,
              const std::vector<int>& ei, const std::vector<int>& tr, const std::vector<int>& ti) {
    for (int pa : {kA4, kT1}) {
      std::vector<int> l;
      for (int w : act)
        if (er[w] == pa) l.push_back(w);
      if (l.empty()) continue;
      const int re = er[l[0]], im = ei[l[0]], ore = tr[l[0]], oim = ti[l[0]];
      std::vector<GSlab> sa;
      std::vector<GProblem> prr, pri;
      for (int w : l) {
        const BWalk& b = walks_[w];
        sa.push_back(GSlab{A(re) + b.off, A(im) + b.off, b.np, b.np, b.np, (int)b.row0, kNoDiag});
        GProblem p{};
        p.a_row0 = p.b_row0 = (int)b.row0;
        p.M = p.N = p.K = b.np;
        p.sym = 1;
        p.alpha = 1.0;
        p.beta = 2.0;
        p.ldc = p.ldd = b.np;
        p.C = A(re) + b.off;
        p.D = A(ore) + b.off;
        prr.push_back(p);
        p.C = A(im) + b.off;
        p.D = A(oim) + b.off;
        pri.push_back(p);
      }
      const int bn = i8_tile_bn(kS);
      std::vector<GTile> tiles;
      for (int i = 0; i < (int)prr.size(); ++i) {
        const int tm = (prr[i].M + 127) / 128, tn = (prr[i].N + bn - 1) / bn;
        for_tiles(tm, tn, [&](int mb, int nb) {
          if ((long long)nb * bn + bn - 1 >= (long long)mb * 128) tiles.push_back(GTile{i, mb, nb, 0, prr[i].K / 64, 0});
        });
      }
      order_tiles(tiles, prr);
      std::sort(sa.begin(), sa.end(), [](const GSlab& x, const GSlab& y) { return x.row0 < y.row0; });
      const size_t o_sa = st.put(sa), o_r = st.put(prr), o_i = st.put(pri), o_t = st.put(tiles);
      const int nsa = (int)sa.size(), nt = (int)tiles.size();
      const std::vector<int> pl = slice_plan(sa);
      const size_t o_pl = st.put(pl);
      const int bl = pl.back();
      const double ops = tile_ops(tiles, 2);
      r.launches += 3;
      r.gemms += 2;
      r.ops.push_back([=]() {
        I8Slices out{};
        for (int q = 0; q < kS; ++q) {
          out.re[q] = slice_plane(0, q);
          out.im[q] = slice_plane(1, q);
          out.neg_im[q] = slice_plane(2, q);
        }
        out.exp = aexp();
        out.ld = pitch_;
        launch_slice_rows_grouped<double>(kS, dev<GSlab>(o_sa), nsa, rows_, out, true, stream_,
                                          SlicePlan{dev<int>(o_pl), bl});
        I8Term t[2];
        // real: Re Re + Im (-Im)
        for (int q = 0; q < kS; ++q) {
          t[0].a[q] = out.re[q];
          t[0].b[q] = out.re[q];
          t[1].a[q] = out.im[q];
          t[1].b[q] = out.neg_im[q];
        }
        size_t pi = prof_begin();
        launch_gemm_i8_grouped<double>(kS, t, 2, pitch_, rows_, rows_, aexp(), aexp(), dev<GProblem>(o_r),
                                       dev<GTile>(o_t), nt, (int*)err_.p, timeout_ms_, stream_, nullptr, nullptr,
                                       next_skip());
        prof_end(pi, ops * kS * (kS + 1) / 2, ops, kTagSquare);
        // imaginary: Re Im + Im Re
        for (int q = 0; q < kS; ++q) {
          t[0].a[q] = out.re[q];
          t[0].b[q] = out.im[q];
          t[1].a[q] = out.im[q];
          t[1].b[q] = out.re[q];
        }
        pi = prof_begin();
        launch_gemm_i8_grouped<double>(kS, t, 2, pitch_, rows_, rows_, aexp(), aexp(), dev<GProblem>(o_i),
                                       dev<GTile>(o_t), nt, (int*)err_.p, timeout_ms_, stream_, nullptr, nullptr,
                                       next_skip());
        prof_end(pi, ops * kS * (kS + 1) / 2, ops, kTagSquare);
      });
    }
  }

  // Mixed form: R = G^-1 P2 by the Newton-Schulz iteration X <- X (2I - G X) for G^-1, instead of
  // the blocked Cholesky (79 dependent 128-wide steps at N = 10000, each a latency-bound block
  // factorisation on one SM and short-K products).  In the eigenbasis of the walk's generator G is
  // g(x) = |q_m(ix)|^2, x = lambda / 2^s, with q_m the Pade denominator (unnormalised coefficients,
  // as the combinations use them); over |x| <= x_max = rho / 2^s its range [g_lo, g_hi] is taken on
  // a fine grid on the host (rho: the rigorous bound min(||Y||_1, d4, d6), or 1.25 x the Lanczos
  // estimate when that is smaller).  X1 = a (2I - a G), a = 2 / (g_lo + g_hi), has the residual
  // ||I - G X1|| <= r^2, r = (g_hi - g_lo) / (g_hi + g_lo), and every step squares it: the count of
  // steps to reach 1e-13 is fixed per walk before the launch sequence is recorded.  Every iterate
  // is a polynomial in G (symmetric, commuting with G), so the products compute upper triangles;
  // the fixed point attracts (the map's derivative vanishes there), so rounding does not build up.
  // Scratch arenas: T1 / V hold the iterates, T2 = G X.
  static double pade_denominator_sq(const std::vector<double>& b, double x) {
    std::complex<double> acc(0.0, 0.0);
    const std::complex<double> z(0.0, -x);   // q(ix) = sum_j b_j (-ix)^j
    for (int j = (int)b.size() - 1; j >= 0; --j) acc = acc * z + b[j];
    return std::norm(acc);
  }
  void newton_solve(Staging& st, Rec& r, const std::vector<int>& list) {
    const int W = count();
    tag_ = kTagNewton;
    std::vector<int> iters(W, 0), lo_steps(W, 0);
    std::vector<std::array<double, 5>> cf(W, {0.0, 0.0, 0.0, 0.0, 0.0});
    for (int w : list) {
      const std::vector<double> b = pade_coeffs(sel_m_[w]);
      const double rho = std::min(rho_up_[w], 1.25 * rho_lan_[w] > 0.0 ? 1.25 * rho_lan_[w] : rho_up_[w]);
      const double xmax = std::ldexp(rho, -sel_s_[w]);
      double glo = 1e300, ghi = 0.0;
      for (int i = 0; i <= 512; ++i) {
        const double g = pade_denominator_sq(b, xmax * i / 512.0);
        glo = std::min(glo, g);
        ghi = std::max(ghi, g);
      }
      ghi *= 1.0 + 1e-6;   // between the grid points
      const double a = 2.0 / (glo + ghi);
      double res = (ghi - glo) / (ghi + glo);
      res *= res;   // after X1
      int k = 0;
      while (res > 1e-13 && k < 16) {
        res *= res;
        ++k;
      }
      iters[w] = k;
      // steps whose model residual stays above kNewtonLoRes take newton_S_ slices: the
      // iteration corrects their rounding (its fixed point attracts), and the later steps at
      // the full slice count square the residual as in exact arithmetic
      double rk = (ghi - glo) / (ghi + glo);
      rk *= rk;
      for (int j = 0; j < k; ++j) {
        rk *= rk;
        if (rk > kNewtonLoRes) lo_steps[w] = j + 1;
      }
      cf[w] = {-a * a, 0.0, 0.0, 0.0, 2.0 * a};
    }
    const int m_g[4] = {kA4, -1, -1, -1};
    combo(st, r, list, kT1, m_g, cf);   // X1 = -a^2 G + 2a I
    std::vector<int> xa(W, kT1), xb(W, kV);
    int kmax = 0;
    for (int w : list) kmax = std::max(kmax, iters[w]);
    for (int k = 0; k < kmax; ++k) {
      std::vector<int> act;
      for (int w : list)
        if (iters[w] > k) act.push_back(w);
      const int full = gS_;
      for (int pa : {kT1, kV}) {
        for (int S : {newton_S_, full}) {
          std::vector<int> l;
          for (int w : act)
            if (xa[w] == pa && (k < lo_steps[w] ? newton_S_ : full) == S) l.push_back(w);
          if (l.empty()) continue;
          const int nx = pa == kT1 ? kV : kT1;
          gS_ = S;
          product(st, r, l, kA4, pa, 1.0, -1, 0.0, 0.0, kT2, true, nullptr, nullptr, true);   // G X
          product(st, r, l, pa, kT2, -1.0, pa, 2.0, 0.0, nx, true, nullptr, nullptr, true);  // 2X - X G X
          if (S == full) break;   // newton_S_ == full: one group
        }
      }
      gS_ = full;
      for (int w : act) std::swap(xa[w], xb[w]);
    }
    tag_ = kTagTriangular;
    for (int pa : {kT1, kV}) {
      std::vector<int> l;
      for (int w : list)
        if (xa[w] == pa) l.push_back(w);
      if (l.empty()) continue;
      product(st, r, l, pa, kA6, 1.0, -1, 0.0, 0.0, kA4, true, nullptr, nullptr, true);    // R re = X P2 re
      product(st, r, l, pa, kY, 1.0, -1, 0.0, 0.0, kA2, true, nullptr, nullptr, true);     // R im = X P2 im
    }
  }

  // Walk w solves the Pade step by Newton-Schulz (else Cholesky).
  bool uses_newton(int w) const {
    return solve_mode_ == 2 || (solve_mode_ == 0 && walks_[w].np >= kNewtonMinNp);
  }
  // Walk w takes the mixed form's reduced slice counts (powers, squarings, early Newton-Schulz
  // steps; the Pade and solve products by pade_slices_of).
  bool reduced(int w) const { return form_ == 1 && walks_[w].np >= kMixedMinNp; }
  // Slice count of walk w's Pade and solve products.
  int pade_slices_of(int w) const { return reduced(w) && sel_s_[w] <= kMixedMaxPadeS ? pade_S_ : kS; }
  // Walk w squares as three split products (square3), else as the exact complex square.
  // Chebyshev-Bessel polynomial stage of the listed walks (cheb_plan above): E = p(Z) - I with
  // Z = B / rho, B = Im Y in arena Y, A2 = -B^2 from phase 1.  Real part into A4, imaginary part
  // into A2, where the Pade walks leave their E.  Arenas: the baby steps T_1..T_5 of C in kBaby
  // (C = T_1 from A2 by a combination; T_2 = 2 C^2 - I, T_3 = 2 C T_2 - C, T_4 = 2 T_2^2 - I,
  // T_5 = 2 T_2 T_3 - C); the Clenshaw chains roll b_g over (A4, T1, T2) by g mod 3 with the
  // C-term r_g - b_{g+2} in A2 (odd chain) or Y (even chain, after the odd one has used B); the
  // odd chain ends in A4 and Z times it goes to A2, the even chain ends in A4.  The products take
  // the Pade stage's slice count and diagonal split.
  static constexpr int kBaby[kChebMaxBaby + 1] = {-1, kA6, kW, kV, kX1, kX2};
  void chebyshev(Staging& st, Rec& r, const std::vector<int>& cw) {
    if (cw.empty()) return;
    const int W = count();
    tag_ = kTagPade;
    const bool psplit = form_ == 1 || (split_ & 4);
    const auto ps = [&](int w) { return pade_slices_of(w); };
    std::vector<std::vector<std::array<double, kChebMaxBaby>>> re(W), ro(W);
    std::vector<int> lin, poly, odd0, odd;   // D <= 1; D >= 2; odd cofactor of degree 0; >= 1
    std::vector<int> top(W, 0);
    std::vector<double> inv_rho(W, 0.0);
    int topmax = 0;
    for (int w : cw) {
      const int D = cheb_deg_[w], m = cheb_baby_[w];
      std::vector<double> e, b;
      cheb_split(std::ldexp(cheb_rho_[w], -sel_s_[w]), D, &e, &b);
      e[0] -= 1.0;   // E = p - I: the identity term of r_0 (T_0 = I, and T_g(G) r_0 = r_0 at g = 0)
      inv_rho[w] = cheb_rho_[w] > 0.0 ? 1.0 / cheb_rho_[w] : 0.0;
      re[w] = cheb_blocks(e, m);
      if (!b.empty()) ro[w] = cheb_blocks(b, m);
      top[w] = cheb_baby_top(D, m);
      topmax = std::max(topmax, top[w]);
      if (D <= 1) lin.push_back(w);
      else poly.push_back(w);
      if (D >= 2) (b.size() == 1 ? odd0 : odd).push_back(w);
    }
    for (int k = 4; k <= topmax; ++k)   // the extra baby-step arenas, once
      if (!arena_[kBaby[k]].p) arena_[kBaby[k]].alloc(sizeof(double) * (size_t)std::max<int64_t>(elems_, 1));
    std::vector<std::array<double, 6>> cf(W);
    const int m_none[5] = {-1, -1, -1, -1, -1};
    const int m_y[5] = {kY, -1, -1, -1, -1};
    // D <= 1: E = (e_0 - 1) I + i (b_0 / rho) B, no products
    for (int w : lin) cf[w] = {0.0, 0.0, 0.0, 0.0, 0.0, re[w][0][0]};
    combo5(st, r, lin, kA4, m_none, cf);
    for (int w : lin) cf[w] = {ro[w].empty() ? 0.0 : ro[w][0][0] * inv_rho[w], 0.0, 0.0, 0.0, 0.0, 0.0};
    combo5(st, r, lin, kA2, m_y, cf);
    if (poly.empty()) return;
    // baby steps: C = 2 Z^2 - I = -(2 / rho^2) A2 - I, then T_2..T_top by products
    const int m_a2[5] = {kA2, -1, -1, -1, -1};
    for (int w : poly) cf[w] = {-2.0 * inv_rho[w] * inv_rho[w], 0.0, 0.0, 0.0, 0.0, -1.0};
    combo5(st, r, poly, kBaby[1], m_a2, cf);
    // T_k = 2 T_i T_j - T_|i-j| (i + j = k): (i, j) = (1, 1), (1, 2), (2, 2), (2, 3).  T_2 and T_4
    // square one operand (its slices in the A planes), which is then the A operand of T_3 and
    // T_5: not sliced again
    static const int kPair[kChebMaxBaby + 1][2] = {{0, 0}, {0, 0}, {1, 1}, {1, 2}, {2, 2}, {2, 3}};
    const std::vector<char> a_in(W, 1);
    for (int k = 2; k <= kChebMaxBaby; ++k) {
      std::vector<int> l;
      for (int w : poly)
        if (top[w] >= k) l.push_back(w);
      const int i = kPair[k][0], j = kPair[k][1], d = j - i;
      by_slices(l, ps, [&](const std::vector<int>& ls) {
        product(st, r, ls, kBaby[i], kBaby[j], 2.0, d > 0 ? kBaby[d] : -1, d > 0 ? -1.0 : 0.0, d > 0 ? 0.0 : -1.0,
                kBaby[k], true, nullptr, nullptr, psplit, nullptr, i != j ? &a_in : nullptr);
      });
    }
    // odd cofactor of degree 0: Im E = (b_0 / rho) B
    for (int w : odd0) cf[w] = {ro[w][0][0] * inv_rho[w], 0.0, 0.0, 0.0, 0.0, 0.0};
    combo5(st, r, odd0, kA2, m_y, cf);
    // odd chain -> A4, then Im E = (1 / rho) B (chain) -> A2
    clenshaw(st, r, odd, ro, kA2);
    std::vector<double> al(W, 1.0);
    for (int w : odd) al[w] = inv_rho[w];
    by_slices(odd, ps, [&](const std::vector<int>& l) {
      product(st, r, l, kY, kA4, 1.0, -1, 0.0, 0.0, kA2, true, &al, nullptr, psplit);
    });
    // even chain (with -I in r_0) -> A4 = Re E
    clenshaw(st, r, poly, re, kY);
  }
  // Clenshaw's recurrence in G = T_m(C) over the listed walks' blocks r[w][g][j]:
  // b_L = r_L; b_g = 2 G b_{g+1} - b_{g+2} + r_g (g = L-1 .. 1); result G b_1 - b_2 + r_0 (or r_0
  // when L = 0), which ends in A4.  b_g lives in the arena kRoll[g mod 3], so that a step never
  // writes an arena it reads; `tmp` holds the C-term r_g - b_{g+2} of each step's product.
  void clenshaw(Staging& st, Rec& r, const std::vector<int>& list,
                const std::vector<std::vector<std::array<double, kChebMaxBaby>>>& blk, int tmp) {
    if (list.empty()) return;
    static const int kRoll[3] = {kA4, kT1, kT2};
    const int W = count();
    const auto ps = [&](int w) { return pade_slices_of(w); };
    const bool psplit = form_ == 1 || (split_ & 4);
    int Lmax = 0;
    for (int w : list) Lmax = std::max(Lmax, (int)blk[w].size() - 1);
    std::vector<std::array<double, 6>> cf(W);
    // G is the B operand of every step's product (G b = b G: both are polynomials in B): its
    // slices, written to the B planes by a walk's first step, serve that walk's later steps
    // (between them only combinations run, and they write no slices and not G)
    std::vector<char> gsliced(W, 0);
    // r_g = sum_{j < m} r[g][j] T_j(C): planes T_1..T_4 (T_0 = I on the diagonal)
    const auto rg = [&](int w, int g, double last) {
      const auto& x = blk[w][g];
      return std::array<double, 6>{x[1], x[2], x[3], x[4], last, x[0]};
    };
    for (int g = Lmax; g >= 0; --g) {
      std::vector<int> start, step;
      for (int w : list) {
        const int L = (int)blk[w].size() - 1;
        if (L == g) start.push_back(w);
        else if (L > g) step.push_back(w);
      }
      // walks whose chain starts here: b_L = r_L
      const int m_t[5] = {kBaby[1], kBaby[2], kBaby[3], kBaby[4], -1};
      for (int w : start) cf[w] = rg(w, g, 0.0);
      combo5(st, r, start, kRoll[g % 3], m_t, cf);
      if (step.empty()) continue;
      // C-term r_g - b_{g+2} (b_{g+2} = 0 above the chain's top), then b_g = alpha G b_{g+1} + C-term
      const int m_c[5] = {kBaby[1], kBaby[2], kBaby[3], kBaby[4], kRoll[(g + 2) % 3]};
      for (int w : step) cf[w] = rg(w, g, g + 2 <= (int)blk[w].size() - 1 ? -1.0 : 0.0);
      combo5(st, r, step, tmp, m_c, cf);
      for (int m = 1; m <= kChebMaxBaby; ++m) {
        std::vector<int> l;
        for (int w : step)
          if (cheb_baby_[w] == m) l.push_back(w);
        by_slices(l, ps, [&](const std::vector<int>& ls) {
          product(st, r, ls, kRoll[(g + 1) % 3], kBaby[m], g >= 1 ? 2.0 : 1.0, tmp, 1.0, 0.0, kRoll[g % 3], true,
                  nullptr, nullptr, psplit, &gsliced);
          for (int w : ls) gsliced[w] = 1;
        });
      }
    }
  }
  bool use_square3(int w) const {
    return walks_[w].np >= kSquare3MinNp || sel_s_[w] >= kSquare3MinS || (split_ & 8);
  }
  // Calls f(group) for the walks of list grouped by slices(w), with gS_ set to the group's count
  // while f records; gS_ is 5 again afterwards.
  template <typename Sl, typename F>
  void by_slices(const std::vector<int>& list, Sl&& slices, F&& f) {
    for (int S : {kS, 4, 3}) {
      std::vector<int> g;
      for (int w : list)
        if (slices(w) == S) g.push_back(w);
      if (g.empty()) continue;
      gS_ = S;
      f(g);
    }
    gS_ = kS;
  }
  // Model residual below which the Newton-Schulz steps run at the full slice count.
  static constexpr double kNewtonLoRes = 1e-4;
  // Slice count of squaring k (0-based) of walk w in the mixed form.
  int sq_slices(int w, int k) const {
    if (!reduced(w)) return kS;
    const int rem = sel_s_[w] - k;   // 1 for the last squaring
    return rem <= sq_n3_ ? 3 : rem <= sq_n3_ + sq_n4_ ? 4 : kS;
  }
  // Upper-triangle tiles of the square problems (all of the same geometry per problem index).
  std::vector<GTile> sym_tiles(const std::vector<GProblem>& pr, int bn) const {
    std::vector<GTile> tiles;
    for (int i = 0; i < (int)pr.size(); ++i) {
      const int tm = (pr[i].M + 127) / 128, tn = (pr[i].N + bn - 1) / bn;
      for_tiles(tm, tn, [&](int mb, int nb) {
        if ((long long)nb * bn + bn - 1 >= (long long)mb * 128) tiles.push_back(GTile{i, mb, nb, 0, pr[i].K / 64, 0});
      });
    }
    return tiles;
  }
  // Mixed-form squaring E <- 2E + E^2 of the listed walks, E = Er + i Ei complex symmetric, as
  // three real products that are symmetric for any symmetric operands (squares of one matrix):
  //   t1 = Er Er, t2 = Ei Ei, t3 = (Er + Ei)(Er + Ei),
  //   Re = 2 Er + t1 - t2,  Im = 2 Ei + t3 - t1 - t2  (= 2 Ei + Er Ei + Ei Er),
  // three products instead of four, and no dependence on Er and Ei commuting (they do in exact
  // arithmetic, but not the rounded iterates: a form whose products are symmetric only for
  // commuting operands, such as (Er + Ei)(Er - Ei), turns that commutator into an error that
  // doubles with every squaring).  Every product takes the diagonal out of its int8 slices and
  // adds it in FP64 (diagonal split): the iterates' rows are dominated by their diagonal, which
  // would otherwise set the row exponent and cost the off-diagonal entries as many bits.
  // Scratch arenas (free during the squarings): V = Er + Ei, Y = t1, A6 = t2, W = t3.
  void square3(Staging& st, Rec& r, const std::vector<int>& act, const std::vector<int>& er,
               const std::vector<int>& ei, const std::vector<int>& tr, const std::vector<int>& ti, int k,
               const std::vector<char>& vready) {
    const int W = count();
    for (int pa : {kA4, kT1}) {
      for (int S : {5, 4, 3}) {
        std::vector<int> l;
        for (int w : act)
          if (er[w] == pa && sq_slices(w, k) == S) l.push_back(w);
        if (l.empty()) continue;
        const int re = er[l[0]], im = ei[l[0]], ore = tr[l[0]], oim = ti[l[0]];
        std::vector<std::array<double, 5>> cf(W, {1.0, 1.0, 0.0, 0.0, 0.0});
        const int m_sum[4] = {re, im, -1, -1};
        std::vector<int> lv;   // Er + Ei not yet formed by the last projection
        for (int w : l)
          if (!vready[w]) lv.push_back(w);
        combo(st, r, lv, kV, m_sum, cf);
        gS_ = S;
        product(st, r, l, re, re, 1.0, -1, 0.0, 0.0, kY, true, nullptr, nullptr, true);    // t1
        product(st, r, l, im, im, 1.0, -1, 0.0, 0.0, kA6, true, nullptr, nullptr, true);   // t2
        product(st, r, l, kV, kV, 1.0, -1, 0.0, 0.0, kW, true, nullptr, nullptr, true);    // t3
        gS_ = kS;
        // Re = 2 Er + t1 - t2, Im = 2 Ei + t3 - t1 - t2, in one pass over the five planes
        const int m_out[5] = {re, im, kY, kA6, kW};
        const std::vector<std::array<double, 12>> c2(
            W, std::array<double, 12>{2.0, 0.0, 1.0, -1.0, 0.0, 0.0, 0.0, 2.0, -1.0, -1.0, 1.0, 0.0});
        combo2_rs(st, r, l, ore, oim, m_out, c2);
      }
    }
  }

  // Diagnostics: unitarity residual of the listed walks' iterates (planes er / ei) into slot[w]
  // of the drift buffer: D1 = Er Er + Ei Ei (symmetric) -> arena V, D2 = Er Ei (full) -> arena W,
  // both with 5 slices, then kb_drift.  V and W are free during the squarings.
  void drift(Staging& st, Rec& r, const std::vector<int>& list, const std::vector<int>& er,
             const std::vector<int>& ei, const std::vector<int>& slot) {
    if (list.empty()) return;
    std::vector<GSlab> sa;
    std::vector<GProblem> p1, p2;
    std::vector<const double*> erp(count(), nullptr);
    for (int w : list) {
      const BWalk& b = walks_[w];
      sa.push_back(GSlab{A(er[w]) + b.off, A(ei[w]) + b.off, b.np, b.np, b.np, (int)b.row0, kNoDiag});
      erp[w] = A(er[w]) + b.off;
      GProblem p{};
      p.a_row0 = p.b_row0 = (int)b.row0;
      p.M = p.N = p.K = b.np;
      p.alpha = 1.0;
      p.ldd = b.np;
      p.sym = 1;
      p.D = A(kV) + b.off;
      p1.push_back(p);
      p.sym = 0;
      p.D = A(kW) + b.off;
      p2.push_back(p);
    }
    const int bn = i8_tile_bn(kS);
    std::vector<GTile> t1 = sym_tiles(p1, bn), t2;
    for (int i = 0; i < (int)p2.size(); ++i) {
      const int tm = (p2[i].M + 127) / 128, tn = (p2[i].N + bn - 1) / bn;
      for_tiles(tm, tn, [&](int mb, int nb) { t2.push_back(GTile{i, mb, nb, 0, p2[i].K / 64, 0}); });
    }
    std::sort(sa.begin(), sa.end(), [](const GSlab& x, const GSlab& y) { return x.row0 < y.row0; });
    const std::vector<RChunk> ch = row_chunks(list, false);
    const size_t o_sa = st.put(sa), o_p1 = st.put(p1), o_p2 = st.put(p2), o_t1 = st.put(t1), o_t2 = st.put(t2);
    const size_t o_ch = st.put(ch), o_er = st.put(erp), o_sl = st.put(slot);
    const int nsa = (int)sa.size(), n1 = (int)t1.size(), n2 = (int)t2.size();
    const std::vector<int> pl = slice_plan(sa);
    const size_t o_pl = st.put(pl);
    const int bl = pl.back();
    const unsigned nch = (unsigned)ch.size();
    const double ops1 = tile_ops(t1, 2), ops2 = tile_ops(t2, 1);
    r.launches += 4;
    r.gemms += 2;
    r.ops.push_back([=]() {
      I8Slices out{};
      for (int q = 0; q < kS; ++q) {
        out.re[q] = slice_plane(0, q);
        out.im[q] = slice_plane(1, q);
      }
      out.exp = aexp();
      out.ld = pitch_;
      launch_slice_rows_grouped<double>(kS, dev<GSlab>(o_sa), nsa, rows_, out, false, stream_,
                                        SlicePlan{dev<int>(o_pl), bl});
      I8Term t[2];
      for (int q = 0; q < kS; ++q) {
        t[0].a[q] = t[0].b[q] = out.re[q];
        t[1].a[q] = t[1].b[q] = out.im[q];
      }
      size_t pi = prof_begin();
      launch_gemm_i8_grouped<double>(kS, t, 2, pitch_, rows_, rows_, aexp(), aexp(), dev<GProblem>(o_p1),
                                     dev<GTile>(o_t1), n1, (int*)err_.p, timeout_ms_, stream_);
      prof_end(pi, ops1 * kS * (kS + 1) / 2, ops1, kTagDrift);
      for (int q = 0; q < kS; ++q) {
        t[0].a[q] = out.re[q];
        t[0].b[q] = out.im[q];
      }
      pi = prof_begin();
      launch_gemm_i8_grouped<double>(kS, t, 1, pitch_, rows_, rows_, aexp(), aexp(), dev<GProblem>(o_p2),
                                     dev<GTile>(o_t2), n2, (int*)err_.p, timeout_ms_, stream_);
      prof_end(pi, ops2 * kS * (kS + 1) / 2, ops2, kTagDrift);
      kb_drift<<<nch, 256, 0, stream_>>>(dev<const double*>(o_er), A(kV), A(kW), dev<RChunk>(o_ch),
                                         (const BWalk*)d_walks_.p, dev<int>(o_sl), (double*)drift_buf_.p);
      FX_LAUNCH_CHECK();
    });
  }

  // D_re / D_im = (P_re, P_im) B^T per walk (two problems per walk, A rows side by side);
  // psym: both planes of P symmetric.
  void complex_by_real(Staging& st, Rec& r, const std::vector<int>& list, int pre, int pim, int bt, int dre,
                       int dim, int tri, bool psym) {
    std::vector<GSlab> sa, sb;
    std::vector<GProblem> pr;
    for (int w : list) {
      const BWalk& b = walks_[w];
      const int dg = (split_ & 2) ? 0 : kNoDiag;
      sa.push_back(GSlab{A(pre) + b.off, nullptr, b.np, b.np, b.np, (int)(2 * b.row0), dg});
      sa.push_back(GSlab{A(pim) + b.off, nullptr, b.np, b.np, b.np, (int)(2 * b.row0 + b.np), dg});
      sb.push_back(GSlab{A(bt) + b.off, nullptr, b.np, b.np, b.np, (int)b.row0, dg});
      GProblem p{};
      p.b_row0 = (int)b.row0;
      p.M = p.N = p.K = b.np;
      p.alpha = 1.0;
      p.ldc = p.ldd = b.np;
      if (split_ & 2) {
        p.split = psym ? 2 : 1;
        p.Btm = A(bt) + b.off;
        p.ldam = p.ldbm = b.np;
      }
      p.a_row0 = (int)(2 * b.row0);
      p.D = A(dre) + b.off;
      p.Am = A(pre) + b.off;
      pr.push_back(p);
      p.a_row0 = (int)(2 * b.row0 + b.np);
      p.D = A(dim) + b.off;
      p.Am = A(pim) + b.off;
      pr.push_back(p);
    }
    grouped(st, r, sa, &sb, pr, false, tri, (split_ & 2) != 0);
  }

  // Blocked right-looking Cholesky of the listed walks' G (in arena g), 128-wide steps.
  void cholesky(Staging& st, Rec& r, int g, const std::vector<int>& list) {
    int jmax = 0;
    for (int w : list) jmax = std::max(jmax, walks_[w].np / kNb);
    for (int j = 0; j < jmax; ++j) {
      std::vector<GChol> jobs;
      std::vector<GSlab> sa21, sb_l;
      std::vector<GProblem> p21, p22;
      for (int w : list) {
        const BWalk& b = walks_[w];
        if (b.np <= j * kNb) continue;
        double* G = A(g) + b.off;
        const int64_t k0 = (int64_t)j * kNb;
        jobs.push_back(GChol{G, b.np, k0, kNb, w, linv(w) + k0 * kNb, linvT(w) + k0 * kNb});
        const int rest = b.np - (j + 1) * kNb;
        if (rest <= 0) continue;
        double* G21 = G + (k0 + kNb) * b.np + k0;
        // L21 = G21 Linv^T: A = G21 (rest x 128), Bt = Linv (128 x 128)
        sa21.push_back(GSlab{G21, nullptr, b.np, rest, kNb, (int)b.row0, kNoDiag});
        sb_l.push_back(GSlab{linv(w) + k0 * kNb, nullptr, kNb, kNb, kNb, (int)b.row0, kNoDiag});
        GProblem p{};
        p.a_row0 = p.b_row0 = (int)b.row0;
        p.M = rest;
        p.N = kNb;
        p.K = kNb;
        p.alpha = 1.0;
        p.D = G21;
        p.ldd = b.np;
        p21.push_back(p);
        // G22 -= L21 L21^T (symmetric)
        GProblem q{};
        q.a_row0 = q.b_row0 = (int)b.row0;
        q.M = q.N = rest;
        q.K = kNb;
        q.sym = 1;
        q.alpha = -1.0;
        q.beta = 1.0;
        q.C = G21 + kNb;
        q.ldc = b.np;
        q.D = G21 + kNb;
        q.ldd = b.np;
        p22.push_back(q);
      }
      const size_t o_j = st.put(jobs);
      const int nj = (int)jobs.size();
      r.launches += 1;
      r.ops.push_back([=]() { launch_potrf_inv_grouped<double>(dev<GChol>(o_j), nj, (int*)err_.p, walk_err(), stream_); });
      if (p21.empty()) continue;
      grouped(st, r, sa21, &sb_l, p21, false, 0);
      // the updated G21 (= L21) is both factors of the trailing update
      std::vector<GSlab> sl;
      for (size_t i = 0; i < p21.size(); ++i) sl.push_back(GSlab{p21[i].D, nullptr, p21[i].ldd, p21[i].M, kNb, p21[i].a_row0, kNoDiag});
      grouped(st, r, sl, nullptr, p22, true, 0);
    }
  }

  // X = L^-1 (arena x) and X^T (arena xt) from L^T (arena lt) and the inverted 128 x 128
  // diagonal blocks, by recursive halving: for a block range split into [first | second],
  //   X21 = -X22 L21 X11,
  // computed as T = X22 L21 (X22 lower triangular: K steps bounded per tile row) and
  // X21 = -T X11 (X11 lower triangular; its transpose X11^T is read by rows), whose epilogue
  // also stores X21^T.  All nodes of one depth, over all walks, form one grouped launch pair,
  // deepest first, so a walk of J blocks takes 2 ceil(log2 J) launches.
  struct Node {
    int w, r0, h1, r1, h2;   // first block [r0, r0 + h1), second block [r1, r1 + h2), elements
  };
  void collect(int w, int a, int b, int depth, std::vector<std::vector<Node>>& lv) {
    if (b - a <= 1) return;
    const int mid = a + (b - a) / 2;
    if ((int)lv.size() <= depth) lv.resize(depth + 1);
    lv[depth].push_back(Node{w, a * kNb, (mid - a) * kNb, mid * kNb, (b - mid) * kNb});
    collect(w, a, mid, depth + 1, lv);
    collect(w, mid, b, depth + 1, lv);
  }
  void inverse(Staging& st, Rec& r, int lt, int x, int xt, int scratch, const std::vector<int>& list) {
    const int W = count();
    std::vector<int64_t> loff(W);
    for (int w = 0; w < W; ++w) loff[w] = (int64_t)walks_[w].row0 * kNb;
    const std::vector<RChunk> ch = row_chunks(list, false);
    const size_t o_lo = st.put(loff), o_ch = st.put(ch);
    double* X = A(x);
    double* XT = A(xt);
    const double* Li = (const double*)linv_.p;
    const double* LiT = (const double*)linv_.p + (size_t)rows_ * kNb;
    const unsigned nch = (unsigned)ch.size();
    r.launches += 2;
    r.ops.push_back([=]() {
      kb_init_inverse<<<nch, 256, 0, stream_>>>(X, Li, dev<RChunk>(o_ch), (const BWalk*)d_walks_.p, dev<int64_t>(o_lo));
      FX_LAUNCH_CHECK();
      kb_init_inverse<<<nch, 256, 0, stream_>>>(XT, LiT, dev<RChunk>(o_ch), (const BWalk*)d_walks_.p, dev<int64_t>(o_lo));
      FX_LAUNCH_CHECK();
    });
    std::vector<std::vector<Node>> lv;
    for (int w : list) collect(w, 0, walks_[w].np / kNb, 0, lv);
    for (int d = (int)lv.size() - 1; d >= 0; --d) {
      std::vector<GSlab> sa, sb, sa2, sb2;
      std::vector<GProblem> pa, pb;
      for (const Node& nd : lv[d]) {
        const BWalk& b = walks_[nd.w];
        const int64_t np = b.np;
        double* T = A(scratch) + b.off + (int64_t)nd.r1 * np + nd.r0;   // h2 x h1, ld np
        // T = X22 L21: A = X22 (rows r1.., cols r1..), Bt = L21^T = rows r0.. of L^T, cols r1..
        sa.push_back(GSlab{X + b.off + (int64_t)nd.r1 * np + nd.r1, nullptr, np, nd.h2, nd.h2,
                           (int)(b.row0 + nd.r1), kNoDiag});
        sb.push_back(GSlab{A(lt) + b.off + (int64_t)nd.r0 * np + nd.r1, nullptr, np, nd.h1, nd.h2,
                           (int)(b.row0 + nd.r0), kNoDiag});
        GProblem p{};
        p.a_row0 = (int)(b.row0 + nd.r1);
        p.b_row0 = (int)(b.row0 + nd.r0);
        p.M = nd.h2;
        p.N = nd.h1;
        p.K = nd.h2;
        p.alpha = 1.0;
        p.D = T;
        p.ldd = np;
        pa.push_back(p);
        // X21 = -T X11: A = T, Bt = X11^T (rows r0.. of X^T, cols r0..); also store X21^T
        sa2.push_back(GSlab{T, nullptr, np, nd.h2, nd.h1, (int)(b.row0 + nd.r1), kNoDiag});
        sb2.push_back(GSlab{XT + b.off + (int64_t)nd.r0 * np + nd.r0, nullptr, np, nd.h1, nd.h1,
                            (int)(b.row0 + nd.r0), kNoDiag});
        GProblem q{};
        q.a_row0 = (int)(b.row0 + nd.r1);
        q.b_row0 = (int)(b.row0 + nd.r0);
        q.M = nd.h2;
        q.N = nd.h1;
        q.K = nd.h1;
        q.alpha = -1.0;
        q.D = X + b.off + (int64_t)nd.r1 * np + nd.r0;
        q.ldd = np;
        q.Dt = XT + b.off + (int64_t)nd.r0 * np + nd.r1;
        q.ldt = np;
        pb.push_back(q);
      }
      grouped(st, r, sa, &sb, pa, false, 3);
      grouped(st, r, sa2, &sb2, pb, false, 2);
    }
  }
};

// ---- interface used by the per-walk engine (fx_engine.cu) for structured walks
BatchPipeline* batch_pipeline_create(int64_t n, int dtype) { return new BatchPipeline({n}, dtype); }
void batch_pipeline_destroy(BatchPipeline* p) { delete p; }
void batch_pipeline_run(BatchPipeline* p, const void* dX, const void* dpsi0, void* dpsi, void* dU,
                        const PipeOpts& o, cudaStream_t s) {
  p->set_selector(o.selector);
  const void* x[1] = {dX};
  const void* p0[1] = {dpsi0};
  void* p1[1] = {dpsi};
  void* u[1] = {dU};
  p->set_profile(o.profile);
  p->set_timeout(o.timeout_ms);
  p->set_inject_stall(o.inject_stall);
  p->set_form(o.form == FX_FORM_MIXED ? 1 : 0, o.sq_n4, o.sq_n3, o.pade_slices, o.newton_slices);
  p->set_solve(o.solve);
  p->set_approx(o.approx);
  p->set_drift(o.drift);
  p->run(x, p0, p1, u, s);
}
const std::vector<ProdRecord>& batch_pipeline_products(const BatchPipeline* p) { return p->prod_list(); }
std::vector<double> batch_pipeline_drift(const BatchPipeline* p) { return p->drift_curve(0); }
void batch_pipeline_spectral(const BatchPipeline* p, double* rho_lanczos, double* rho_up) {
  p->spectral(0, rho_lanczos, rho_up);
}
void batch_pipeline_stats(const BatchPipeline* p, fx_stats* st) {
  p->walk_stats(0, st);
  double f[8];
  int pm, ps, cm, cs, oc;
  p->details(0, f, &pm, &ps, &cm, &cs, &oc);
  st->selector = p->selector();
  st->sel_outcome = oc;
  st->plain_m = pm;
  st->plain_s = ps;
  st->gemm_launches = p->gemm_launches();
  st->launches = p->launches();
  st->flops = p->flops();
}

}  // namespace fx

// ================================================================== C ABI
struct fx_batch {
  std::unique_ptr<fx::BatchPipeline> p;
  int dtype = FX_C64;
  std::vector<int64_t> ns;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  double ms = 0;
  std::vector<void*> h_in;   // device staging of host runs (X, psi0, psi per walk)
  fx::HostStage stage;       // page-locked chunks for the copies of the host matrices
  int sq_n4 = fx::kMixedN4, sq_n3 = fx::kMixedN3;   // mixed-form slice schedule
  int pade_slices = fx::kMixedPade;
  int newton_slices = fx::kMixedNewton;
  std::string last_error;
};

namespace {
std::mutex g_batch_mu;
std::string g_batch_err;
int bfail(fx_batch_handle b, const fx::Error& e) {
  if (b) b->last_error = e.msg;
  std::lock_guard<std::mutex> lk(g_batch_mu);
  g_batch_err = e.msg;
  return e.code;
}
template <typename F>
int bguard(fx_batch_handle b, F&& f) {
  try {
    f();
    return FX_OK;
  } catch (const fx::Error& e) {
    return bfail(b, e);
  } catch (const std::bad_alloc&) {
    return bfail(b, fx::Error{FX_ERR_NOMEM, "host allocation failed"});
  } catch (const std::exception& e) {
    return bfail(b, fx::Error{FX_ERR_CUDA, e.what()});
  }
}
}  // namespace

extern "C" {

int fx_batch_create(size_t count, const int64_t* n, int dtype, fx_batch_handle* out) {
  if (!out || (!n && count)) return bfail(nullptr, fx::Error{FX_ERR_VALUE, "null argument"});
  *out = nullptr;
  if (dtype != FX_C64 && dtype != FX_C128)
    return bfail(nullptr, fx::Error{FX_ERR_TYPE, "batched walks are complex64 or complex128"});
  if (count == 0 || count > 65536) return bfail(nullptr, fx::Error{FX_ERR_VALUE, "batch size must be 1..65536"});
  if (!fx_device_ok()) return bfail(nullptr, fx::Error{FX_ERR_NODEV, "no sm_100 CUDA device"});
  fx_batch_handle b = new (std::nothrow) fx_batch();
  if (!b) return bfail(nullptr, fx::Error{FX_ERR_NOMEM, "host allocation failed"});
  const int rc = bguard(b, [&] {
    b->dtype = dtype;
    b->ns.assign(n, n + count);
    FX_CUDA(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    FX_CUDA(cudaEventCreate(&b->ev0));
    FX_CUDA(cudaEventCreate(&b->ev1));
    b->p.reset(new fx::BatchPipeline(b->ns, dtype));
  });
  if (rc != FX_OK) {
    fx_batch_destroy(b);
    return rc;
  }
  *out = b;
  (void)0;
  return FX_OK;
}

int fx_batch_destroy(fx_batch_handle b) {
  if (!b) return FX_OK;
  b->p.reset();
  for (void* p : b->h_in)
    if (p) cudaFree(p);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return FX_OK;
}

int fx_batch_sample_check(fx_batch_handle b, int32_t* sampled, double* max_infidelity) {
  if (!b || !sampled || !max_infidelity) return bfail(b, fx::Error{FX_ERR_VALUE, "null argument"});
  int c = 0;
  double m = 0.0;
  b->p->sample_check(&c, &m);
  *sampled = c;
  *max_infidelity = m;
  return FX_OK;
}

int fx_batch_schedule(fx_batch_handle b, int32_t* tile_group, int32_t* tile_order, double* tuned, int32_t* ntuned) {
  if (!b || !tile_group || !tile_order) return bfail(b, fx::Error{FX_ERR_VALUE, "null argument"});
  int g = 0, o = 0;
  b->p->schedule(&g, &o);
  *tile_group = g;
  *tile_order = o;
  const auto& t = b->p->tuned();
  if (ntuned) *ntuned = (int32_t)t.size();
  if (tuned)
    for (size_t i = 0; i < t.size(); ++i)
      for (int k = 0; k < 3; ++k) tuned[3 * i + k] = t[i][k];
  return FX_OK;
}

int fx_batch_set_option(fx_batch_handle b, int key, double value) {
  if (!b) return bfail(nullptr, fx::Error{FX_ERR_VALUE, "null handle"});
  switch (key) {
    case FX_BATCH_OPT_GRAPH: b->p->set_graph(value != 0.0); return FX_OK;
    case FX_BATCH_OPT_TIMEOUT_MS:
      if (value < 1) return bfail(b, fx::Error{FX_ERR_VALUE, "timeout must be >= 1 ms"});
      b->p->set_timeout((unsigned)value);
      return FX_OK;
    case FX_BATCH_OPT_FORCE_M: b->p->force((int)value, -1); return FX_OK;
    case FX_BATCH_OPT_SELECTOR:
      if (value != 0 && value != 1 && value != 2 && value != 3)
        return bfail(b, fx::Error{FX_ERR_VALUE,
                                  "selector must be 0 (plain), 1 (certified), 2 (learned) or 3 (estimated)"});
      b->p->set_selector((int)value);
      return FX_OK;
    case FX_BATCH_OPT_ANALYZE_ONLY: b->p->set_analyze_only(value != 0.0); return FX_OK;
    case FX_BATCH_OPT_AUTOTUNE: b->p->set_autotune(value != 0.0); return FX_OK;
    case FX_BATCH_OPT_SAMPLE_WALKS:
      if (value < 0 || value > 64) return bfail(b, fx::Error{FX_ERR_VALUE, "sampled walks must be 0..64"});
      b->p->set_sample_walks((int)value);
      return FX_OK;
    case FX_BATCH_OPT_TILE_GROUP: {
      int g = 0, o = 0;
      b->p->schedule(&g, &o);
      if (value != 4 && value != 8 && value != 16)
        return bfail(b, fx::Error{FX_ERR_VALUE, "tile group must be 4, 8 or 16"});
      b->p->set_schedule((int)value, o);
      return FX_OK;
    }
    case FX_BATCH_OPT_TILE_ORDER: {
      int g = 0, o = 0;
      b->p->schedule(&g, &o);
      if (value != 0 && value != 1) return bfail(b, fx::Error{FX_ERR_VALUE, "tile order must be 0 or 1"});
      b->p->set_schedule(g, (int)value);
      return FX_OK;
    }
    case FX_BATCH_OPT_DIAG_SPLIT:
      if (value < 0 || value > 15 || value != (double)(int)value)
        return bfail(b, fx::Error{FX_ERR_VALUE, "diagonal split must be a mask of 1, 2, 4 and 8"});
      b->p->set_diag_split((int)value);
      return FX_OK;
    case FX_BATCH_OPT_FORM:
      if (value != FX_FORM_PLAIN && value != FX_FORM_MIXED)
        return bfail(b, fx::Error{FX_ERR_VALUE, "batch form must be FX_FORM_PLAIN or FX_FORM_MIXED"});
      b->p->set_form(value == FX_FORM_MIXED ? 1 : 0, b->sq_n4, b->sq_n3, b->pade_slices, b->newton_slices);
      return FX_OK;
    case FX_BATCH_OPT_SQ_N4:
    case FX_BATCH_OPT_SQ_N3: {
      if (value < 0 || value > 64) return bfail(b, fx::Error{FX_ERR_VALUE, "squaring counts must be 0..64"});
      (key == FX_BATCH_OPT_SQ_N4 ? b->sq_n4 : b->sq_n3) = (int)value;
      b->p->set_form(b->p->form(), b->sq_n4, b->sq_n3, b->pade_slices, b->newton_slices);
      return FX_OK;
    }
    case FX_BATCH_OPT_PADE_SLICES:
      if (value != 3 && value != 4 && value != 5)
        return bfail(b, fx::Error{FX_ERR_VALUE, "Pade slice count must be 3, 4 or 5"});
      b->pade_slices = (int)value;
      b->p->set_form(b->p->form(), b->sq_n4, b->sq_n3, b->pade_slices, b->newton_slices);
      return FX_OK;
    case FX_BATCH_OPT_SOLVE:
      if (value != 0 && value != 1 && value != 2)
        return bfail(b, fx::Error{FX_ERR_VALUE, "solve must be 0 (by form and size), 1 or 2"});
      b->p->set_solve((int)value);
      return FX_OK;
    case FX_BATCH_OPT_NEWTON_SLICES:
      if (value != 3 && value != 4 && value != 5)
        return bfail(b, fx::Error{FX_ERR_VALUE, "Newton slice count must be 3, 4 or 5"});
      b->newton_slices = (int)value;
      b->p->set_form(b->p->form(), b->sq_n4, b->sq_n3, b->pade_slices, b->newton_slices);
      return FX_OK;
    case FX_BATCH_OPT_DRIFT: b->p->set_drift(value != 0.0); return FX_OK;
    case FX_BATCH_OPT_APPROX:
      if (value != 0 && value != 1)
        return bfail(b, fx::Error{FX_ERR_VALUE, "approximant must be 0 (Pade) or 1 (Chebyshev)"});
      b->p->set_approx((int)value);
      return FX_OK;
  }
  return bfail(b, fx::Error{FX_ERR_VALUE, "unknown batch option"});
}

int fx_batch_walk_device(fx_batch_handle b, const void* const* dX, const void* const* dpsi0, void* const* dpsi,
                         void* stream) {
  if (!b || !dX || !dpsi0 || !dpsi) return FX_ERR_VALUE;
  return bguard(b, [&] {
    cudaStream_t s = stream ? (cudaStream_t)stream : b->stream;
    FX_CUDA(cudaEventRecord(b->ev0, s));
    b->p->run(dX, dpsi0, dpsi, nullptr, s);
    FX_CUDA(cudaEventRecord(b->ev1, s));
    FX_CUDA(cudaEventSynchronize(b->ev1));
    float ms = 0;
    FX_CUDA(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
    b->ms = ms;
  });
}

int fx_batch_walk_host(fx_batch_handle b, const void* const* X, const void* const* psi0, void* const* psi) {
  if (!b || !X || !psi0 || !psi) return FX_ERR_VALUE;
  return bguard(b, [&] {
    const size_t W = b->ns.size();
    const size_t es = b->dtype == FX_C64 ? 8 : 16;
    if (b->h_in.empty()) {
      b->h_in.assign(3 * W, nullptr);
      for (size_t w = 0; w < W; ++w) {
        const size_t n = (size_t)b->ns[w];
        fx::dev_malloc(&b->h_in[w], n * n * es);
        fx::dev_malloc(&b->h_in[W + w], n * es);
        fx::dev_malloc(&b->h_in[2 * W + w], n * es);
      }
    }
    for (size_t w = 0; w < W; ++w) {
      const size_t n = (size_t)b->ns[w];
      b->stage.h2d(b->h_in[w], X[w], n * n * es, b->stream);
      FX_CUDA(cudaMemcpyAsync(b->h_in[W + w], psi0[w], n * es, cudaMemcpyHostToDevice, b->stream));
    }
    b->p->run((const void* const*)b->h_in.data(), (const void* const*)(b->h_in.data() + W),
              (void* const*)(b->h_in.data() + 2 * W), nullptr, b->stream);
    for (size_t w = 0; w < W; ++w) {
      const size_t n = (size_t)b->ns[w];
      FX_CUDA(cudaMemcpyAsync(psi[w], b->h_in[2 * W + w], n * es, cudaMemcpyDeviceToHost, b->stream));
    }
    FX_CUDA(cudaStreamSynchronize(b->stream));
  });
}

int fx_batch_force_selection(fx_batch_handle b, const int32_t* m, const int32_t* s) {
  if (!b || (m && !s)) return bfail(b, fx::Error{FX_ERR_VALUE, "null argument"});
  if (m) {
    for (size_t w = 0; w < b->ns.size(); ++w) {
      const int mw = m[w];
      if (mw > 0 && mw != 3 && mw != 5 && mw != 7 && mw != 9 && mw != 13)
        return bfail(b, fx::Error{FX_ERR_VALUE, "forced Pade degree must be 3, 5, 7, 9 or 13"});
      if (mw > 0 && (s[w] < 0 || s[w] > 60)) return bfail(b, fx::Error{FX_ERR_VALUE, "forced s must be 0..60"});
    }
    std::vector<int> mm(m, m + b->ns.size()), ss(s, s + b->ns.size());
    b->p->force_each(mm.data(), ss.data());
  } else {
    b->p->force_each(nullptr, nullptr);
  }
  return FX_OK;
}

int fx_batch_spectral(fx_batch_handle b, double* rho_lanczos, double* rho_up) {
  if (!b || !rho_lanczos || !rho_up) return bfail(b, fx::Error{FX_ERR_VALUE, "null argument"});
  for (size_t w = 0; w < b->ns.size(); ++w) b->p->spectral((int)w, rho_lanczos + w, rho_up + w);
  return FX_OK;
}

int fx_batch_drift(fx_batch_handle b, int64_t w, double* out, int32_t cap, int32_t* count) {
  if (!b || !count || (cap > 0 && !out)) return bfail(b, fx::Error{FX_ERR_VALUE, "null argument"});
  if (w < 0 || w >= (int64_t)b->ns.size()) return bfail(b, fx::Error{FX_ERR_VALUE, "walk index out of range"});
  const std::vector<double> v = b->p->drift_curve((int)w);
  for (int32_t i = 0; i < cap && i < (int32_t)v.size(); ++i) out[i] = v[i];
  *count = (int32_t)v.size();
  return FX_OK;
}

int fx_chebyshev_plan(double rho, double tol, int32_t* s, int32_t* degree, int32_t* baby, int32_t* cost) {
  if (!s || !degree || !baby || !cost) return bfail(nullptr, fx::Error{FX_ERR_VALUE, "null argument"});
  if (!(rho >= 0.0) || !std::isfinite(rho) || !(tol > 0.0))
    return bfail(nullptr, fx::Error{FX_ERR_VALUE, "the plan needs a finite rho >= 0 and tol > 0"});
  const fx::ChebPlan p = fx::cheb_plan(rho, tol);
  if (!p.ok) return bfail(nullptr, fx::Error{FX_ERR_VALUE, "no plan: rho / 2^60 is above 1024"});
  *s = p.s;
  *degree = p.degree;
  *baby = p.baby;
  *cost = p.cost;
  return FX_OK;
}

int fx_batch_selection(fx_batch_handle b, int32_t* m, int32_t* s) {
  if (!b || !m || !s) return FX_ERR_VALUE;
  for (int w = 0; w < b->p->count(); ++w) b->p->selection(w, &m[w], &s[w]);
  return FX_OK;
}

int fx_batch_info(fx_batch_handle b, double* ms, double* flops, int32_t* launches) {
  if (!b) return FX_ERR_VALUE;
  if (ms) *ms = b->ms;
  if (flops) *flops = b->p->flops();
  if (launches) *launches = b->p->launches();
  return FX_OK;
}

int fx_batch_details(fx_batch_handle b, double* features, int32_t* plain_m, int32_t* plain_s, int32_t* cert_m,
                     int32_t* cert_s, int32_t* outcome) {
  if (!b || !features || !plain_m || !plain_s || !cert_m || !cert_s || !outcome)
    return bfail(b, fx::Error{FX_ERR_VALUE, "null argument"});
  for (int w = 0; w < b->p->count(); ++w) {
    int pm, ps, cm, cs, oc;
    b->p->details(w, features + 8 * w, &pm, &ps, &cm, &cs, &oc);
    plain_m[w] = pm;
    plain_s[w] = ps;
    cert_m[w] = cm;
    cert_s[w] = cs;
    outcome[w] = oc;
  }
  return FX_OK;
}

int fx_selector_set_weights(const float* w, int64_t n) {
  try {
    if (!w || n != fx_mlp_param_count())
      throw fx::Error{FX_ERR_VALUE, "selector weights: expected " + std::to_string(fx_mlp_param_count()) + " floats"};
    std::lock_guard<std::mutex> lk(fx::g_sel_mu);
    int dev = -1;
    FX_CUDA(cudaGetDevice(&dev));
    if (fx::g_sel_weights && fx::g_sel_device != dev) {
      cudaFree(fx::g_sel_weights);
      fx::g_sel_weights = nullptr;
    }
    if (!fx::g_sel_weights) FX_CUDA(cudaMalloc((void**)&fx::g_sel_weights, sizeof(float) * n));
    fx::g_sel_device = dev;
    FX_CUDA(cudaMemcpy(fx::g_sel_weights, w, sizeof(float) * n, cudaMemcpyHostToDevice));
  } catch (const fx::Error& e) {
    return bfail(nullptr, e);
  }
  return FX_OK;
}

const char* fx_batch_last_error(fx_batch_handle b) {
  if (b) return b->last_error.c_str();
  std::lock_guard<std::mutex> lk(g_batch_mu);
  return g_batch_err.c_str();
}

}  // extern "C"
