// Matrix product on the int8 tensor cores (tcgen05.mma kind::i8) with EXACT accumulation:
// an Ozaki-style splitting (Ozaki, Ogita, Oishi, Rump 2012, "Error-free transformations of
// matrix multiplication by using fast routines of matrix multiplication").
//
// Every row i of the left factor A (and every row j of the transposed right factor Bt) is
// scaled by a power of two 2^-e so that |x| < 127/128, rounded to the nearest multiple of
// 2^-7S (unbiased -- truncation toward zero biases every product coherently) and cut into S
// signed balanced base-128 digits:
//     x = sum_{p=1..S} s_p 2^(-7p) + r,   s_1 in [-127, 127], s_p in [-64, 63],  |r| <= 2^-(7S+1).
// The product sum_k x_ik y_jk is assembled from the slice products with p + q <= S + 1,
// grouped by "level" l = p + q in S int32 accumulators in tensor memory (TMEM):
//     L_l = sum_{p+q=l} S_p T_q^T        (exact for K <= 32768)
// and the epilogue forms  D = 2^(e_i + f_j - 14) * sum_l 2^(-7(l-2)) L_l  in FP64 before the
// single rounding to the output type.  There is no accumulation error; the error is the slice
// remainder (2^-(7S+1) relative to the row maximum) and the final rounding.  The FP32
// accumulator of the BF16 MMAs, by contrast, truncates at every K = 16 step (error linear in
// K), which the 2^s amplification of the squaring phase cannot afford.
//
//   S = 4: 10 int8 MMAs per K step (the time of 5 BF16 products), 28-bit slices, 128 x 128
//          tiles, 4 x 128 TMEM columns.
//   S = 5: 15 int8 MMAs (7.5 BF16 products), 35-bit slices for FP64 operands whose rows are
//          dominated by a few entries (the diagonal of the walk generators), 128 x 96 tiles,
//          5 x 96 TMEM columns.
//   S = 3: 6 int8 MMAs (3 BF16 products), 21-bit slices, 128 x 96 tiles, 3 x 96 TMEM columns:
//          the reduced-precision form's last squarings, whose errors are not amplified by
//          later squarings.
//
// Kernel layout: persistent CTAs, K step 64 bytes (64B swizzle), one stage = S A-slice tiles +
// S Bt-slice tiles, 3 stages; warp 0 TMA producer, warp 1 MMA issuer (B slices in pairs, one
// N = 2 x tile-width MMA for two adjacent levels), warps 2-17 epilogue (four warps per TMEM
// lane quarter, each draining a quarter of the tile columns).
// Symmetric-output mode computes only tiles touching the upper triangle and mirrors them.
// All waits are bounded (see fx_tc_common.cuh).
#include <algorithm>
#include <type_traits>

#include "fx_kernels.cuh"
#include "fx_tc_common.cuh"

namespace fx {
namespace {
using namespace tc;

constexpr int kBM = 128, kBK = 64;  // kBK in int8 elements (= bytes)
constexpr int kMaxSlices = 5;
constexpr int kEpiWarps = 16;   // epilogue warps: kEpiWarps / 4 per TMEM lane quarter
constexpr int kThreads = 64 + 32 * kEpiWarps;   // warp 0 TMA, warp 1 MMA, then the epilogue
constexpr int kMaxTerms = 2;
constexpr int kStages = 3;

template <int S>
struct I8Cfg {
  static constexpr int kBN = S == 4 ? 128 : 96;          // S levels x kBN TMEM columns <= 512
  static constexpr int kATile = kBM * kBK;                 // bytes of one A slice tile
  static constexpr int kBTile = kBN * kBK;
  static constexpr int kStage = S * (kATile + kBTile);
  static constexpr int kSmem = kStages * kStage + 1024;
};

struct I8Params {
  CUtensorMap map_a[kMaxTerms][kMaxSlices];
  CUtensorMap map_b[kMaxTerms][kMaxSlices];
  int nterms;
  int M, N, K;
  int tiles_m, tiles_n, ntiles;
  int bn;
  int sym;
  const int* aexp;   // per row of D
  const int* bexp;   // per column of D
  double alpha, beta, gamma;
  const void* C;
  int64_t ldc;
  void* D;
  int64_t ldd;
  int* err;
  unsigned long long timeout_ns;
  // grouped mode: per-tile jobs and per-problem descriptors (device memory)
  const GProblem* probs;
  const GTile* tiles;
  const double* adg;   // diagonal split: removed diagonals by stacked row
  const double* bdg;
  int skip_tile;       // diagnostics: the producer skips the first K step's loads of this tile
};

__host__ __device__ constexpr uint32_t idesc_i8(int m, int n) {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}
__device__ __forceinline__ void umma_i8(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc,
                                        uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, int* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
      "%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = (int)r[i];
}
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, int* v) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = (int)r[i];
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Tile id -> (mb, nb).  Symmetric mode enumerates, row by row, the tiles that touch the upper
// triangle: in tile row mb those with nb >= floor(mb * kBM / bn).
__device__ __forceinline__ void tile_of(const I8Params& p, int tile, int& mb, int& nb) {
  if (p.sym) {
    int r = 0, rem = tile;
    for (;;) {
      const int first = (r * kBM) / p.bn;
      const int cnt = p.tiles_n - first;
      if (rem < cnt) {
        mb = r;
        nb = first + rem;
        return;
      }
      rem -= cnt;
      ++r;
    }
  }
  constexpr int G = 8;
  const int per_group = G * p.tiles_n;
  const int g = tile / per_group;
  const int first_m = g * G;
  const int gsize = min(G, p.tiles_m - first_m);
  const int rr = tile - g * per_group;
  mb = first_m + rr % gsize;
  nb = rr / gsize;
}

// 2^k as a normal double for -1022 <= k <= 1023, +inf above, 0 below.
__device__ __forceinline__ double pow2_normal(int k) {
  return k > 1023 ? __longlong_as_double(0x7ff0000000000000ll)
                  : (k < -1022 ? 0.0 : __longlong_as_double((long long)(k + 1023) << 52));
}
// x 2^k for any k that two double exponents can sum to, as two exact power-of-two products (no
// branch and no ldexp: an ldexp fallback, though almost never needed, was evaluated for every
// element of the epilogue and cost a quarter of its time).  Equal to ldexp(x, k) whenever the
// result is a normal number; results below 2^-1022 flush to zero.
__device__ __forceinline__ double scale_pow2(double x, int k) {
  const int k1 = k >> 1;
  return x * pow2_normal(k1) * pow2_normal(k - k1);
}

// Everything a role needs to know about one output tile.
struct TileJob {
  int mb, nb;          // tile coordinates inside its problem
  int kb0, kb1;        // K steps [kb0, kb1) of kBK bytes
  int arow, brow;      // first slice row of the A / Bt tile in the (stacked) slice planes
  int M, N;            // problem extent (stores are clipped to it)
  int sym;
  int prob;            // problem index (grouped) or -1
};

// L2 prefetch of the blocks a grouped tile's epilogue reads (the C block, and the FP64 masters
// of a split problem), issued by the epilogue threads one tile ahead, while the MMAs run: the
// epilogue's loads then find them in L2.  A hint only: ranges that are not 16-byte aligned
// multiples of 16 bytes are skipped.
__device__ __forceinline__ void prefetch_l2(const void* a, int64_t bytes) {
  if ((reinterpret_cast<uintptr_t>(a) & 15) == 0 && bytes > 0 && (bytes & 15) == 0)
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a), "r"((uint32_t)bytes) : "memory");
}
template <typename TO>
__device__ __forceinline__ void prefetch_tile(const I8Params& p, int tile, int bn, int et, int nthreads) {
  const GTile t = p.tiles[tile];
  const GProblem& q = p.probs[t.prob];
  const int64_t r0 = (int64_t)t.mb * kBM, c0 = (int64_t)t.nb * bn;
  const int rows = (int)min((int64_t)kBM, (int64_t)q.M - r0), cols = (int)min((int64_t)bn, (int64_t)q.N - c0);
  if (rows <= 0 || cols <= 0) return;
  const int nc = (q.beta != 0.0 && q.C) ? rows : 0;                 // C rows (row-major)
  const int na = q.split == 2 ? cols : (q.split == 1 ? rows : 0);   // A: columns (symmetric) or rows
  const int nb = (q.split && !(q.split == 2 && q.Am == q.Btm && q.ldam == q.ldbm)) ? cols : 0;
  for (int k = et; k < nc + na + nb; k += nthreads) {
    if (k < nc) {
      prefetch_l2((const TO*)q.C + (r0 + k) * q.ldc + c0, (int64_t)cols * sizeof(TO));
    } else if (k < nc + na) {
      const int i = k - nc;
      if (q.split == 2)
        prefetch_l2((const TO*)q.Am + (c0 + i) * q.ldam + r0, (int64_t)rows * sizeof(TO));
      else
        prefetch_l2((const TO*)q.Am + (r0 + i) * q.ldam + c0, (int64_t)cols * sizeof(TO));
    } else {
      const int j = k - nc - na;
      prefetch_l2((const TO*)q.Btm + (c0 + j) * q.ldbm + r0, (int64_t)rows * sizeof(TO));
    }
  }
}

template <bool G>
__device__ __forceinline__ TileJob job_of(const I8Params& p, int tile) {
  TileJob j;
  if constexpr (G) {
    const GTile t = p.tiles[tile];
    const GProblem& q = p.probs[t.prob];
    j.mb = t.mb;
    j.nb = t.nb;
    j.kb0 = t.kb0;
    j.kb1 = t.kb1;
    j.arow = q.a_row0 + t.mb * kBM;
    j.brow = q.b_row0 + t.nb * p.bn;
    j.M = q.M;
    j.N = q.N;
    j.sym = q.sym;
    j.prob = t.prob;
  } else {
    tile_of(p, tile, j.mb, j.nb);
    j.kb0 = 0;
    j.kb1 = p.K / kBK;
    j.arow = j.mb * kBM;
    j.brow = j.nb * p.bn;
    j.M = p.M;
    j.N = p.N;
    j.sym = p.sym;
    j.prob = -1;
  }
  return j;
}

template <int S, typename TO, bool G>
__global__ void __launch_bounds__(kThreads, 1) k_gemm_i8(const __grid_constant__ I8Params p) {
  using Cf = I8Cfg<S>;
  constexpr int kBN = Cf::kBN;
  constexpr int kStage = Cf::kStage;
  const TO* Cp = (const TO*)p.C;
  TO* Dp = (TO*)p.D;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  __shared__ __align__(8) uint64_t full_bar[kStages], empty_bar[kStages];
  __shared__ __align__(8) uint64_t tfull_bar, tempty_bar, drain_bar;
  __shared__ uint32_t s_tmem;
  __shared__ volatile int s_abort;

  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
    }
    mbar_init(&tfull_bar, 1);
    mbar_init(&tempty_bar, 32 * kEpiWarps);
    mbar_init(&drain_bar, 1);
    s_abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&s_tmem)),
                 "r"(512));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = s_tmem;

  if (warp == 0) {
    if (lane == 0) {
      for (int t = 0; t < p.nterms; ++t)
        for (int q = 0; q < S; ++q) {
          prefetch_map(&p.map_a[t][q]);
          prefetch_map(&p.map_b[t][q]);
        }
      uint32_t kit = 0;
      bool ok = true;
      int issued[kStages];
      for (int s = 0; s < kStages; ++s) issued[s] = -1;
      for (int tile = blockIdx.x; tile < p.ntiles && ok; tile += gridDim.x) {
        const TileJob jb = job_of<G>(p, tile);
        for (int t = 0; t < p.nterms && ok; ++t) {
          for (int kb = jb.kb0; kb < jb.kb1; ++kb, ++kit) {
            const int s = kit % kStages;
            const uint32_t ph = (kit / kStages) & 1;
            if (!mbar_wait(&empty_bar[s], ph ^ 1, &s_abort, p.timeout_ns, p.err)) {
              ok = false;
              break;
            }
            // Failure-path diagnostics: leave one stage unfilled, so that the MMA warp's bounded
            // wait runs out and every role takes its timeout exit.
            if (tile == p.skip_tile && t == 0 && kb == jb.kb0) continue;
            uint8_t* st = smem + (size_t)s * kStage;
            mbar_expect_tx(&full_bar[s], kStage);
            for (int q = 0; q < S; ++q) {
              tma_load_2d(st + q * Cf::kATile, &p.map_a[t][q], &full_bar[s], kb * kBK, jb.arow);
              tma_load_2d(st + S * Cf::kATile + q * Cf::kBTile, &p.map_b[t][q], &full_bar[s], kb * kBK,
                          jb.brow);
            }
            issued[s] = (int)(kit / kStages);
          }
        }
      }
      if (!ok) {
        for (int s = 0; s < kStages; ++s) {
          if (issued[s] < 0) continue;
          const unsigned long long t0 = gtimer();
          while (!mbar_try(&full_bar[s], (uint32_t)issued[s] & 1))
            if (gtimer() - t0 > p.timeout_ns) break;
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      const uint32_t idesc = idesc_i8(kBM, kBN), idesc2 = idesc_i8(kBM, 2 * kBN);
      uint32_t kit = 0;
      int it = 0;
      bool ok = true, issued_any = false;
      for (int tile = blockIdx.x; tile < p.ntiles && ok; tile += gridDim.x, ++it) {
        if (!mbar_wait(&tempty_bar, (it & 1) ^ 1, &s_abort, p.timeout_ns, p.err)) break;
        tc_fence_after();
        const TileJob jb = job_of<G>(p, tile);
        bool first[S];
#pragma unroll
        for (int l = 0; l < S; ++l) first[l] = true;
        for (int t = 0; t < p.nterms && ok; ++t) {
          for (int kb = jb.kb0; kb < jb.kb1; ++kb, ++kit) {
            const int s = kit % kStages;
            const uint32_t ph = (kit / kStages) & 1;
            if (!mbar_wait(&full_bar[s], ph, &s_abort, p.timeout_ns, p.err)) {
              ok = false;
              break;
            }
            tc_fence_after();
            const uint32_t st = smem_u32(smem + (size_t)s * kStage);
            // Two B slices per instruction: slices pb and pb + 1 lie back to back in shared
            // memory and their levels pa + pb and pa + pb + 1 in adjacent TMEM column blocks, so
            // one MMA of N = 2 kBN covers both (one A read for twice the columns; 6 instructions
            // per 32 bytes of K instead of 10 at S = 4, 9 instead of 15 at S = 5).  Row pa = 0
            // writes every level first, in pairs of equal first-write state.
#pragma unroll
            for (int pa = 0; pa < S; ++pa) {
#pragma unroll
              for (int pb = 0; pb < S; pb += 2) {
                const int lvl = pa + pb;  // 0..S-1 <=> level l = 2..S+1
                if (lvl > S - 1) continue;
                const bool two = lvl + 1 <= S - 1;
                const uint32_t a_addr = st + pa * Cf::kATile;
                const uint32_t b_addr = st + S * Cf::kATile + pb * Cf::kBTile;
                const uint32_t tmem_d = tmem_base + (uint32_t)(lvl * kBN);
#pragma unroll
                for (int k32 = 0; k32 < kBK / 32; ++k32) {
                  umma_i8(tmem_d, desc_sw64(a_addr + k32 * 32), desc_sw64(b_addr + k32 * 32), two ? idesc2 : idesc,
                          first[lvl] ? 0u : 1u);
                  first[lvl] = false;
                  if (two) first[lvl + 1] = false;
                  issued_any = true;
                }
              }
            }
            umma_commit(&empty_bar[s]);
          }
        }
        if (ok) umma_commit(&tfull_bar);
      }
      if (issued_any) {
        umma_commit(&drain_bar);
        const unsigned long long t0 = gtimer();
        while (!mbar_try(&drain_bar, 0)) {
          if (gtimer() - t0 > p.timeout_ns) {
            atomicOr(p.err, kDevTimeout);
            break;
          }
        }
      }
    }
  } else {
    // kEpiWarps / 4 epilogue warps per TMEM lane quarter (warp % 4), each draining an equal share
    // of the columns in chunks of kW.
    const int q = warp & 3;
    const int half = (warp - 2) >> 2;        // this warp's share of the columns
    constexpr int kParts = kEpiWarps / 4;
    constexpr int kCols = kBN / kParts;       // columns per warp
    constexpr int kW = kEpiWarps == 16 ? 8 : 16;
    constexpr int kChunks = kCols / kW;
    static_assert(kCols % kW == 0, "epilogue chunks");
    // drain all of a warp's columns before handing TMEM back when they fit in registers: with
    // 16 epilogue warps up to 32 folded columns (the 128-column tiles of 4 slices too, whose
    // few spills cost less than an MMA warp idle for the whole epilogue: products of the
    // N = 10000 walk 167 -> 153 ms)
    constexpr bool kEarly = kCols <= (kEpiWarps == 16 ? 32 : 48);
    int it = 0;
    for (int tile = blockIdx.x; tile < p.ntiles; tile += gridDim.x, ++it) {
      if constexpr (G) {
        const int et = (int)threadIdx.x - 64;
        if (it == 0) prefetch_tile<TO>(p, tile, kBN, et, kThreads - 64);
        if (tile + (int)gridDim.x < p.ntiles) prefetch_tile<TO>(p, tile + gridDim.x, kBN, et, kThreads - 64);
      }
      if (!mbar_wait(&tfull_bar, it & 1, &s_abort, p.timeout_ns, p.err)) break;
      tc_fence_after();
      const TileJob jb = job_of<G>(p, tile);
      const bool acc = jb.kb1 > jb.kb0;   // an empty K range leaves the accumulator unwritten
      const int64_t row = (int64_t)jb.mb * kBM + q * 32 + lane;
      const bool row_ok = row < jb.M;
      // Columns col0 .. col0 + 15 of this thread's row from the folded levels x: scaling,
      // diagonal split terms, alpha / beta C / gamma I, stores.  The launch's or the problem's
      // parameters are read here, after the TMEM reads, to keep them out of the fold's registers.
      auto finish = [&](const auto& x, int64_t col0) {
        constexpr int W = (int)(sizeof(x) / sizeof(double));
        double alpha = p.alpha, beta = p.beta, gamma = p.gamma;
        const TO* Cq = Cp;
        TO* Dq = Dp;
        TO* Dt = nullptr;
        int64_t ldc = p.ldc, ldd = p.ldd, ldt = 0;
        const int* aexp = p.aexp;
        const int* bexp = p.bexp;
        int split = 0;
        const TO* Am = nullptr;
        const TO* Btm = nullptr;
        int64_t ldam = 0, ldbm = 0;
        const double* bdg = nullptr;
        double adiag = 0.0;
        if constexpr (G) {
          const GProblem& pr = p.probs[jb.prob];
          alpha = pr.alpha;
          beta = pr.beta;
          gamma = pr.gamma;
          Cq = (const TO*)pr.C;
          Dq = (TO*)pr.D;
          Dt = (TO*)pr.Dt;
          ldc = pr.ldc;
          ldd = pr.ldd;
          ldt = pr.ldt;
          aexp += pr.a_row0;
          bexp += pr.b_row0;
          split = pr.split;
          if (split) {
            Am = (const TO*)pr.Am;
            Btm = (const TO*)pr.Btm;
            ldam = pr.ldam;
            ldbm = pr.ldbm;
            bdg = p.bdg + pr.b_row0;
            adiag = p.adg[pr.a_row0 + row];
          }
        }
        const int ea = aexp[row];
        const bool same_ab = split == 2 && Am == Btm && ldam == ldbm;   // B = A: one read
        // Eight columns at a time: all loads first, then the stores (loads placed after a
        // store of the same type could not be hoisted above it).  The masters, diagonals and
        // exponents take the read-only path (D never overlaps them); C is read plainly, as D
        // may be C.  split 1: the thread's A row segment in 16-byte loads (the lanes hold
        // different rows); split 2: A symmetric, read down the columns across the lanes.
#pragma unroll
        for (int h = 0; h < W; h += 8) {
          const int64_t c0 = col0 + h;
          double arow[8];
          if (split == 1) {
            const TO* ar = Am + row * ldam + c0;
            if constexpr (sizeof(TO) == 8) {
#pragma unroll
              for (int i = 0; i < 8; i += 2) {
                const double2 t2 = __ldg(reinterpret_cast<const double2*>(ar + i));
                arow[i] = t2.x;
                arow[i + 1] = t2.y;
              }
            } else {
#pragma unroll
              for (int i = 0; i < 8; ++i) arow[i] = (double)__ldg(ar + i);
            }
          }
          double v[8];
#pragma unroll
          for (int i = 0; i < 8; ++i) {
            const int64_t col = c0 + i;
            double t = 0.0;
            if (acc) {
              const int eb = __ldg(bexp + col);
              t = scale_pow2(x[h + i], ea + eb - 14);
            }
            if (split) {
              double aij = split == 2 ? (double)__ldg(Am + col * ldam + row) : arow[i];
              const double bji = same_ab ? aij : (double)__ldg(Btm + col * ldbm + row);
              if (col == row) aij = 0.0;
              t += adiag * bji + aij * __ldg(bdg + col);
            }
            t *= alpha;
            if (beta != 0.0) t += beta * (double)Cq[row * ldc + col];
            if (col == row) t += gamma;
            v[i] = t;
          }
          if (!jb.sym) {
#pragma unroll
            for (int i = 0; i < 8; ++i) Dq[row * ldd + c0 + i] = (TO)v[i];
            if (Dt) {
#pragma unroll
              for (int i = 0; i < 8; ++i) Dt[(c0 + i) * ldt + row] = (TO)v[i];
            }
          } else {
#pragma unroll
            for (int i = 0; i < 8; ++i) {
              const int64_t col = c0 + i;
              if (col >= row) Dq[row * ldd + col] = (TO)v[i];
              if (col > row) Dq[col * ldd + row] = (TO)v[i];
            }
          }
        }
      };
      // x = sum_l 2^(-7 l) L_l of 16 columns, from the top level down, the levels read two at a
      // time (for |L_l| < 2^31 every step but the last of five levels is exact in FP64).
      auto fold = [&](uint32_t ta, auto& x) {
        constexpr int W = (int)(sizeof(x) / sizeof(double));
#pragma unroll
        for (int i = 0; i < W; ++i) x[i] = 0.0;
#pragma unroll
        for (int l = S - 1; l >= 0; l -= 2) {
          int hi[W], lo[W];
          if constexpr (W == 16) {
            tmem_ld16(ta + l * kBN, hi);
            if (l >= 1) tmem_ld16(ta + (l - 1) * kBN, lo);
          } else {
            tmem_ld8(ta + l * kBN, hi);
            if (l >= 1) tmem_ld8(ta + (l - 1) * kBN, lo);
          }
          tmem_wait_ld();
#pragma unroll
          for (int i = 0; i < W; ++i) {
            double t = x[i] * 0x1p-7 + (double)hi[i];
            if (l >= 1) t = t * 0x1p-7 + (double)lo[i];
            x[i] = t;
          }
        }
      };
      const uint32_t tq = tmem_base + ((uint32_t)(q * 32) << 16);
      if constexpr (kEarly) {
        // All of this warp's columns fit in registers once folded: drain TMEM first and hand it
        // back to the MMA warp, so that the next tile's products overlap the rest of the epilogue.
        double xv[kChunks][kW];
#pragma unroll
        for (int c = 0; c < kChunks; ++c) fold(tq + (uint32_t)((half * kChunks + c) * kW), xv[c]);
        tc_fence_before();
        mbar_arrive(&tempty_bar);
        if (row_ok) {
#pragma unroll
          for (int c = 0; c < kChunks; ++c) {
            const int64_t col0 = (int64_t)jb.nb * kBN + (half * kChunks + c) * kW;
            if (col0 < jb.N) finish(xv[c], col0);
          }
        }
      } else {
        for (int cc = half * kChunks; cc < (half + 1) * kChunks; ++cc) {
          double x[kW];
          fold(tq + (uint32_t)(cc * kW), x);
          const int64_t col0 = (int64_t)jb.nb * kBN + cc * kW;
          if (row_ok && col0 < jb.N) finish(x, col0);
        }
        tc_fence_before();
        mbar_arrive(&tempty_bar);
      }
    }
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(512));
  }
}

// ---- slicing: warp per row; the row exponent is shared by the real and imaginary planes.
//
// With the row maximum mx = m 2^e (m in [0.5, 1), e raised by one when 128 m >= 127.5), every
// x of the row becomes the integer v = rint(x 2^(7S - e)) (exact scaling by a power of two,
// one rounding: |x 2^-e - v 2^-7S| <= 2^-(7S+1)), and v is cut into digits from the top, each
// the round-to-nearest-even of what is left: d_1 = rint(v / 2^7(S-1)) in [-127, 127], then
// d_q = rint(r / 2^7(S-q)) in [-64, 64] of the remainder r.  These are the digits of the
// greedy expansion x 128 -> rint -> remainder; they are symmetric about zero, so the
// cross terms that the product leaves out (p + q > S + 1) average out instead of adding up
// along K (bottom-up digits in [-64, 63] carry a bias of -1/2 that the squarings amplify).
template <typename TI>
struct Vec4;
template <>
struct Vec4<double> {
  static __device__ __forceinline__ void load(const double* p, double v[4]) {
    const double2 a = reinterpret_cast<const double2*>(p)[0], b = reinterpret_cast<const double2*>(p)[1];
    v[0] = a.x;
    v[1] = a.y;
    v[2] = b.x;
    v[3] = b.y;
  }
};
template <>
struct Vec4<float> {
  static __device__ __forceinline__ void load(const float* p, double v[4]) {
    const float4 a = reinterpret_cast<const float4*>(p)[0];
    v[0] = a.x;
    v[1] = a.y;
    v[2] = a.z;
    v[3] = a.w;
  }
};

template <typename TI>
__device__ __forceinline__ void load4(const TI* src, int64_t k0, int64_t K, bool vec, double v[4]) {
  if (vec && k0 + 4 <= K) {
    Vec4<TI>::load(src + k0, v);
  } else {
#pragma unroll
    for (int j = 0; j < 4; ++j) v[j] = (k0 + j < K) ? (double)src[k0 + j] : 0.0;
  }
}

// Digits of four values xs[0..3] (|xs| < 2^(7S), FP64), packed one byte each (two's complement)
// into w[q] for digit q: v = rint(xs) (round half to even), then from the top
// d_q = round-half-even(r / 2^k), k = 7 (S - 1 - q), r -= d_q 2^k, the last digit the remainder.
// Rounding to an integer by adding M = 1.5 * 2^52 (the sum lies in [2^52, 2^53), where the
// spacing of doubles is 1, so the addition rounds to the nearest integer, ties to even, and the
// low 32 bits of the sum hold that integer; the classic technique of, e.g., Muller et al.,
// Handbook of Floating-Point Arithmetic): every step is exact FP64 arithmetic on the FMA pipe,
// r / 2^k and t 2^k being powers-of-two scalings of integers below 2^36.  Integer shift forms
// of the same rule kept the integer ALU busy for three quarters of the slicer's time.
__device__ __forceinline__ void cut_digits4(const double xs[4], int S, uint32_t w[kMaxSlices]) {
  constexpr double M = 0x1.8p52;
  double r[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) r[j] = (xs[j] + M) - M;
#pragma unroll
  for (int q = 0; q < kMaxSlices; ++q) {
    if (q >= S) continue;
    uint32_t d[4];
    if (q < S - 1) {
      const int k = 7 * (S - 1 - q);
      const double down = pow2_normal(-k), up = pow2_normal(k);
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const double tm = fma(r[j], down, M);
        d[j] = (uint32_t)__double2loint(tm);
        r[j] = fma(-(tm - M), up, r[j]);
      }
    } else {
#pragma unroll
      for (int j = 0; j < 4; ++j) d[j] = (uint32_t)__double2loint(r[j] + M);
    }
    w[q] = __byte_perm(__byte_perm(d[0], d[1], 0x0040), __byte_perm(d[2], d[3], 0x0040), 0x5410);
  }
}

// rre / rim: the source row (rim may be null); orow: offset of the row in the slice planes;
// NEG: also write the slices of -im (out.neg_im).
template <typename TI, bool NEG>
__device__ __forceinline__ void slice_row(const TI* rre, const TI* rim, int64_t K, int S, const I8Slices& out,
                                          int64_t orow, int lane, int64_t dcol = -1) {
  // dcol >= 0: the element at that column (the diagonal of a real plane) is left out of the
  // slices and stored to out.dg[orow]
  const bool vec = ((reinterpret_cast<uintptr_t>(rre) | reinterpret_cast<uintptr_t>(rim)) & 15) == 0;
  double mx = 0.0;
#pragma unroll 4
  for (int64_t k0 = (int64_t)lane * 4; k0 < K; k0 += 128) {
    double v[4];
    load4<TI>(rre, k0, K, vec, v);
#pragma unroll
    for (int j = 0; j < 4; ++j) mx = fmax(mx, k0 + j == dcol ? 0.0 : fabs(v[j]));
    if (rim) {
      load4<TI>(rim, k0, K, vec, v);
#pragma unroll
      for (int j = 0; j < 4; ++j) mx = fmax(mx, fabs(v[j]));
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  int e = 0;
  if (mx > 0.0) {
    const double m = frexp(mx, &e);
    if (m * 128.0 >= 127.5) e += 1;
  }
  if (lane == 0) out.exp[orow] = e;
  if (dcol >= 0 && lane == 0) out.dg[orow] = (double)rre[dcol];
  // 2^(7S - e) as one factor when it is a normal double (always, unless the row is tiny)
  const int sh = 7 * S - e;
  const bool one_factor = sh <= 1000;
  const double scale = one_factor ? ldexp(1.0, sh) : 0.0;
  // Second pass: the next step's values are loaded before this step's digits are cut, so
  // that every lane has two loads in flight.
  double cur[2][4] = {}, nxt[2][4] = {};
  int64_t k0 = (int64_t)lane * 4;
  if (k0 < K) {
    load4<TI>(rre, k0, K, vec, cur[0]);
    if (rim) load4<TI>(rim, k0, K, vec, cur[1]);
  }
  for (; k0 < K; k0 += 128) {
    if (k0 + 128 < K) {
      load4<TI>(rre, k0 + 128, K, vec, nxt[0]);
      if (rim) load4<TI>(rim, k0 + 128, K, vec, nxt[1]);
    }
#pragma unroll
    for (int plane = 0; plane < 2; ++plane) {
      const TI* src = plane == 0 ? rre : rim;
      if (!src) continue;
      double* x = cur[plane];
      uint32_t packed[kMaxSlices];
      const bool neg = NEG && plane == 1;
      double xs[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        if (plane == 0 && k0 + j == dcol) x[j] = 0.0;
        xs[j] = one_factor ? x[j] * scale : ldexp(ldexp(x[j], -e), 7 * S);
      }
      cut_digits4(xs, S, packed);
#pragma unroll
      for (int q = 0; q < kMaxSlices; ++q) {
        if (q >= S) continue;
        int8_t* dst = plane == 0 ? out.re[q] : out.im[q];
        if (dst) *reinterpret_cast<uint32_t*>(dst + orow * out.ld + k0) = packed[q];
        if (neg && out.neg_im[q]) *reinterpret_cast<uint32_t*>(out.neg_im[q] + orow * out.ld + k0) = __vneg4(packed[q]);
      }
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      cur[0][j] = nxt[0][j];
      cur[1][j] = nxt[1][j];
    }
  }
}

template <typename TI, bool NEG>
__global__ void __launch_bounds__(256, 2) k_slice_rows(const TI* re, const TI* im, int64_t ld, int64_t rows, int64_t K, int S,
                             I8Slices out) {
  const int lane = threadIdx.x & 31;
  const int64_t row = (int64_t)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  if (row >= rows) return;
  slice_row<TI, NEG>(re + row * ld, im ? im + row * ld : nullptr, K, S, out, row, lane);
}

// Grouped slicing: warp per stacked row; the slab is found by binary search on row0.
template <typename TI, bool NEG>
__global__ void __launch_bounds__(256, 2) k_slice_rows_grouped(const GSlab* slabs, int nslabs, int64_t total_rows, int S, I8Slices out) {
  const int lane = threadIdx.x & 31;
  const int64_t row = (int64_t)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  if (row >= total_rows) return;
  int lo = 0, hi = nslabs - 1;
  while (lo < hi) {   // last slab with row0 <= row
    const int mid = (lo + hi + 1) >> 1;
    if (slabs[mid].row0 <= row) lo = mid;
    else hi = mid - 1;
  }
  const GSlab sb = slabs[lo];
  const int64_t local = row - sb.row0;
  if (local < 0 || local >= sb.rows) return;
  const TI* re = (const TI*)sb.re + local * sb.ld;
  const TI* im = sb.im ? (const TI*)sb.im + local * sb.ld : nullptr;
  const int64_t dcol = (sb.diag0 != kNoDiag && out.dg && !sb.im) ? local + sb.diag0 : -1;
  slice_row<TI, NEG>(re, im, sb.K, S, out, row, lane, (dcol >= 0 && dcol < sb.K) ? dcol : -1);
}

// ---- helpers of the streaming slicing kernels below.
__device__ __forceinline__ int row_exponent(double mx) {
  int e = 0;
  if (mx > 0.0) {
    const double m = frexp(mx, &e);
    if (m * 128.0 >= 127.5) e += 1;
  }
  return e;
}
__device__ __forceinline__ double scale_for(int S, int e, bool& one) {
  const int sh = 7 * S - e;
  one = sh <= 1000;
  return one ? ldexp(1.0, sh) : 0.0;
}

// ---- grouped slicing of wide rows in two streaming passes.  The warp-per-row kernel above
// reads a row twice (the maximum first); with thousands of 80 KB rows in flight the second read
// misses L2, and a warp per row keeps few loads in flight.  Here (1) a warp per row takes the
// row maximum with four 16-byte loads in flight per lane and writes the row exponent (and the
// split-off diagonal), and (2) a block per (row, 2048-column chunk) cuts the digits with that
// exponent: both passes stream at full occupancy.  Digits and exponents are the same as
// slice_row's.  re (and im) share one row exponent (with -im too when NEG); the diagonal of a
// single-plane slab is optionally left out (the diagonal split).
__device__ __forceinline__ int find_slab(const GSlab* slabs, int nslabs, int64_t row) {
  int lo = 0, hi = nslabs - 1;
  while (lo < hi) {   // last slab with row0 <= row
    const int mid = (lo + hi + 1) >> 1;
    if (slabs[mid].row0 <= row) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}
template <typename TI>
__global__ void __launch_bounds__(256) k_row_exp_grouped(const GSlab* slabs, int nslabs, int64_t total_rows,
                                                         I8Slices out) {
  const int lane = threadIdx.x & 31;
  const int64_t row = (int64_t)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  if (row >= total_rows) return;
  const GSlab sb = slabs[find_slab(slabs, nslabs, row)];
  const int64_t local = row - sb.row0;
  if (local < 0 || local >= sb.rows) return;
  const int64_t K = sb.K;
  const TI* re = (const TI*)sb.re + local * sb.ld;
  const TI* im = sb.im ? (const TI*)sb.im + local * sb.ld : nullptr;
  int64_t dcol = (sb.diag0 != kNoDiag && out.dg && !im) ? local + sb.diag0 : -1;
  if (dcol >= K) dcol = -1;
  const bool vec = ((reinterpret_cast<uintptr_t>(re) | reinterpret_cast<uintptr_t>(im)) & 15) == 0;
  double mx = 0.0;
#pragma unroll 4
  for (int64_t k0 = (int64_t)lane * 4; k0 < K; k0 += 128) {
    double v[4];
    load4<TI>(re, k0, K, vec, v);
#pragma unroll
    for (int j = 0; j < 4; ++j) mx = fmax(mx, k0 + j == dcol ? 0.0 : fabs(v[j]));
    if (im) {
      load4<TI>(im, k0, K, vec, v);
#pragma unroll
      for (int j = 0; j < 4; ++j) mx = fmax(mx, fabs(v[j]));
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if (lane == 0) {
    out.exp[row] = row_exponent(mx);
    if (dcol >= 0) out.dg[row] = (double)re[dcol];
  }
}
// Digit pass over a block plan: block b serves slab i with plan[i] <= b < plan[i + 1] and covers
// kPlanGroups 4-column groups of that slab's rows x K elements in row-major order, so that
// narrow rows leave no thread idle and no block searches rows; two groups' loads are in flight
// per thread before their digits are cut.
template <typename TI, bool NEG>
__global__ void __launch_bounds__(256, 3) k_slice_digits_planned(const GSlab* slabs, const int* plan, int nslabs, int S,
                                                              I8Slices out) {
  int lo = 0, hi = nslabs - 1;
  while (lo < hi) {   // last slab whose first block is <= this block
    const int mid = (lo + hi + 1) >> 1;
    if (plan[mid] <= (int)blockIdx.x) lo = mid;
    else hi = mid - 1;
  }
  const GSlab sb = slabs[lo];
  const uint32_t gpr = (uint32_t)(sb.K + 3) / 4, total = (uint32_t)sb.rows * gpr;
  const uint32_t first = ((uint32_t)blockIdx.x - (uint32_t)plan[lo]) * (uint32_t)kPlanGroups + threadIdx.x;
  const TI* re0 = (const TI*)sb.re;
  const TI* im0 = (const TI*)sb.im;
  const bool split = sb.diag0 != kNoDiag && out.dg && !im0;
  const bool vec = ((reinterpret_cast<uintptr_t>(re0) | reinterpret_cast<uintptr_t>(im0) |
                     (uintptr_t)(sb.ld * (int64_t)sizeof(TI))) & 15) == 0;
  const int64_t ld = out.ld;
  const double inv_gpr = 1.0 / (double)gpr;
  // each thread takes two adjacent groups (8 columns) per step: when they lie in one row and
  // its column offset is a multiple of 8, the digits of both go out as one 8-byte store per
  // plane; otherwise group by group
  const uint32_t end = min(first - threadIdx.x + (uint32_t)kPlanGroups, total);
#pragma unroll 1
  for (uint32_t g0 = first - threadIdx.x + 2u * threadIdx.x; g0 < end; g0 += 512) {
    double x[2][2][4] = {};
    uint32_t rr[2], kk[2];
    bool ok[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const uint32_t g = g0 + (uint32_t)h;
      ok[h] = g < end;
      uint32_t q = 0;
      if (ok[h]) {   // g / gpr through the reciprocal (the FP64 pipe has room, the integer ALU not)
        q = (uint32_t)((double)g * inv_gpr);
        if (q * gpr > g) --q;
        else if ((q + 1) * gpr <= g) ++q;
      }
      rr[h] = q;
      kk[h] = ok[h] ? 4 * (g - rr[h] * gpr) : 0;
      if (ok[h]) {
        load4<TI>(re0 + (int64_t)rr[h] * sb.ld, kk[h], sb.K, vec, x[h][0]);
        if (im0) load4<TI>(im0 + (int64_t)rr[h] * sb.ld, kk[h], sb.K, vec, x[h][1]);
      }
    }
    const bool pair = ok[1] && rr[0] == rr[1] && (kk[0] & 7) == 0;
    double sc[2];
    bool one[2];
    int ex[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      ex[h] = ok[h] ? out.exp[(int64_t)sb.row0 + rr[h]] : 0;
      sc[h] = scale_for(S, ex[h], one[h]);
    }
#pragma unroll
    for (int plane = 0; plane < 2; ++plane) {
      if (plane == 1 && !im0) continue;
      uint32_t pk[2][kMaxSlices];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        if (!ok[h]) continue;
        const int64_t dcol = split ? (int64_t)rr[h] + sb.diag0 : -1;
        double xs[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          double v = x[h][plane][j];
          if (plane == 0 && (int64_t)kk[h] + j == dcol) v = 0.0;
          xs[j] = one[h] ? v * sc[h] : ldexp(ldexp(v, -ex[h]), 7 * S);
        }
        cut_digits4(xs, S, pk[h]);
      }
#pragma unroll
      for (int q = 0; q < kMaxSlices; ++q) {
        if (q >= S) continue;
        int8_t* dst = plane == 0 ? out.re[q] : out.im[q];
        int8_t* ndst = (NEG && plane == 1) ? out.neg_im[q] : nullptr;
        if (pair) {
          const int64_t o = ((int64_t)sb.row0 + rr[0]) * ld + kk[0];
          const uint2 v = make_uint2(pk[0][q], pk[1][q]);
          if (dst) *reinterpret_cast<uint2*>(dst + o) = v;
          if (ndst) *reinterpret_cast<uint2*>(ndst + o) = make_uint2(__vneg4(v.x), __vneg4(v.y));
        } else {
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            if (!ok[h]) continue;
            const int64_t o = ((int64_t)sb.row0 + rr[h]) * ld + kk[h];
            if (dst) *reinterpret_cast<uint32_t*>(dst + o) = pk[h][q];
            if (ndst) *reinterpret_cast<uint32_t*>(ndst + o) = __vneg4(pk[h][q]);
          }
        }
      }
    }
  }
}
void make_map_u8(CUtensorMap* m, const int8_t* base, int64_t rows, int64_t cols, int64_t ld, int box_rows);

}  // namespace

// Host-side tensor maps (int8 data via the UINT8 TMA type; only bytes are moved).
namespace {
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*,
                                  CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                                  CUtensorMapFloatOOBfill);
EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* ptr = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(ptr);
  }
  return fn;
}
void make_map_u8(CUtensorMap* m, const int8_t* base, int64_t rows, int64_t cols, int64_t ld, int box_rows) {
  EncodeTiledFn enc = encode_fn();
  if (!enc) throw Error{FX_ERR_CUDA, "cuTensorMapEncodeTiled unavailable"};
  if (((uintptr_t)base & 15) != 0 || ld % 16 != 0) throw Error{FX_ERR_VALUE, "int8 TMA operand not 16-byte aligned"};
  cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)ld};
  cuuint32_t box[2] = {(cuuint32_t)kBK, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, (void*)base, dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) throw Error{FX_ERR_CUDA, "cuTensorMapEncodeTiled (int8) failed"};
}
int sm_count() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}
}  // namespace

template <typename TI>
void launch_slice_rows(int S, const TI* re, const TI* im, int64_t ld, int64_t rows, int64_t K, I8Slices out,
                       bool want_neg_im, cudaStream_t s) {
  if (S < 4 || S > kMaxSlices) throw Error{FX_ERR_VALUE, "slice count must be 4 or 5"};
  if (K % 4 != 0 || out.ld % 16 != 0) throw Error{FX_ERR_VALUE, "slice: K and ld must be multiples of 4/16"};
  if (!im) {
    for (int q = 0; q < kMaxSlices; ++q) out.im[q] = out.neg_im[q] = nullptr;
  }
  if (want_neg_im && im != nullptr)
    k_slice_rows<TI, true><<<cdiv(rows, 8), 256, 0, s>>>(re, im, ld, rows, K, S, out);
  else
    k_slice_rows<TI, false><<<cdiv(rows, 8), 256, 0, s>>>(re, im, ld, rows, K, S, out);
  FX_LAUNCH_CHECK();
}
template void launch_slice_rows<float>(int, const float*, const float*, int64_t, int64_t, int64_t, I8Slices, bool,
                                       cudaStream_t);
template void launch_slice_rows<double>(int, const double*, const double*, int64_t, int64_t, int64_t, I8Slices,
                                        bool, cudaStream_t);

std::vector<int> slice_plan(const std::vector<GSlab>& sorted) {
  std::vector<int> plan(sorted.size() + 1, 0);
  for (size_t i = 0; i < sorted.size(); ++i) {
    const int64_t groups = (int64_t)sorted[i].rows * ((sorted[i].K + 3) / 4);
    plan[i + 1] = plan[i] + (int)cdiv(groups, kPlanGroups);
  }
  return plan;
}

template <typename TI>
void launch_slice_rows_grouped(int S, const GSlab* slabs, int nslabs, int64_t total_rows, I8Slices out,
                               bool want_neg_im, cudaStream_t s, SlicePlan plan, int kind) {
  if (S < 3 || S > kMaxSlices) throw Error{FX_ERR_VALUE, "slice count must be 3, 4 or 5"};
  if (out.ld % 16 != 0) throw Error{FX_ERR_VALUE, "grouped slice: pitch must be a multiple of 16"};
  if (nslabs <= 0 || total_rows <= 0) return;
  if (kind < 0) kind = plan.plan ? 1 : 0;
  if (kind == 1) {
    if (!plan.plan) throw Error{FX_ERR_VALUE, "grouped slice: the two-pass slicer needs a block plan"};
    k_row_exp_grouped<TI><<<(unsigned)cdiv(total_rows, 8), 256, 0, s>>>(slabs, nslabs, total_rows, out);
    FX_LAUNCH_CHECK();
    if (plan.blocks <= 0) return;
    if (want_neg_im)
      k_slice_digits_planned<TI, true><<<plan.blocks, 256, 0, s>>>(slabs, plan.plan, nslabs, S, out);
    else
      k_slice_digits_planned<TI, false><<<plan.blocks, 256, 0, s>>>(slabs, plan.plan, nslabs, S, out);
    FX_LAUNCH_CHECK();
    return;
  }
  if (want_neg_im)
    k_slice_rows_grouped<TI, true><<<cdiv(total_rows, 8), 256, 0, s>>>(slabs, nslabs, total_rows, S, out);
  else
    k_slice_rows_grouped<TI, false><<<cdiv(total_rows, 8), 256, 0, s>>>(slabs, nslabs, total_rows, S, out);
  FX_LAUNCH_CHECK();
}
template void launch_slice_rows_grouped<float>(int, const GSlab*, int, int64_t, I8Slices, bool, cudaStream_t,
                                               SlicePlan, int);
template void launch_slice_rows_grouped<double>(int, const GSlab*, int, int64_t, I8Slices, bool, cudaStream_t,
                                                SlicePlan, int);


namespace {
template <int S, typename TO>
void launch_i8_cfg(I8Params& p, const I8Term* terms, int nterms, int64_t M, int64_t N, int64_t K, int64_t lda,
                   int64_t ldb, cudaStream_t s) {
  using Cf = I8Cfg<S>;
  static bool attr = false;
  if (!attr) {
    FX_CUDA(cudaFuncSetAttribute(k_gemm_i8<S, TO, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, Cf::kSmem));
    attr = true;
  }
  for (int t = 0; t < nterms; ++t)
    for (int q = 0; q < S; ++q) {
      make_map_u8(&p.map_a[t][q], terms[t].a[q], M, K, lda, kBM);
      make_map_u8(&p.map_b[t][q], terms[t].b[q], N, K, ldb, Cf::kBN);
    }
  p.tiles_m = (int)cdiv(M, kBM);
  p.tiles_n = (int)cdiv(N, Cf::kBN);
  p.bn = Cf::kBN;
  if (p.sym) {
    p.ntiles = 0;
    for (int r = 0; r < p.tiles_m; ++r) p.ntiles += p.tiles_n - (r * kBM) / Cf::kBN;
  } else {
    p.ntiles = p.tiles_m * p.tiles_n;
  }
  const int grid = p.ntiles < sm_count() ? p.ntiles : sm_count();
  k_gemm_i8<S, TO, false><<<grid, kThreads, Cf::kSmem, s>>>(p);
  FX_LAUNCH_CHECK();
}
}  // namespace

template <typename TO>
void launch_gemm_i8(int S, int64_t M, int64_t N, int64_t K, const I8Term* terms, int nterms, int64_t lda,
                    int64_t ldb, const int* aexp, const int* bexp, double alpha, double beta, const TO* C,
                    int64_t ldc, double gamma, TO* D, int64_t ldd, bool sym, int* err, unsigned timeout_ms,
                    cudaStream_t s) {
  if (nterms < 1 || nterms > kMaxTerms) throw Error{FX_ERR_VALUE, "int8 product: 1 or 2 terms"};
  if (M <= 0 || N <= 0) return;
  if (M % 16 || N % 16 || K % kBK || K <= 0 || K > 32768)
    throw Error{FX_ERR_VALUE, "int8 product: M, N multiples of 16, K multiple of 64 and <= 32768"};
  if (sym && M != N) throw Error{FX_ERR_VALUE, "symmetric product needs M == N"};
  if (beta != 0.0 && !C) throw Error{FX_ERR_VALUE, "int8 product: beta without C"};
  I8Params p;
  memset(&p, 0, sizeof(p));
  p.nterms = nterms;
  p.M = (int)M;
  p.N = (int)N;
  p.K = (int)K;
  p.sym = sym ? 1 : 0;
  p.aexp = aexp;
  p.bexp = bexp;
  p.alpha = alpha;
  p.beta = beta;
  p.gamma = gamma;
  p.C = C;
  p.ldc = ldc;
  p.D = D;
  p.ldd = ldd;
  p.err = err;
  p.timeout_ns = (unsigned long long)timeout_ms * 1000000ull;
  p.skip_tile = -1;
  if (S == 4)
    launch_i8_cfg<4, TO>(p, terms, nterms, M, N, K, lda, ldb, s);
  else if (S == 5)
    launch_i8_cfg<5, TO>(p, terms, nterms, M, N, K, lda, ldb, s);
  else
    throw Error{FX_ERR_VALUE, "slice count must be 4 or 5"};
}
template void launch_gemm_i8<float>(int, int64_t, int64_t, int64_t, const I8Term*, int, int64_t, int64_t,
                                    const int*, const int*, double, double, const float*, int64_t, double,
                                    float*, int64_t, bool, int*, unsigned, cudaStream_t);
template void launch_gemm_i8<double>(int, int64_t, int64_t, int64_t, const I8Term*, int, int64_t, int64_t,
                                     const int*, const int*, double, double, const double*, int64_t, double,
                                     double*, int64_t, bool, int*, unsigned, cudaStream_t);

int i8_tile_bn(int S) { return S == 4 ? I8Cfg<4>::kBN : S == 3 ? I8Cfg<3>::kBN : I8Cfg<5>::kBN; }

namespace {
template <int S, typename TO>
void set_i8_grouped_attr() {
  static bool attr = false;
  if (!attr) {
    FX_CUDA(cudaFuncSetAttribute(k_gemm_i8<S, TO, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 I8Cfg<S>::kSmem));
    attr = true;
  }
}
template <int S, typename TO>
void launch_i8_grouped_cfg(I8Params& p, const I8Term* terms, int nterms, int64_t pitch, int64_t a_rows,
                           int64_t b_rows, int ntiles, cudaStream_t s) {
  using Cf = I8Cfg<S>;
  set_i8_grouped_attr<S, TO>();
  for (int t = 0; t < nterms; ++t)
    for (int q = 0; q < S; ++q) {
      make_map_u8(&p.map_a[t][q], terms[t].a[q], a_rows, pitch, pitch, kBM);
      make_map_u8(&p.map_b[t][q], terms[t].b[q], b_rows, pitch, pitch, Cf::kBN);
    }
  p.bn = Cf::kBN;
  p.ntiles = ntiles;
  const int grid = ntiles < sm_count() ? ntiles : sm_count();
  k_gemm_i8<S, TO, true><<<grid, kThreads, Cf::kSmem, s>>>(p);
  FX_LAUNCH_CHECK();
}
}  // namespace

void prepare_gemm_i8_grouped(int S) {
  if (S == 3) {
    set_i8_grouped_attr<3, double>();
  } else if (S == 4) {
    set_i8_grouped_attr<4, double>();
    set_i8_grouped_attr<4, float>();
  } else {
    set_i8_grouped_attr<5, double>();
    set_i8_grouped_attr<5, float>();
  }
}

template <typename TO>
void launch_gemm_i8_grouped(int S, const I8Term* terms, int nterms, int64_t pitch, int64_t a_rows, int64_t b_rows,
                            const int* aexp, const int* bexp, const GProblem* probs, const GTile* tiles, int ntiles,
                            int* err, unsigned timeout_ms, cudaStream_t s, const double* adg, const double* bdg,
                            int skip_tile) {
  if (nterms < 1 || nterms > kMaxTerms) throw Error{FX_ERR_VALUE, "int8 product: 1 or 2 terms"};
  if (ntiles <= 0) return;
  if (pitch % kBK || pitch <= 0 || pitch > 32768) throw Error{FX_ERR_VALUE, "grouped int8 product: bad pitch"};
  I8Params p;
  memset(&p, 0, sizeof(p));
  p.nterms = nterms;
  p.aexp = aexp;
  p.bexp = bexp;
  p.err = err;
  p.timeout_ns = (unsigned long long)timeout_ms * 1000000ull;
  p.probs = probs;
  p.tiles = tiles;
  p.adg = adg;
  p.bdg = bdg;
  p.skip_tile = skip_tile;
  if (S == 3)
    launch_i8_grouped_cfg<3, TO>(p, terms, nterms, pitch, a_rows, b_rows, ntiles, s);
  else if (S == 4)
    launch_i8_grouped_cfg<4, TO>(p, terms, nterms, pitch, a_rows, b_rows, ntiles, s);
  else if (S == 5)
    launch_i8_grouped_cfg<5, TO>(p, terms, nterms, pitch, a_rows, b_rows, ntiles, s);
  else
    throw Error{FX_ERR_VALUE, "slice count must be 3, 4 or 5"};
}
template void launch_gemm_i8_grouped<float>(int, const I8Term*, int, int64_t, int64_t, int64_t, const int*,
                                            const int*, const GProblem*, const GTile*, int, int*, unsigned,
                                            cudaStream_t, const double*, const double*, int);
template void launch_gemm_i8_grouped<double>(int, const I8Term*, int, int64_t, int64_t, int64_t, const int*,
                                             const int*, const GProblem*, const GTile*, int, int*, unsigned,
                                             cudaStream_t, const double*, const double*, int);

}  // namespace fx
