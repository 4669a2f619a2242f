// Shared definitions of the B200 expm engine (internal header).
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <nvtx3/nvToolsExt.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <mutex>
#include <string>

#include "fastctqw_b200.h"

namespace fx {

// Every dense matrix of the engine is Np x Np, row-major, leading dimension Np, with
// Np = n rounded up to kPad.  The padding rows/columns hold the corresponding block of a
// function of the zero matrix (0 for powers, I for the rational approximant) so that
// products, the LU and the squarings can run on whole tiles without edge cases.
constexpr int kPad = 128;

inline int64_t pad_n(int64_t n) { return ((n + kPad - 1) / kPad) * kPad; }

struct Error {
  int code;
  std::string msg;
};

#define FX_CUDA(call)                                                                  \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess)                                                             \
      throw ::fx::Error{FX_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)}; \
  } while (0)

#define FX_LAUNCH_CHECK()                                                              \
  do {                                                                                 \
    cudaError_t e_ = cudaGetLastError();                                               \
    if (e_ != cudaSuccess)                                                             \
      throw ::fx::Error{FX_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e_)}; \
  } while (0)

inline unsigned cdiv(int64_t a, int64_t b) { return (unsigned)((a + b - 1) / b); }

// Host-side fault injection for the failure-path tests: with FX_INJECT_ALLOC_FAIL=k in the
// environment, the k-th workspace allocation (k = 0, 1, ...; counted from the first allocation
// after the variable took its current value) fails as if the device were out of memory, so the
// call returns FX_ERR_NOMEM.  Unset (or empty), nothing is injected.  No GPU fault is involved.
inline bool inject_alloc_failure() {
  static std::mutex mu;
  static std::string last;
  static long count = 0;
  const char* v = getenv("FX_INJECT_ALLOC_FAIL");
  std::lock_guard<std::mutex> lk(mu);
  if (!v || !*v) {
    last.clear();
    return false;
  }
  if (last != v) {
    last = v;
    count = 0;
  }
  return count++ == strtol(v, nullptr, 10);
}

// cudaMalloc of a workspace: FX_ERR_NOMEM (not a CUDA error) when the device has no room, or
// when FX_INJECT_ALLOC_FAIL selects this allocation.
inline void dev_malloc(void** p, size_t bytes) {
  if (inject_alloc_failure() || cudaMalloc(p, bytes) != cudaSuccess) {
    *p = nullptr;
    cudaGetLastError();
    throw Error{FX_ERR_NOMEM, "device allocation of " + std::to_string(bytes) + " bytes failed"};
  }
}

// NVTX range over a scope (named phases of a run in an Nsight timeline; free without a tool).
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

// Device-side error word shared by all kernels of a handle (bit flags).
enum DevErr : int {
  kDevTimeout = 1,     // a bounded wait gave up
  kDevNonFinite = 2,   // NaN/Inf seen in input
  kDevSingular = 4,    // zero pivot
  kDevBadArg = 8       // a kernel was handed sizes it cannot take
};

// Split of an FP32 value into up to 4 BF16 parts, hi first: v = p0 + p1 + p2 (+ p3) with
// each part the BF16 rounding of the remainder.  Three parts carry the full 24-bit
// significand of an FP32 value.
__device__ __forceinline__ void split_bf16(float v, __nv_bfloat16* parts, int nparts) {
  float r = v;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    if (i < nparts) {
      __nv_bfloat16 h = __float2bfloat16_rn(r);
      parts[i] = h;
      r = r - __bfloat162float(h);
    }
  }
}

}  // namespace fx
