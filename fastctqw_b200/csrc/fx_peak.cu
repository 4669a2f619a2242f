// Tensor-core peak of this GPU, measured (fx_tensor_peak).
//
// The roofline of the int8 product kernel needs the dense int8 rate of the part it runs on.
// This kernel measures it directly: one persistent CTA per SM issues a long chain of
// tcgen05.mma (kind::i8, or kind::f16 with BF16 operands as a cross-check against a cuBLAS BF16
// figure) on operand tiles that stay in shared memory, accumulating into tensor memory, so that
// nothing but the tensor pipe is exercised.  Shape per instruction: M = 128, N = 256 (the widest
// single-CTA form), K = 32 bytes of operands (32 int8 or 16 BF16 values).
//
// Roles: all threads fill the tiles with pseudo-random operands (random bytes for int8; BF16
// values of random sign and mantissa near 2^-7), warp 0 allocates 256 TMEM columns, and thread 0
// issues the MMAs, commits them to an mbarrier and waits for it with a deadline (globaltimer).
// On a timeout the kernel sets its error word, waits once more (again bounded) for the MMAs in
// flight and frees TMEM before returning.  The host caps the chain at 2^21 instructions (well
// under a second at any clock), far inside the 2 s deadline.
#include "fx_kernels.cuh"
#include "fx_tc_common.cuh"

namespace fx {
namespace {
using namespace tc;

constexpr int kPM = 128, kPN = 256;
constexpr int kPeakThreads = 128;
constexpr int kATileBytes = kPM * 64;   // 64-byte rows (SW64 K-major)
constexpr int kBTileBytes = kPN * 64;
// more than half of the SM's shared memory, so that exactly one CTA runs on every SM
constexpr int kPeakSmem = 160 * 1024;

__host__ __device__ constexpr uint32_t idesc_i8_peak(int m, int n) {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

// kind: 0 int8, 1 BF16.  iters MMAs of each K = 32-byte half of the 64-byte tile row.
__global__ void __launch_bounds__(kPeakThreads, 1)
    k_tensor_peak(int kind, long long iters, int* err, unsigned long long timeout_ns) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  __shared__ __align__(8) uint64_t done_bar;
  __shared__ uint32_t s_tmem;
  const int warp = threadIdx.x / 32;
  // operands that toggle like real data (the tensor pipe's power, and so its clock under the
  // power cap, depends on them)
  for (int i = threadIdx.x; i < (kATileBytes + kBTileBytes) / 4; i += blockDim.x) {
    uint32_t h = (uint32_t)i * 2654435761u + 0x9E3779B9u * (uint32_t)(blockIdx.x + 1);
    h ^= h >> 15;
    h *= 2246822519u;
    h ^= h >> 13;
    if (kind == 1) h = (h & 0x807F807Fu) | 0x3C003C00u;   // two BF16 values: sign, 7 mantissa bits
    reinterpret_cast<uint32_t*>(smem)[i] = h;
  }
  if (threadIdx.x == 0) {
    mbar_init(&done_bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                 "r"(kPN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  if (threadIdx.x == 0) {
    const uint32_t a0 = smem_u32(smem), b0 = smem_u32(smem + kATileBytes);
    const uint32_t idesc = kind == 0 ? idesc_i8_peak(kPM, kPN) : idesc_bf16(kPM, kPN, 0);
    for (long long it = 0; it < iters; ++it) {
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const uint64_t da = desc_sw64(a0 + k * 32), db = desc_sw64(b0 + k * 32);
        if (kind == 0)
          mma_i8(tmem, da, db, idesc, (it | k) ? 1u : 0u);
        else
          umma_bf16(tmem, da, db, idesc, (it | k) ? 1u : 0u);
      }
    }
    umma_commit(&done_bar);
    const unsigned long long t0 = gtimer();
    bool ok = true;
    while (!mbar_try(&done_bar, 0)) {
      if (gtimer() - t0 > timeout_ns) {
        ok = false;
        break;
      }
    }
    if (!ok) {
      atomicOr(err, kDevTimeout);
      const unsigned long long t1 = gtimer();   // one more bounded wait for the MMAs in flight
      while (!mbar_try(&done_bar, 0))
        if (gtimer() - t1 > timeout_ns) break;
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kPN));
  }
}

}  // namespace
}  // namespace fx

extern "C" {

int fx_tensor_peak(int kind, int64_t iters, double* tops, double* ms, void* stream) {
  if (!tops || !ms || (kind != 0 && kind != 1) || iters <= 0 || iters > ((int64_t)1 << 20)) {
    fx::set_product_error("fx_tensor_peak: kind must be 0 (int8) or 1 (BF16), iters in 1..2^20, non-null outputs");
    return FX_ERR_VALUE;
  }
  cudaStream_t s = (cudaStream_t)stream;
  int* d_err = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = FX_OK;
  try {
    int dev = 0, sms = 0;
    FX_CUDA(cudaGetDevice(&dev));
    FX_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    FX_CUDA(cudaFuncSetAttribute(fx::k_tensor_peak, cudaFuncAttributeMaxDynamicSharedMemorySize, fx::kPeakSmem));
    FX_CUDA(cudaMalloc(&d_err, sizeof(int)));
    FX_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int), s));
    FX_CUDA(cudaEventCreate(&e0));
    FX_CUDA(cudaEventCreate(&e1));
    FX_CUDA(cudaEventRecord(e0, s));
    fx::k_tensor_peak<<<sms, fx::kPeakThreads, fx::kPeakSmem, s>>>(kind, (long long)iters, d_err,
                                                                    2000ull * 1000ull * 1000ull);
    FX_LAUNCH_CHECK();
    FX_CUDA(cudaEventRecord(e1, s));
    FX_CUDA(cudaEventSynchronize(e1));
    int h_err = 0;
    FX_CUDA(cudaMemcpy(&h_err, d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (h_err) throw fx::Error{FX_ERR_TIMEOUT, "fx_tensor_peak: device wait timed out"};
    float t = 0.f;
    FX_CUDA(cudaEventElapsedTime(&t, e0, e1));
    // ops per instruction: 2 M N K with K = 32 int8 values or 16 BF16 values
    const double k_elems = kind == 0 ? 32.0 : 16.0;
    const double ops = (double)sms * (double)iters * 2.0 * 2.0 * fx::kPM * fx::kPN * k_elems;
    *ms = t;
    *tops = ops / (t * 1e-3) / 1e12;
  } catch (const fx::Error& e) {
    fx::set_product_error(e.msg);
    rc = e.code;
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (d_err) cudaFree(d_err);
  return rc;
}

}  // extern "C"
