// Allocation-free variant of the int8 tensor-core product (fx_product_f32_noalloc).
//
// Some callers cannot allocate device memory at the moment they want a product: code that
// runs while a memory pool owns the whole device and forbids outside cudaMalloc calls, code
// inside an allocator's own callbacks, and embedded hosts that size every GPU allocation once at
// start-up and treat any later cudaMalloc / cudaFree (and their implicit device synchronisation)
// as a failure.  fx_product_f32 allocates its slice scratch on every call, so those callers
// cannot use it.  This entry point computes the same product -- D = alpha A Bt^T + beta C +
// gamma I in FP32, through 4 int8 Ozaki slices with exact int32 accumulation on tcgen05 -- with
// its scratch in one fixed array of device memory that is part of the library image:
//
//   g_noalloc_scratch: kNoAllocScratchBytes (16 MiB), loaded on every GPU that loads the
//   library and held there until the process exits.
//
// Layout of one call in the array (every offset a multiple of 256 bytes):
//   [0, 256)               device error word (cleared at the start of every call)
//   [256, 256 + E)         row exponents of A (M ints) and of Bt (N ints), E rounded up to 256
//   then 4 slice planes of A (M x K int8 each), then 4 slice planes of Bt (N x K int8 each)
// so a call needs 256 + E + 4 (M + N) K bytes; larger sizes are rejected with FX_ERR_VALUE
// before anything is launched (M = N = K = 1024 needs 8.0 MiB, M = N = K = 1408 fits).
//
// Host code may not hand the array's name to a kernel: on the host that name is a stand-in
// symbol, not a device address.  The first call on each device therefore looks up the
// device address with cudaGetSymbolAddress while that device is current, checks the result and
// caches it per device; make that first call before any stream capture.  Later calls on the
// device reuse the cached address.
//
// All calls on a device share the one array and it keeps the previous call's contents.  Calls
// whose work overlaps on the GPU (different streams, or different host threads) race on it;
// order them on one stream or synchronise between them.
//
// Every call waits for its stream before it returns: it copies the kernel's error word (the
// bounded-wait status) back into a host variable and synchronises the stream to read it.
#include <mutex>
#include <string>

#include "fx_kernels.cuh"

namespace {

constexpr size_t kNoAllocScratchBytes = (size_t)16 << 20;
constexpr int kNoAllocSlices = 4;
constexpr int kMaxDevices = 64;
// Per-size limits checked before any size arithmetic: a row count above the array's byte size
// can never fit, and the int8 level sums are exact in int32 only up to K = 32768.
constexpr int64_t kMaxRows = (int64_t)kNoAllocScratchBytes;
constexpr int64_t kMaxK = 32768;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_scratch_mu;
unsigned char* g_scratch_addr[kMaxDevices] = {};

size_t round256(size_t b) { return (b + 255) & ~(size_t)255; }

// Device address of g_noalloc_scratch on the current device (looked up once per device).
unsigned char* scratch_on_current_device() {
  int dev = -1;
  FX_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) throw fx::Error{FX_ERR_VALUE, "device ordinal out of range"};
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    const cudaError_t rc = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (rc != cudaSuccess || !p) {
      cudaGetLastError();
      throw fx::Error{FX_ERR_CUDA, std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") +
                                       cudaGetErrorString(rc)};
    }
    g_scratch_addr[dev] = (unsigned char*)p;
  }
  return g_scratch_addr[dev];
}

}  // namespace

extern "C" {

int fx_product_f32_noalloc(int64_t M, int64_t N, int64_t K, const float* A, int64_t lda, const float* Bt,
                           int64_t ldb, float alpha, float beta, const float* C, int64_t ldc, float gamma,
                           float* D, int64_t ldd, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  try {
    if (M <= 0 || N <= 0 || K <= 0) throw fx::Error{FX_ERR_VALUE, "noalloc product: sizes must be positive"};
    if (M % 16 || N % 16 || K % 64)
      throw fx::Error{FX_ERR_VALUE, "noalloc product: M, N must be multiples of 16 and K of 64"};
    if (!A || !Bt || !D || (beta != 0.f && !C)) throw fx::Error{FX_ERR_VALUE, "noalloc product: null operand"};
    // Bound each size before the scratch arithmetic so that 4 (M + N) K cannot wrap: a huge M or
    // N would otherwise give a small product and pass the check below.  K <= 32768 is also the
    // exactness bound of the int32 level sums.
    if (M > kMaxRows || N > kMaxRows || K > kMaxK)
      throw fx::Error{FX_ERR_VALUE, "noalloc product: M, N must be at most " + std::to_string(kMaxRows) +
                                        " and K at most " + std::to_string(kMaxK) +
                                        " (the fixed scratch array holds " +
                                        std::to_string(kNoAllocScratchBytes) + " bytes)"};
    const size_t exp_bytes = round256(sizeof(int) * (size_t)(M + N));
    const size_t need = 256 + exp_bytes + (size_t)kNoAllocSlices * (size_t)(M + N) * (size_t)K;
    if (need > kNoAllocScratchBytes)
      throw fx::Error{FX_ERR_VALUE, "noalloc product: needs " + std::to_string(need) +
                                        " bytes of scratch, the fixed array holds " +
                                        std::to_string(kNoAllocScratchBytes) + " (4 (M + N) K + 4 (M + N) + 512)"};
    unsigned char* base = scratch_on_current_device();
    int* err = (int*)base;
    int* aexp = (int*)(base + 256);
    int* bexp = aexp + M;
    int8_t* sl = (int8_t*)(base + 256 + exp_bytes);
    FX_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
    fx::I8Slices sa{}, sb{};
    for (int q = 0; q < kNoAllocSlices; ++q) {
      sa.re[q] = sl + (size_t)q * M * K;
      sb.re[q] = sl + (size_t)kNoAllocSlices * M * K + (size_t)q * N * K;
    }
    sa.exp = aexp;
    sb.exp = bexp;
    sa.ld = sb.ld = K;
    fx::launch_slice_rows<float>(kNoAllocSlices, A, nullptr, lda, M, K, sa, false, s);
    fx::launch_slice_rows<float>(kNoAllocSlices, Bt, nullptr, ldb, N, K, sb, false, s);
    fx::I8Term t{};
    for (int q = 0; q < kNoAllocSlices; ++q) {
      t.a[q] = sa.re[q];
      t.b[q] = sb.re[q];
    }
    fx::launch_gemm_i8<float>(kNoAllocSlices, M, N, K, &t, 1, K, K, aexp, bexp, alpha, beta, C, ldc, gamma, D,
                              ldd, false, err, 2000, s);
    int h_err = 0;
    FX_CUDA(cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, s));
    FX_CUDA(cudaStreamSynchronize(s));
    if (h_err) throw fx::Error{FX_ERR_TIMEOUT, "device wait timed out in the product kernel"};
  } catch (const fx::Error& e) {
    fx::set_product_error(e.msg);
    return e.code;
  }
  return FX_OK;
}

}  // extern "C"
