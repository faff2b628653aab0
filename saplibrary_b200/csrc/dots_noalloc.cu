// Allocation-free fused dot products (sap_blas_dots_noalloc).
//
// Some callers of this library cannot allocate device memory at the point
// where they need a reduction: code that runs under another framework's
// caching allocator which already owns the free device memory, applications
// that budget all GPU memory once at start-up, and latency-critical loops in
// which a cudaMalloc / cudaFree pair would synchronise the device.  This
// entry point computes the same dot products as sap_blas_dots but keeps its
// block partial sums in a fixed scratch array compiled into the library, so
// it performs no allocation of any kind.
//
// The scratch is a file-scope __device__ array: every GPU that loads the
// library holds it (SCRATCH_BYTES below) until the process exits.  Host code
// cannot use the array's name as a device address; the device address is
// looked up with cudaGetSymbolAddress on the first call made in a device's
// context and cached with that context.  A call made in another context of
// the same device (a context the caller created and made current, or the
// primary context re-created after cudaDeviceReset with a different handle)
// looks the address up again.  cudaDeviceReset unloads the library's device
// code: after a reset, the first call should come from a fresh primary
// context, before any stream capture.
#include <cuda.h>

#include <mutex>

#include "common.cuh"
#include "krylov_kernels.cuh"

namespace sapb {

// Largest grid the scratch can serve, hence the largest vector length:
// kNoAllocMaxBlocks * kDotThreads * kDotItems = 16,777,216 elements.
constexpr int kNoAllocMaxBlocks = 2048;
constexpr long long kNoAllocMaxN = (long long)kNoAllocMaxBlocks * kDotThreads * kDotItems;
// 4 partials per block (one per dot product) followed by the completion counter.
constexpr size_t kPartialBytes = sizeof(double) * 4 * kNoAllocMaxBlocks;
constexpr size_t kScratchBytes = kPartialBytes + 256;

static __device__ __align__(256) unsigned char g_dots_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
static std::mutex g_scratch_mu;
static void* g_scratch_addr[kMaxDevices] = {};
static CUcontext g_scratch_ctx[kMaxDevices] = {};

// The calling thread's current driver context (the runtime makes the
// device's primary context current on its first call); reached through the
// runtime's driver entry-point table, so the library does not link libcuda.
static CUcontext current_context() {
  using GetCurrent = CUresult (*)(CUcontext*);
  static GetCurrent fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<GetCurrent>(f);
  }();
  CUcontext c = nullptr;
  if (!fn || fn(&c) != CUDA_SUCCESS) throw Error(SAP_ERR_CUDA, "cuCtxGetCurrent is not available");
  return c;
}

// Device address of the scratch in the current context of the current
// device (looked up on the first call made in that context).
static unsigned char* scratch_on_current_device() {
  int dev = 0;
  SAPB_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) throw Error(SAP_ERR_UNSUPPORTED, "device ordinal beyond 63");
  const CUcontext ctx = current_context();  // null before the runtime's first context is made current
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if (!ctx || !g_scratch_addr[dev] || g_scratch_ctx[dev] != ctx) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_dots_scratch);  // makes the primary context current if none is
    if (e != cudaSuccess || !p)
      throw Error(SAP_ERR_CUDA, std::string("cudaGetSymbolAddress of the dot-product scratch failed: ") +
                                    cudaGetErrorString(e));
    g_scratch_addr[dev] = p;
    g_scratch_ctx[dev] = current_context();
  }
  return static_cast<unsigned char*>(g_scratch_addr[dev]);
}

}  // namespace sapb

extern "C" {

int sap_blas_dots_noalloc(int n, int nq, const double* const* x, const double* const* y, double* out,
                          void* stream) {
  using namespace sapb;
  try {
    if (n < 0 || nq < 1 || nq > 4 || !x || !y || !out)
      throw Error(SAP_ERR_INVALID_ARGUMENT, "invalid dot-product arguments");
    if ((long long)n > kNoAllocMaxN)
      throw Error(SAP_ERR_INVALID_ARGUMENT,
                  "sap_blas_dots_noalloc: vector length " + std::to_string(n) + " exceeds the fixed scratch limit of " +
                      std::to_string(kNoAllocMaxN) + " elements; use sap_blas_dots");
    DotArgs a{};
    a.nq = nq;
    for (int q = 0; q < nq; q++) {
      if (!x[q] || !y[q]) throw Error(SAP_ERR_INVALID_ARGUMENT, "null vector");
      a.x[q] = x[q];
      a.y[q] = y[q];
    }
    unsigned char* base = scratch_on_current_device();
    double* part = reinterpret_cast<double*>(base);
    unsigned int* ctr = reinterpret_cast<unsigned int*>(base + kPartialBytes);
    cudaStream_t st = (cudaStream_t)stream;
    const int grid = dot_grid_for(n);
    // the completion counter must start at zero; the partials are overwritten
    SAPB_CUDA(cudaMemsetAsync(ctr, 0, sizeof(unsigned int), st));
    k_dots<<<grid, kDotThreads, 0, st>>>(n, a, part, ctr, out);
    SAPB_LAUNCHED();
    return SAP_OK;
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.code;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return SAP_ERR_CUDA;
  }
}

}  // extern "C"
