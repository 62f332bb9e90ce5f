// Cholesky factorization that allocates no device memory.
//
// egpu_dpotrf (api.cu) keeps the inverse of the current diagonal block in a
// workspace that its handle allocates.  Some callers cannot let a library
// allocate: for example a host process that hands all device memory to its
// own pool at start-up (a framework's caching allocator, a fixed HBM budget
// shared by many solvers) and must not see an allocation fail or synchronise
// the device in the middle of its work.  This entry point takes the caller's
// stream instead of a handle and keeps its scratch -- one nb x nb diagonal
// block inverse and the status word -- in a file-scope __device__ array that
// exists on every GPU which loads the library, from load until exit.
//
// The scratch is shared by every call on a device and keeps the previous
// call's contents; the status word is cleared at the start of each call and
// the inverse block is always written before it is read.  Calls whose work
// overlaps on the GPU (other streams, other host threads) race on the array.
// Under CUDA's lazy module loading (the default) the driver loads this file's
// module, and with it the array, and the kernels' modules on the first call on
// a device: that call is where device memory is taken, so callers make one
// small call at start-up (or run with CUDA_MODULE_LOADING=EAGER).  An odd nb
// is rounded down to the next even value (the diagonal kernels work on column
// pairs), as egpu_set_blocksize does for a handle.
#include <mutex>

#include "internal.h"

namespace egpu {

constexpr int kNoAllocMaxNB = 128;
constexpr size_t kNoAllocInvBytes = sizeof(double) * kNoAllocMaxNB * kNoAllocMaxNB;  // 128 KiB
constexpr size_t kNoAllocBytes = kNoAllocInvBytes + 256;                              // + status word

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// Device address of the scratch array, looked up once per device with that
// device current (host code may only name the symbol, not dereference it).
struct NoAllocSlot {
  bool done = false;
  cudaError_t err = cudaSuccess;
  void* ptr = nullptr;
};
static std::mutex g_noalloc_mu;
static NoAllocSlot g_noalloc_slot[64];

static cudaError_t noalloc_scratch(int dev, void** out) {
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  NoAllocSlot& s = g_noalloc_slot[dev];
  if (!s.done) {
    s.err = cudaGetSymbolAddress(&s.ptr, g_noalloc_scratch);
    s.done = true;
  }
  *out = s.ptr;
  return s.err;
}

}  // namespace egpu

using namespace egpu;

extern "C" int egpu_dpotrf_noalloc(void* stream, int uplo, int n, double* dA, int lda, int nb, int* info) {
  if (info) *info = 0;
  if (n < 0 || lda < std::max(1, n) || (uplo != EGPU_LOWER && uplo != EGPU_UPPER)) return EGPU_ERR_ARG;
  if (nb < 2 || nb > kNoAllocMaxNB) {
    set_last_error(cudaErrorInvalidValue, "egpu_dpotrf_noalloc: nb must lie in [2, 128] (scratch holds one 128x128 block)",
                   __FILE__, __LINE__);
    return EGPU_ERR_UNSUPPORTED;
  }
  if (n == 0) return EGPU_OK;
  if (!tma_compatible(dA, lda)) return EGPU_ERR_ALIGN;  // no room to repack without allocating
  nb &= ~1;
  int dev = 0;
  EGPU_CUDA_TRY(cudaGetDevice(&dev));
  void* scratch = nullptr;
  EGPU_CUDA_TRY(noalloc_scratch(dev, &scratch));
  double* W = static_cast<double*>(scratch);
  DevStatus* status = reinterpret_cast<DevStatus*>(static_cast<unsigned char*>(scratch) + kNoAllocInvBytes);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  EGPU_CUDA_TRY(cudaMemsetAsync(status, 0, sizeof(DevStatus), st));
  // Blocked right-looking sweep (Cholesky/LVar3.hpp:83-123, UVar3.hpp:85-125)
  // on the caller's stream, one step after the other.
  for (int k = 0; k < n; k += nb) {
    const int b = std::min(nb, n - k);
    const int m2 = n - k - b;
    int rc = launch_potrf_diag(st, uplo, dA + k + (size_t)k * lda, lda, b, W, nb, status, k);
    if (rc != EGPU_OK) return rc;
    if (m2 == 0) continue;
    if (uplo == EGPU_LOWER) {
      double* A21 = dA + (k + b) + (size_t)k * lda;
      double* A22 = dA + (k + b) + (size_t)(k + b) * lda;
      rc = launch_dgemm(st, false, false, m2, b, b, 1.0, A21, lda, W, nb, 0.0, A21, lda, 0, true, status);
      if (rc == EGPU_OK)
        rc = launch_dgemm(st, false, false, m2, m2, b, -1.0, A21, lda, A21, lda, 1.0, A22, lda, 1, false, status);
    } else {
      double* A12 = dA + k + (size_t)(k + b) * lda;
      double* A22 = dA + (k + b) + (size_t)(k + b) * lda;
      rc = launch_dgemm(st, true, true, b, m2, b, 1.0, W, nb, A12, lda, 0.0, A12, lda, 0, false, status);
      if (rc == EGPU_OK)
        rc = launch_dgemm(st, true, true, m2, m2, b, -1.0, A12, lda, A12, lda, 1.0, A22, lda, 2, false, status);
    }
    if (rc != EGPU_OK) return rc;
  }
  DevStatus hs;
  EGPU_CUDA_TRY(cudaMemcpyAsync(&hs, status, sizeof(DevStatus), cudaMemcpyDeviceToHost, st));
  EGPU_CUDA_TRY(cudaStreamSynchronize(st));
  if (info) *info = hs.code ? hs.info : 0;
  switch (hs.code) {
    case kOk: return EGPU_OK;
    case kNotHPD: return EGPU_NOT_HPD;
    case kSingular: return EGPU_SINGULAR;
    default: return EGPU_TIMEOUT;
  }
}
