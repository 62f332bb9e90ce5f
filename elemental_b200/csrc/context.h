// Handle state shared by the C-ABI translation units: the egpu_context
// behind egpu_handle, its workspace, status word, trace and streams, and
// the blocked drivers other files call.
#pragma once
#include <string>
#include <vector>

#include "internal.h"

namespace egpu {

struct Trace {
  struct Rec {
    int kind;
    double flops, bytes;
    cudaEvent_t e0, e1;
    cudaStream_t st;  // the launch's stream (timeline dumps)
  };
  bool on = false;
  std::vector<Rec> recs;
  std::vector<cudaEvent_t> pool;
  cudaEvent_t get() {
    if (pool.empty()) {
      cudaEvent_t e;
      if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
      return e;
    }
    cudaEvent_t e = pool.back();
    pool.pop_back();
    return e;
  }
  void clear() {
    for (auto& r : recs) {
      if (r.e0) pool.push_back(r.e0);
      if (r.e1) pool.push_back(r.e1);
    }
    recs.clear();
  }
  ~Trace() {
    clear();
    for (auto e : pool) cudaEventDestroy(e);
  }
};

extern thread_local Trace* t_trace;

}  // namespace egpu

using namespace egpu;

struct egpu_context {
  int device = 0;
  int sm_count = 148;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  int nb = 128;
  void* ws = nullptr;
  size_t ws_bytes = 0;
  DevStatus* dstatus = nullptr;
  DevStatus* hstatus = nullptr;  // pinned
  // host-API staging buffers
  // staging slots: 0, 1 operand copies; 2 pivots (+ small results); 3 the
  // n x n right-hand side of the inverses / the determinant's copy of A
  static constexpr int kStageSlots = 4;
  void* stage[kStageSlots] = {nullptr, nullptr, nullptr, nullptr};
  size_t stage_bytes[kStageSlots] = {0, 0, 0, 0};
  Trace trace;
  // look-ahead: a high-priority side stream for the panel chain and events
  // joining it with the update chain on `stream`
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  cudaEvent_t ev_panel[2] = {nullptr, nullptr}, ev_rest[2] = {nullptr, nullptr};
  // a lowest-priority stream for work that only fills idle SMs (the mixed
  // path's prescaled solve copies), joined before its results are read
  cudaStream_t aux = nullptr;
  cudaEvent_t ev_split[2] = {nullptr, nullptr}, ev_aux = nullptr;
  // the mixed chain: a block column's rows below its diagonal block updated
  // (and split) -- the next panel's L21 product waits for it
  cudaEvent_t ev_a21[2] = {nullptr, nullptr};
  // grouped FP64 Cholesky: the next group's first block column updated
  cudaEvent_t ev_next[2] = {nullptr, nullptr};
  int lookahead = -1;  // -1 auto groups, 0 sequential, 1 per-panel, G >= 2 fixed groups (Cholesky)
  int async = 0;  // device API: enqueue only; status read by egpu_get_status
  int gmres_inner = 0;  // GMRES iterations of the last mixed solve
  // mixed solve: 0 adaptive (condition estimate when the first correction
  // contracts slowly), 1 estimate after every factorization
  int mixed_policy = 0;
  double mixed_kappa = -1.0;
  int mixed_mode = 0;  // how the last mixed solve finished: 0 refinement, 1 GMRES-IR, 2 FP64 factors  // last 1-norm condition estimate (-1: none)
};

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

inline int ensure_ws(egpu_context* h, size_t bytes) {
  if (bytes <= h->ws_bytes) return EGPU_OK;
  if (h->ws) {
    cudaStreamSynchronize(h->stream);
    cudaFree(h->ws);
    h->ws = nullptr;
    h->ws_bytes = 0;
  }
  bytes = (bytes + (1 << 20) - 1) & ~size_t((1 << 20) - 1);
  cudaError_t e = cudaMalloc(&h->ws, bytes);
  if (e != cudaSuccess) {
    set_last_error(e, "workspace cudaMalloc", __FILE__, __LINE__);
    cudaGetLastError();
    return EGPU_ERR_ALLOC;
  }
  h->ws_bytes = bytes;
  return EGPU_OK;
}

inline int ensure_stage(egpu_context* h, int slot, size_t bytes) {
  if (bytes <= h->stage_bytes[slot]) return EGPU_OK;
  if (h->stage[slot]) {
    cudaStreamSynchronize(h->stream);
    cudaFree(h->stage[slot]);
    h->stage[slot] = nullptr;
    h->stage_bytes[slot] = 0;
  }
  bytes = (bytes + (1 << 20) - 1) & ~size_t((1 << 20) - 1);
  cudaError_t e = cudaMalloc(&h->stage[slot], bytes);
  if (e != cudaSuccess) {
    set_last_error(e, "staging cudaMalloc", __FILE__, __LINE__);
    cudaGetLastError();
    return EGPU_ERR_ALLOC;
  }
  h->stage_bytes[slot] = bytes;
  return EGPU_OK;
}

// Entered by every C-ABI call: selects the handle's device and makes its
// trace the calling thread's active trace.
struct Enter {
  DeviceGuard g;
  Trace* prev;
  explicit Enter(egpu_context* h) : g(h->device), prev(t_trace) { t_trace = &h->trace; }
  ~Enter() { t_trace = prev; }
};

// Host-memory entry points are synchronous whatever the handle's mode.
struct SyncScope {
  egpu_context* h;
  int saved;
  explicit SyncScope(egpu_context* hh) : h(hh), saved(hh->async) { hh->async = 0; }
  ~SyncScope() { h->async = saved; }
};

inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }
inline long long ld_aligned(int rows) { return std::max<long long>(32, align_up((size_t)std::max(rows, 1), 32)); }

// Simple bump allocator over the handle workspace.
struct Carve {
  unsigned char* base;
  size_t off = 0;
  explicit Carve(void* b) : base(static_cast<unsigned char*>(b)) {}
  template <class T>
  T* take(size_t count) {
    off = align_up(off, 256);
    T* p = reinterpret_cast<T*>(base + off);
    off += sizeof(T) * count;
    return p;
  }
};

inline int reset_status(egpu_context* h) {
  if (h->async) return EGPU_OK;  // async: the first failure stays until egpu_get_status
  EGPU_CUDA_TRY(cudaMemsetAsync(h->dstatus, 0, sizeof(DevStatus), h->stream));
  return EGPU_OK;
}

inline int read_status_now(egpu_context* h, int* info) {
  EGPU_CUDA_TRY(cudaMemcpyAsync(h->hstatus, h->dstatus, sizeof(DevStatus), cudaMemcpyDeviceToHost, h->stream));
  EGPU_CUDA_TRY(cudaStreamSynchronize(h->stream));
  if (info) *info = h->hstatus->code ? h->hstatus->info : 0;
  switch (h->hstatus->code) {
    case kOk: return EGPU_OK;
    case kNotHPD: return EGPU_NOT_HPD;
    case kSingular: return EGPU_SINGULAR;
    default: return EGPU_TIMEOUT;
  }
}

// Synchronous mode: wait and map the status.  Async mode: return at once.
inline int read_status(egpu_context* h, int* info) {
  if (h->async) {
    if (info) *info = 0;
    return EGPU_OK;
  }
  return read_status_now(h, info);
}

#define TRY(x)               \
  do {                       \
    int _r = (x);            \
    if (_r != EGPU_OK) return _r; \
  } while (0)

// Drivers defined in api.cu.
int potrf_core(egpu_context* h, int uplo, int n, double* A, long long lda);
int potrs_core(egpu_context* h, int uplo, int n, int nrhs, const double* A, long long lda, double* B, long long ldb);
int trsm_core(egpu_context* h, int side, int uplo, int trans, int unit, int m, int n, double alpha, const double* A,
              long long lda, double* B, long long ldb, size_t ws_offset);
size_t winv_bytes(int nt, int nb);
// Mixed-precision HPD solve (mixed.cu).
int dposv_mixed_core(egpu_context* h, int uplo, int n, int nrhs, const double* A, long long lda, const double* B,
                     long long ldb, double* X, long long ldx, int max_iter, double tol, int* iters, double* berr);
int trsm_blocked(cudaStream_t st, int side, int uplo, int trans, int m, int n, const double* A, long long lda,
                 const double* Winv, int nb, double* B, long long ldb, DevStatus* status);

