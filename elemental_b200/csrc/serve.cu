// Request server: continuous batching of HPD (Cholesky) and general (LU)
// solve requests on one GPU.
//
// submit() queues a request (host buffers A, B, X; they stay valid until the
// request completes).  A dispatcher thread admits requests in arrival order
// against an HBM budget and hands them to `slots` worker threads, each with
// its own egpu handle (stream + workspace), so the work of up to `slots` jobs
// overlaps on the device.  When a worker frees up, every queued small
// request (n <= 512, nrhs <= 16) of the kind at the head of the queue is
// taken as one job and solved in one batched launch; a larger request is a
// job of its own.  Mode 1 solves HPD requests of order >= mixed_min_n with
// the mixed-precision solver (egpu_dposv_mixed) and falls back to the FP64
// path for a request it cannot bring to the tolerance; smaller HPD requests
// (where the FP64 path is faster on this hardware) take the FP64 path.  A GE
// request in mode 1 first gets the structure test of a general-purpose
// backslash: when A is exactly symmetric with a positive diagonal, the HPD
// solvers are tried (Cholesky exists iff A is HPD; the mixed solver from the
// same order threshold), and only when that factorization fails does the
// request go to the LU path (egpu_dgesv) -- the same x either way.  Mode 0
// runs every GE request through egpu_dgesv.
//
// Resident matrices: egpu_server_register copies a matrix to the device once
// (charged to the budget with room for its factor) and requests on it
// (egpu_server_submit_resident) send only B and X.  The first request on a
// resident matrix factors a device copy of it (Cholesky for HPD; in mode 1 a
// GE matrix that passes the structure test above is tried with Cholesky
// first, else LU with partial pivoting) and later requests reuse the factor:
// each is one FP64 solve (cholesky::SolveAfter or lu::SolveAfter).  Requests
// that arrive while the factor is being formed wait for it.  Completion times are recorded per request (latency =
// completion - submission, host steady clock).
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "context.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Resident {
  unsigned long long mid = 0;
  int kind = 0, n = 0, ld = 0;
  double* dA = nullptr;  // the matrix, as registered
  double* dF = nullptr;  // its factor (Cholesky L or LU) once formed
  int* dpiv = nullptr;   // LU pivots
  int state = 0;         // 0 not factored, 1 being factored, 2 Cholesky, 3 LU, 4 failed
  int fail_status = 0;
  int users = 0;         // requests queued or running on it
  size_t bytes = 0;      // budget charge
};

struct Request {
  unsigned long long id = 0;
  Resident* res = nullptr;  // a request on a resident matrix (A unused)
  int kind = 0, n = 0, nrhs = 0, lda = 0, ldb = 0, ldx = 0;
  const double* A = nullptr;
  const double* B = nullptr;
  double* X = nullptr;
  size_t bytes = 0;  // device bytes while in flight
  Clock::time_point t_submit, t_done;
  int status = 0;
  bool done = false;
  // 0 single FP64, 1 mixed, 2 batched, 3 mixed fell back to FP64, 4 GE request
  // solved by the FP64 HPD path, 5 GE request solved by the mixed HPD path,
  // 6 resident matrix factored by this request, 7 resident factor reused
  int path = 0;
  int iters = 0;
  double berr = 0.0;
};

constexpr int kSmallN = 512, kSmallRhs = 16, kMaxBatch = 1024;

size_t request_bytes(int mode, int kind, int n, int nrhs) {
  const size_t nn = (size_t)n * n, nr = (size_t)n * std::max(nrhs, 1);
  size_t b = 8 * (nn + 2 * nr);                                                    // A, B, X on the device
  if (mode == 1 && n > kSmallN) b += 8 * nn * 2 + 4 * nn + 8 * 4 * nr;  // mixed working copies
  else b += 8 * (size_t)128 * 128 + 8 * nr;                                         // diagonal-block workspace
  return b;
}

// *flag |= 1 when some A(i, j) != A(j, i), |= 2 when some A(i, i) <= 0 (or
// NaN): 32 x 32 tiles of the lower triangle against their mirror tiles
// through shared memory, so both reads are coalesced.
__global__ void sym_posdiag_kernel(int n, const double* A, long long lda, int* flag) {
  __shared__ double up[32][33];
  const int bi = blockIdx.x, bj = blockIdx.y;  // tile row, tile column (bi >= bj)
  if (bj > bi) return;
  const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
  for (int q = ty; q < 32; q += 8) {             // the mirror tile A(bj, bi), transposed into up
    const int r = bj * 32 + tx, c = bi * 32 + q;
    up[tx][q] = (r < n && c < n) ? A[r + (long long)c * lda] : 0.0;
  }
  __syncthreads();
  int bad = 0;
  for (int q = ty; q < 32; q += 8) {
    const int r = bi * 32 + tx, c = bj * 32 + q;  // A(r, c), r in tile bi, c in tile bj
    if (r >= n || c >= n) continue;
    const double v = A[r + (long long)c * lda];
    if (r > c && v != up[q][tx]) bad |= 1;
    if (r == c && !(v > 0.0)) bad |= 2;
  }
  bad = __reduce_or_sync(0xffffffffu, bad);
  if (bad && (threadIdx.x & 31) == 0) atomicOr(flag, bad);
}

}  // namespace

struct egpu_server_s {
  int device = 0, slots = 1, mode = 0;
  size_t budget = 0, in_use = 0;
  double tol = 1e-14;
  int mixed_min_n = 6144;  // mode 1: smaller HPD requests take the FP64 path (faster there on average)
  std::mutex mu;
  std::condition_variable cv_dispatch, cv_done;
  std::deque<Request*> queue;
  std::unordered_map<unsigned long long, Request*> all;
  std::unordered_map<unsigned long long, Resident*> resident;
  std::condition_variable cv_res;  // a resident factor finished
  unsigned long long next_id = 1;
  bool stop = false;
  struct Worker {
    egpu_handle h = nullptr;
    int* flag = nullptr;  // device word of the structure test
    std::vector<Request*> job;
    bool busy = false;
    std::condition_variable cv;
    std::thread th;
  };
  std::vector<Worker*> workers;
  std::thread dispatcher;
};

namespace {

// Does A (device, ld) pass the structure test: exactly symmetric with a
// positive diagonal?  (false also when the test cannot run)
bool symmetric_posdiag(egpu_server_s::Worker* w, cudaStream_t st, int n, const double* A, int ld) {
  if (!w->flag) return false;
  cudaMemsetAsync(w->flag, 0, sizeof(int), st);
  const int nt = (n + 31) / 32;
  sym_posdiag_kernel<<<dim3(nt, nt), dim3(32, 8), 0, st>>>(n, A, ld, w->flag);
  int flag = -1;
  return cudaGetLastError() == cudaSuccess &&
         cudaMemcpyAsync(&flag, w->flag, sizeof(int), cudaMemcpyDeviceToHost, st) == cudaSuccess &&
         cudaStreamSynchronize(st) == cudaSuccess && flag == 0;
}

// A request on a resident matrix: form the factor if no request has, wait
// for it if another request is forming it, then one FP64 solve.
template <class Finish>
void run_resident(egpu_server_s* s, egpu_server_s::Worker* w, Request* r, cudaStream_t st, Finish& finish) {
  Resident* R = r->res;
  egpu_handle h = w->h;
  const int n = R->n, ld = R->ld;
  bool mine = false;
  {
    std::unique_lock<std::mutex> lk(s->mu);
    s->cv_res.wait(lk, [&] { return R->state != 1; });
    if (R->state == 0) {
      R->state = 1;
      mine = true;
    }
  }
  if (mine) {
    int state = 4, status = EGPU_ERR_CUDA, info = 0;
    const size_t pitch = sizeof(double) * ld;
    if (cudaMemcpy2DAsync(R->dF, pitch, R->dA, pitch, sizeof(double) * n, n, cudaMemcpyDeviceToDevice, st) ==
        cudaSuccess) {
      bool hpd = R->kind == 0 || (s->mode == 1 && symmetric_posdiag(w, st, n, R->dA, ld));
      if (hpd) {
        status = egpu_dpotrf(h, EGPU_LOWER, n, R->dF, ld, &info);
        if (status == EGPU_OK) state = 2;
        else if (R->kind == 1) {  // not HPD after all: LU on a fresh copy
          cudaMemcpy2DAsync(R->dF, pitch, R->dA, pitch, sizeof(double) * n, n, cudaMemcpyDeviceToDevice, st);
          hpd = false;
        }
      }
      if (!hpd) {
        status = egpu_dgetrf(h, n, n, R->dF, ld, R->dpiv, &info);
        if (status == EGPU_OK) state = 3;
      }
    }
    {
      std::lock_guard<std::mutex> lk(s->mu);
      R->state = state;
      R->fail_status = status;
    }
    s->cv_res.notify_all();
  }
  r->path = mine ? 6 : 7;
  if (R->state == 4) {
    finish(r, R->fail_status == EGPU_OK ? EGPU_ERR_CUDA : R->fail_status);
    return;
  }
  const int nrhs = std::max(r->nrhs, 1);
  double* dB = nullptr;
  if (cudaMallocAsync(reinterpret_cast<void**>(&dB), sizeof(double) * ld * (size_t)nrhs, st) != cudaSuccess) {
    cudaGetLastError();
    cudaStreamSynchronize(st);
    finish(r, EGPU_ERR_ALLOC);
    return;
  }
  cudaMemcpy2DAsync(dB, sizeof(double) * ld, r->B, sizeof(double) * r->ldb, sizeof(double) * n, r->nrhs,
                    cudaMemcpyHostToDevice, st);
  const int rc = R->state == 2 ? egpu_dpotrs(h, EGPU_LOWER, EGPU_NORMAL, n, r->nrhs, R->dF, ld, dB, ld)
                               : egpu_dgetrs(h, EGPU_NORMAL, n, r->nrhs, R->dF, ld, R->dpiv, dB, ld);
  if (rc == EGPU_OK)
    cudaMemcpy2DAsync(r->X, sizeof(double) * r->ldx, dB, sizeof(double) * ld, sizeof(double) * n, r->nrhs,
                      cudaMemcpyDeviceToHost, st);
  cudaFreeAsync(dB, st);
  const cudaError_t e = cudaStreamSynchronize(st);
  finish(r, rc != EGPU_OK ? rc : (e != cudaSuccess ? EGPU_ERR_CUDA : EGPU_OK));
}

// Solve one job on worker w (its handle's stream; synchronous).
void run_job(egpu_server_s* s, egpu_server_s::Worker* w, std::vector<Request*>& job) {
  egpu_handle h = w->h;
  cudaStream_t st = static_cast<cudaStream_t>(egpu_get_stream(h));
  auto finish = [&](Request* r, int status) {
    r->status = status;
    r->t_done = Clock::now();
  };
  if (job.size() == 1 && job[0]->res) {  // a request on a resident matrix
    run_resident(s, w, job[0], st, finish);
    return;
  }
  if (job.size() > 1 || (job[0]->n <= kSmallN && job[0]->nrhs <= kSmallRhs)) {
    // batched job: one arena for all matrices and right-hand sides
    const int cnt = (int)job.size();
    std::vector<size_t> offA(cnt), offB(cnt);
    size_t tot = 0;
    for (int i = 0; i < cnt; ++i) {
      const int n = job[i]->n, ld = std::max(2, n + (n & 1));
      offA[i] = tot;
      tot += (size_t)ld * n;
      offB[i] = tot;
      tot += (size_t)ld * std::max(job[i]->nrhs, 1);
    }
    double* arena = nullptr;
    cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(&arena), sizeof(double) * std::max<size_t>(tot, 1), st);
    if (e != cudaSuccess) {
      cudaGetLastError();
      for (Request* r : job) finish(r, EGPU_ERR_ALLOC);
      return;
    }
    std::vector<int> n(cnt), nr(cnt), ld(cnt), info(cnt, 0);
    std::vector<double*> pa(cnt), pb(cnt);
    for (int i = 0; i < cnt; ++i) {
      Request* r = job[i];
      n[i] = r->n;
      nr[i] = r->nrhs;
      ld[i] = std::max(2, r->n + (r->n & 1));
      pa[i] = arena + offA[i];
      pb[i] = arena + offB[i];
      cudaMemcpy2DAsync(pa[i], sizeof(double) * ld[i], r->A, sizeof(double) * r->lda, sizeof(double) * r->n, r->n,
                        cudaMemcpyHostToDevice, st);
      cudaMemcpy2DAsync(pb[i], sizeof(double) * ld[i], r->B, sizeof(double) * r->ldb, sizeof(double) * r->n, r->nrhs,
                        cudaMemcpyHostToDevice, st);
    }
    const int kind = job[0]->kind;
    int rc = kind == 0 ? egpu_dposv_batched(h, cnt, n.data(), nr.data(), pa.data(), ld.data(), pb.data(), ld.data(),
                                            info.data())
                       : egpu_dgesv_batched(h, cnt, n.data(), nr.data(), pa.data(), ld.data(), pb.data(), ld.data(),
                                            info.data());
    for (int i = 0; i < cnt; ++i) {
      Request* r = job[i];
      if (rc == EGPU_OK && info[i] == 0)
        cudaMemcpy2DAsync(r->X, sizeof(double) * r->ldx, pb[i], sizeof(double) * ld[i], sizeof(double) * r->n,
                          r->nrhs, cudaMemcpyDeviceToHost, st);
    }
    cudaFreeAsync(arena, st);
    e = cudaStreamSynchronize(st);
    for (int i = 0; i < cnt; ++i) {
      job[i]->path = 2;
      int status = rc;
      if (status == EGPU_OK && e != cudaSuccess) status = EGPU_ERR_CUDA;
      if (status == EGPU_OK && info[i]) status = job[i]->kind == 0 ? EGPU_NOT_HPD : EGPU_SINGULAR;
      finish(job[i], status);
    }
    return;
  }
  Request* r = job[0];
  const int n = r->n, ldd = std::max(32, (n + 31) / 32 * 32), nrhs = std::max(r->nrhs, 1);
  double *dA = nullptr, *dB = nullptr, *dX = nullptr;
  cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(&dA), sizeof(double) * ldd * (size_t)n, st);
  if (e == cudaSuccess) e = cudaMallocAsync(reinterpret_cast<void**>(&dB), sizeof(double) * ldd * (size_t)nrhs, st);
  if (e == cudaSuccess) e = cudaMallocAsync(reinterpret_cast<void**>(&dX), sizeof(double) * ldd * (size_t)nrhs, st);
  if (e != cudaSuccess) {
    cudaGetLastError();
    if (dA) cudaFreeAsync(dA, st);
    if (dB) cudaFreeAsync(dB, st);
    cudaStreamSynchronize(st);
    finish(r, EGPU_ERR_ALLOC);
    return;
  }
  cudaMemcpy2DAsync(dA, sizeof(double) * ldd, r->A, sizeof(double) * r->lda, sizeof(double) * n, n,
                    cudaMemcpyHostToDevice, st);
  cudaMemcpy2DAsync(dB, sizeof(double) * ldd, r->B, sizeof(double) * r->ldb, sizeof(double) * n, r->nrhs,
                    cudaMemcpyHostToDevice, st);
  int rc, info = 0;
  double* sol = dB;
  if (r->kind == 0 && s->mode == 1 && n >= s->mixed_min_n) {
    rc = egpu_dposv_mixed(h, EGPU_LOWER, n, r->nrhs, dA, ldd, dB, ldd, dX, ldd, 30, s->tol, &r->iters, &r->berr);
    r->path = 1;
    sol = dX;
    if (rc == EGPU_NOT_HPD || rc == EGPU_NO_CONVERGENCE) {  // FP64 fallback on the untouched inputs
      rc = egpu_dposv(h, EGPU_LOWER, EGPU_NORMAL, n, r->nrhs, dA, ldd, dB, ldd, &info);
      r->path = 3;
      sol = dB;
    }
  } else if (r->kind == 0) {
    rc = egpu_dposv(h, EGPU_LOWER, EGPU_NORMAL, n, r->nrhs, dA, ldd, dB, ldd, &info);
  } else {
    bool hpd_done = false;
    rc = EGPU_OK;
    if (s->mode == 1 && w->flag) {
      // the structure test; on success the HPD path, else (or when that
      // factorization fails) LU on freshly copied inputs
      cudaMemsetAsync(w->flag, 0, sizeof(int), st);
      const int nt = (n + 31) / 32;
      sym_posdiag_kernel<<<dim3(nt, nt), dim3(32, 8), 0, st>>>(n, dA, ldd, w->flag);
      int flag = -1;
      if (cudaGetLastError() == cudaSuccess &&
          cudaMemcpyAsync(&flag, w->flag, sizeof(int), cudaMemcpyDeviceToHost, st) == cudaSuccess &&
          cudaStreamSynchronize(st) == cudaSuccess && flag == 0) {
        if (n >= s->mixed_min_n) {
          rc = egpu_dposv_mixed(h, EGPU_LOWER, n, r->nrhs, dA, ldd, dB, ldd, dX, ldd, 30, s->tol, &r->iters,
                                &r->berr);
          if (rc == EGPU_OK) { hpd_done = true; r->path = 5; sol = dX; }
        } else {
          rc = egpu_dposv(h, EGPU_LOWER, EGPU_NORMAL, n, r->nrhs, dA, ldd, dB, ldd, &info);
          if (rc == EGPU_OK) {
            hpd_done = true;
            r->path = 4;
          } else {  // the factorization overwrote A and B: copy them again
            cudaMemcpy2DAsync(dA, sizeof(double) * ldd, r->A, sizeof(double) * r->lda, sizeof(double) * n, n,
                              cudaMemcpyHostToDevice, st);
            cudaMemcpy2DAsync(dB, sizeof(double) * ldd, r->B, sizeof(double) * r->ldb, sizeof(double) * n,
                              r->nrhs, cudaMemcpyHostToDevice, st);
          }
        }
      }
    }
    if (!hpd_done) {
      r->path = 0;
      sol = dB;
      rc = egpu_dgesv(h, n, r->nrhs, dA, ldd, dB, ldd, &info);
    }
  }
  if (rc == EGPU_OK)
    cudaMemcpy2DAsync(r->X, sizeof(double) * r->ldx, sol, sizeof(double) * ldd, sizeof(double) * n, r->nrhs,
                      cudaMemcpyDeviceToHost, st);
  cudaFreeAsync(dA, st);
  cudaFreeAsync(dB, st);
  cudaFreeAsync(dX, st);
  e = cudaStreamSynchronize(st);
  finish(r, rc != EGPU_OK ? rc : (e != cudaSuccess ? EGPU_ERR_CUDA : EGPU_OK));
}

void worker_main(egpu_server_s* s, egpu_server_s::Worker* w) {
  cudaSetDevice(s->device);
  for (;;) {
    std::vector<Request*> job;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      w->cv.wait(lk, [&] { return s->stop || !w->job.empty(); });
      if (w->job.empty() && s->stop) return;
      job.swap(w->job);
    }
    run_job(s, w, job);
    {
      std::lock_guard<std::mutex> lk(s->mu);
      for (Request* r : job) {
        r->done = true;
        s->in_use -= r->bytes;
        if (r->res) --r->res->users;
      }
      w->busy = false;
    }
    s->cv_dispatch.notify_one();
    s->cv_done.notify_all();
  }
}

// Admission and batching: runs whenever a request arrives or a worker frees.
void dispatcher_main(egpu_server_s* s) {
  std::unique_lock<std::mutex> lk(s->mu);
  for (;;) {
    s->cv_dispatch.wait(lk, [&] {
      if (s->stop) return true;
      if (s->queue.empty()) return false;
      for (auto* w : s->workers)
        if (!w->busy) return true;
      return false;
    });
    if (s->stop) return;
    egpu_server_s::Worker* free_w = nullptr;
    for (auto* w : s->workers)
      if (!w->busy) { free_w = w; break; }
    if (!free_w || s->queue.empty()) continue;
    Request* head = s->queue.front();
    std::vector<Request*> job;
    if (!head->res && head->n <= kSmallN && head->nrhs <= kSmallRhs) {
      // every queued small request of the head's kind, within the budget
      size_t bytes = 0;
      for (auto it = s->queue.begin(); it != s->queue.end() && (int)job.size() < kMaxBatch;) {
        Request* r = *it;
        if (!r->res && r->kind == head->kind && r->n <= kSmallN && r->nrhs <= kSmallRhs &&
            s->in_use + bytes + r->bytes <= s->budget) {
          bytes += r->bytes;
          job.push_back(r);
          it = s->queue.erase(it);
        } else {
          ++it;
        }
      }
      if (job.empty()) {
        s->cv_dispatch.wait_for(lk, std::chrono::milliseconds(1));
        continue;
      }
      s->in_use += bytes;
    } else {
      if (s->in_use + head->bytes > s->budget) {  // wait for memory to free up
        s->cv_dispatch.wait_for(lk, std::chrono::milliseconds(1));
        continue;
      }
      s->queue.pop_front();
      s->in_use += head->bytes;
      job.push_back(head);
    }
    free_w->busy = true;
    free_w->job = std::move(job);
    free_w->cv.notify_one();
  }
}

}  // namespace

extern "C" {

int egpu_server_create(int device, size_t hbm_budget_bytes, int slots, int mode, egpu_server* out) {
  if (!out || slots < 1 || slots > 64 || (mode != 0 && mode != 1) || hbm_budget_bytes == 0) return EGPU_ERR_ARG;
  *out = nullptr;
  auto* s = new (std::nothrow) egpu_server_s;
  if (!s) return EGPU_ERR_ALLOC;
  s->device = device;
  s->slots = slots;
  s->mode = mode;
  s->budget = hbm_budget_bytes;
  cudaSetDevice(device);
  // stream-ordered allocations come back to the pool, not to the driver
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    unsigned long long thr = hbm_budget_bytes;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  cudaGetLastError();
  for (int i = 0; i < slots; ++i) {
    auto* w = new egpu_server_s::Worker;
    int rc = egpu_create(&w->h, device);
    if (rc == EGPU_OK && cudaMalloc(reinterpret_cast<void**>(&w->flag), sizeof(int)) != cudaSuccess) {
      cudaGetLastError();
      egpu_destroy(w->h);
      rc = EGPU_ERR_ALLOC;
    }
    if (rc != EGPU_OK) {
      delete w;
      for (auto* x : s->workers) { cudaFree(x->flag); egpu_destroy(x->h); delete x; }
      delete s;
      return rc;
    }
    s->workers.push_back(w);
  }
  for (auto* w : s->workers) w->th = std::thread(worker_main, s, w);
  s->dispatcher = std::thread(dispatcher_main, s);
  *out = s;
  return EGPU_OK;
}

int egpu_server_set_mixed_min_n(egpu_server s, int n) {
  if (!s || n < 0) return EGPU_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  s->mixed_min_n = n;
  return EGPU_OK;
}

int egpu_server_set_tolerance(egpu_server s, double tol) {
  if (!s || !(tol > 0.0)) return EGPU_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  s->tol = tol;
  return EGPU_OK;
}

int egpu_server_submit(egpu_server s, int kind, int n, int nrhs, const double* A, int lda, const double* B, int ldb,
                       double* X, int ldx, unsigned long long* id) {
  if (!s || !id || (kind != 0 && kind != 1) || n < 1 || nrhs < 1 || !A || !B || !X || lda < n || ldb < n || ldx < n)
    return EGPU_ERR_ARG;
  auto* r = new (std::nothrow) Request;
  if (!r) return EGPU_ERR_ALLOC;
  r->kind = kind; r->n = n; r->nrhs = nrhs; r->A = A; r->lda = lda; r->B = B; r->ldb = ldb; r->X = X; r->ldx = ldx;
  r->bytes = request_bytes(s->mode, kind, n, nrhs);
  r->t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (r->bytes > s->budget) {
      delete r;
      return EGPU_ERR_ALLOC;  // can never be admitted
    }
    r->id = s->next_id++;
    s->all[r->id] = r;
    s->queue.push_back(r);
    *id = r->id;
  }
  s->cv_dispatch.notify_one();
  return EGPU_OK;
}

int egpu_server_register(egpu_server s, int kind, int n, const double* A, int lda, unsigned long long* mid) {
  if (!s || !mid || (kind != 0 && kind != 1) || n < 1 || !A || lda < n) return EGPU_ERR_ARG;
  auto* R = new (std::nothrow) Resident;
  if (!R) return EGPU_ERR_ALLOC;
  R->kind = kind;
  R->n = n;
  R->ld = std::max(32, (n + 31) / 32 * 32);
  R->bytes = 2 * sizeof(double) * (size_t)R->ld * n + sizeof(int) * (size_t)n;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->in_use + R->bytes > s->budget) {
      delete R;
      return EGPU_ERR_ALLOC;
    }
    s->in_use += R->bytes;
  }
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(s->device);
  cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&R->dA), sizeof(double) * R->ld * (size_t)n);
  if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&R->dF), sizeof(double) * R->ld * (size_t)n);
  if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&R->dpiv), sizeof(int) * (size_t)n);
  if (e == cudaSuccess)
    e = cudaMemcpy2D(R->dA, sizeof(double) * R->ld, A, sizeof(double) * lda, sizeof(double) * n, n,
                     cudaMemcpyHostToDevice);
  cudaSetDevice(prev);
  if (e != cudaSuccess) {
    cudaGetLastError();
    cudaFree(R->dA);
    cudaFree(R->dF);
    cudaFree(R->dpiv);
    std::lock_guard<std::mutex> lk(s->mu);
    s->in_use -= R->bytes;
    delete R;
    return EGPU_ERR_ALLOC;
  }
  std::lock_guard<std::mutex> lk(s->mu);
  R->mid = s->next_id++;
  s->resident[R->mid] = R;
  *mid = R->mid;
  return EGPU_OK;
}

int egpu_server_submit_resident(egpu_server s, unsigned long long mid, int nrhs, const double* B, int ldb, double* X,
                                int ldx, unsigned long long* id) {
  if (!s || !id || nrhs < 1 || !B || !X) return EGPU_ERR_ARG;
  auto* r = new (std::nothrow) Request;
  if (!r) return EGPU_ERR_ALLOC;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->resident.find(mid);
    if (it == s->resident.end() || ldb < it->second->n || ldx < it->second->n) {
      delete r;
      return EGPU_ERR_ARG;
    }
    Resident* R = it->second;
    r->res = R;
    r->kind = R->kind; r->n = R->n; r->nrhs = nrhs; r->B = B; r->ldb = ldb; r->X = X; r->ldx = ldx;
    r->bytes = sizeof(double) * (size_t)R->ld * nrhs;  // the right-hand side on the device
    if (r->bytes > s->budget) {
      delete r;
      return EGPU_ERR_ALLOC;
    }
    r->t_submit = Clock::now();
    ++R->users;
    r->id = s->next_id++;
    s->all[r->id] = r;
    s->queue.push_back(r);
    *id = r->id;
  }
  s->cv_dispatch.notify_one();
  return EGPU_OK;
}

int egpu_server_unregister(egpu_server s, unsigned long long mid) {
  if (!s) return EGPU_ERR_ARG;
  Resident* R = nullptr;
  {
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->resident.find(mid);
    if (it == s->resident.end()) return EGPU_ERR_ARG;
    R = it->second;
    s->cv_done.wait(lk, [&] { return R->users == 0; });
    s->resident.erase(it);
    s->in_use -= R->bytes;
  }
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(s->device);
  cudaFree(R->dA);
  cudaFree(R->dF);
  cudaFree(R->dpiv);
  cudaSetDevice(prev);
  delete R;
  return EGPU_OK;
}

int egpu_server_query(egpu_server s, unsigned long long id, int wait, int* done, int* status, double* latency_ms,
                      int* path, int* iters, double* berr) {
  if (!s) return EGPU_ERR_ARG;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->all.find(id);
  if (it == s->all.end()) return EGPU_ERR_ARG;
  Request* r = it->second;
  if (wait) s->cv_done.wait(lk, [&] { return r->done; });
  if (done) *done = r->done ? 1 : 0;
  if (r->done) {
    if (status) *status = r->status;
    if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
    if (path) *path = r->path;
    if (iters) *iters = r->iters;
    if (berr) *berr = r->berr;
  }
  return EGPU_OK;
}

int egpu_server_release(egpu_server s, unsigned long long id) {
  if (!s) return EGPU_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->all.find(id);
  if (it == s->all.end() || !it->second->done) return EGPU_ERR_ARG;
  delete it->second;
  s->all.erase(it);
  return EGPU_OK;
}

int egpu_server_drain(egpu_server s) {
  if (!s) return EGPU_ERR_ARG;
  std::unique_lock<std::mutex> lk(s->mu);
  s->cv_done.wait(lk, [&] {
    if (!s->queue.empty()) return false;
    for (auto* w : s->workers)
      if (w->busy) return false;
    return true;
  });
  return EGPU_OK;
}

int egpu_server_destroy(egpu_server s) {
  if (!s) return EGPU_OK;
  egpu_server_drain(s);
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_dispatch.notify_all();
  for (auto* w : s->workers) w->cv.notify_all();
  if (s->dispatcher.joinable()) s->dispatcher.join();
  for (auto* w : s->workers) {
    if (w->th.joinable()) w->th.join();
    if (w->flag) cudaFree(w->flag);
    egpu_destroy(w->h);
    delete w;
  }
  for (auto& kv : s->all) delete kv.second;
  cudaSetDevice(s->device);
  for (auto& kv : s->resident) {
    cudaFree(kv.second->dA);
    cudaFree(kv.second->dF);
    cudaFree(kv.second->dpiv);
    delete kv.second;
  }
  delete s;
  return EGPU_OK;
}

}  // extern "C"
