// Triangular solve X := inv(T) X with few right-hand sides (nrhs <= 64), the
// Trsm(LEFT, ...) calls of cholesky::SolveAfter (Cholesky/SolveAfter.hpp:
// 20-75) and lu::SolveAfter (LU/SolveAfter.hpp:101-146), in one cooperative
// launch.  The triangle T is described by the stored matrix A and two flags:
//   amode 0: T's block (r, j) is A's block (r, j)        (T = A)
//   amode 1: T's block (r, j) is A's block (j, r)^T      (T = A^T)
//   bwd    : T is upper triangular (solve from the last block up)
// so lower L x = b is (fwd, 0), L^T x = b is (bwd, 1), U^T x = b is (fwd, 1)
// and U x = b is (bwd, 0).  Winv holds inv(A_rr) of every diagonal block
// (transposed on use when amode is 1).
//
// Block rows of X (nb rows each) are owned round-robin by the CTAs; a CTA
// processes its block rows in solve order, left-looking: acc = B_r -
// sum_j T(r, j) X_j over the blocks j already solved, then X_r = inv(T_rr)
// acc with the pre-inverted diagonal block, and publishes X_r with a release
// flag.  Each off-diagonal block is read once, so the sweep streams the
// triangle from HBM once while the dependency chain only waits on flags
// (bounded spins), not on kernel boundaries.  The first chunk of each
// off-diagonal block is requested before the wait for the X block it
// multiplies.
//
// Prescaled form (Y != NULL): A holds the off-diagonal blocks already
// multiplied by the inverse of the diagonal block of the column they act on,
// M(r, j) = T(r, j) inv(T_jj).  Then z_r = b_r - sum_j M(r, j) z_j needs no
// inverse on the dependency chain: a CTA publishes z_r (in X) as soon as the
// sum is done and forms Y_r = inv(T_rr) z_r afterwards.
//
// Products are 16 x 8 x 8 DMMA fragments from shared memory: the 128 x 32
// chunk of the block (ld 132, or its transpose with ld 36: conflict-free
// fragment loads) and the 32 x nrhs chunk of X_j (ld 36), two cp.async stages
// of 16-byte copies.  Requires nrhs <= 64, nb <= 128 even, lda and ldx even,
// A, Winv, X (and Y) 16-byte aligned.
#include "internal.h"

namespace egpu {

namespace {

constexpr int kTsThreads = 256;  // 8 warps: warp w owns rows 16w .. 16w+15 of the block
constexpr int kTsKC = 32;        // k chunk
constexpr int kTsLDA = 132;      // column-major chunk [a + k * 132]
constexpr int kTsLDK = 36;       // transposed chunk [k + a * 36]
constexpr int kTsLDX = 36;
constexpr int kTsMaxRhs = 64;
constexpr int kTsStageA = 128 * kTsLDK > kTsKC * kTsLDA ? 128 * kTsLDK : kTsKC * kTsLDA;  // doubles
constexpr int kTsStageX = kTsMaxRhs * kTsLDX;       // doubles: the X chunk, [k + c * 36]
constexpr int kTsStage = kTsStageA + kTsStageX;
constexpr int kTsAccLD = 132;                       // acc staging [a + c * 132]
constexpr int kTsSmemDoubles = 2 * kTsStage + kTsMaxRhs * kTsAccLD;

struct TsParams {
  const double* L;
  long long lda;
  const double* Winv;  // block i at Winv + i*nb*nb, ld nb
  double* X;
  long long ldx;
  double* Y;  // prescaled form: X_r receives the unscaled block (published), Y_r = inv(T_rr) X_r
  int n, nrhs, nb, nblk, bwd, amode;
  int* flags;
  int epoch;
  DevStatus* status;
};

// block row of solve step s
__device__ __forceinline__ int ts_block(const TsParams& p, int s) { return p.bwd ? p.nblk - 1 - s : s; }

// Stage the k chunk [k0, k0+32) of an m x K operand A (m <= 128 rows) into
// shared memory with 16-byte .cg copies.  amode 0: A(a, k) = G[a + k lda]
// (column-major block), kept as sA[a + k * 132]; amode 1: A(a, k) =
// G[k + a lda] (the transpose of a column-major block), kept as
// sA[k + a * 36].  Out-of-range entries are zero.  lda even, G 16-byte
// aligned, k0 even.
__device__ __forceinline__ void ts_stage_a(double* sA, const double* G, long long lda, int amode, int m, int K,
                                           int k0) {
  const int tid = threadIdx.x;
  if (amode == 0) {
    for (int e = tid; e < 64 * kTsKC; e += kTsThreads) {  // row pairs
      const int a = 2 * (e & 63), k = e >> 6;
      double* d = &sA[a + k * kTsLDA];
      const double* src = &G[a + (long long)(k0 + k) * lda];
      if (k0 + k < K && a + 1 < m) cp_async16_cg(d, src);
      else {
        d[0] = (k0 + k < K && a < m) ? src[0] : 0.0;
        d[1] = 0.0;
      }
    }
  } else {
    for (int e = tid; e < 128 * (kTsKC / 2); e += kTsThreads) {  // k pairs
      const int k = 2 * (e & 15), a = e >> 4;
      double* d = &sA[k + a * kTsLDK];
      const double* src = &G[(k0 + k) + (long long)a * lda];
      if (a < m && k0 + k + 1 < K) cp_async16_cg(d, src);
      else {
        d[0] = (a < m && k0 + k < K) ? src[0] : 0.0;
        d[1] = 0.0;
      }
    }
  }
}

// The matching rows [k0, k0+32) of X (K x nrhs) into sX[k + c * 36].
__device__ __forceinline__ void ts_stage_x(double* sX, int K, int k0, const double* Xg, long long ldx, int nrhs,
                                           bool x_shared) {
  // X rows in pairs: 16-byte .cg copies (L2, never a stale L1 line of a block
  // another CTA has just published); ldx even and X 16-byte aligned
  for (int e = threadIdx.x; e < (kTsKC / 2) * nrhs; e += kTsThreads) {
    const int k = 2 * (e & 15), c = e >> 4;
    double* d = &sX[k + c * kTsLDX];
    const double* src = &Xg[(k0 + k) + (long long)c * ldx];
    if (x_shared) {  // operand staged in this CTA's shared memory
      d[0] = (k0 + k < K) ? src[0] : 0.0;
      d[1] = (k0 + k + 1 < K) ? src[1] : 0.0;
    } else if (k0 + k + 1 < K) {
      cp_async16_cg(d, src);
    } else {
      d[0] = (k0 + k < K) ? __ldcg(src) : 0.0;
      d[1] = 0.0;
    }
  }
}

// Bounded wait (thread 0) for *flag == epoch, then a CTA barrier.  Returns
// false (all threads) when the wait ran out.
__device__ __forceinline__ bool ts_wait_flag(const int* flag, int epoch, DevStatus* status) {
  __shared__ int s_ok;
  if (threadIdx.x == 0) {
    int ok = 1;
    long long it = 0;
    while (true) {
      int v;
      asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(flag) : "memory");
      if (v == epoch) break;
      if (++it > kSpinLimit) { ok = 0; set_status(status, kTimeout, 201); break; }
      if (it > 16) __nanosleep(64);
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// acc[nt] (16 x 8 fragments, rows 16 warp.., columns 8 nt..) += sign * A(m x K) * Xg(K x nrhs).
// With `flag` set, the first A chunk is requested before waiting for X to be published.
__device__ bool ts_product(double (&acc)[8][4], double sign, double* sm, const double* G, long long lda, int amode,
                           int m, int K, const double* Xg, long long ldx, int nrhs, bool x_shared,
                           const int* flag = nullptr, int epoch = 0, DevStatus* status = nullptr) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int nchunks = (K + kTsKC - 1) / kTsKC;
  const int ntn = (nrhs + 7) / 8;
  ts_stage_a(sm, G, lda, amode, m, K, 0);
  if (flag != nullptr && !ts_wait_flag(flag, epoch, status)) {
    asm volatile("cp.async.commit_group;\n cp.async.wait_group 0;" ::: "memory");
    return false;
  }
  ts_stage_x(sm + kTsStageA, K, 0, Xg, ldx, nrhs, x_shared);
  asm volatile("cp.async.commit_group;" ::: "memory");
  for (int ch = 0; ch < nchunks; ++ch) {
    double* cur = sm + (ch & 1) * kTsStage;
    if (ch + 1 < nchunks) {
      double* nxt = sm + ((ch + 1) & 1) * kTsStage;
      ts_stage_a(nxt, G, lda, amode, m, K, (ch + 1) * kTsKC);
      ts_stage_x(nxt + kTsStageA, K, (ch + 1) * kTsKC, Xg, ldx, nrhs, x_shared);
      asm volatile("cp.async.commit_group;" ::: "memory");
      asm volatile("cp.async.wait_group 1;" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;" ::: "memory");
    }
    __syncthreads();
    const double* sA = cur;
    const double* sX = cur + kTsStageA;
#pragma unroll
    for (int kk = 0; kk < kTsKC; kk += 8) {
      double a[4];
      const int ra = 16 * warp + g;
      if (amode == 0) {
        a[0] = sA[ra + (kk + t) * kTsLDA];
        a[1] = sA[ra + 8 + (kk + t) * kTsLDA];
        a[2] = sA[ra + (kk + t + 4) * kTsLDA];
        a[3] = sA[ra + 8 + (kk + t + 4) * kTsLDA];
      } else {
        a[0] = sA[(kk + t) + ra * kTsLDK];
        a[1] = sA[(kk + t) + (ra + 8) * kTsLDK];
        a[2] = sA[(kk + t + 4) + ra * kTsLDK];
        a[3] = sA[(kk + t + 4) + (ra + 8) * kTsLDK];
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) a[q] *= sign;
#pragma unroll
      for (int nt = 0; nt < 8; ++nt) {
        if (nt < ntn) {
          double bf[2];
          bf[0] = sX[(kk + t) + (8 * nt + g) * kTsLDX];
          bf[1] = sX[(kk + t + 4) + (8 * nt + g) * kTsLDX];
          dmma_16x8x8(acc[nt], a, bf);
        }
      }
    }
    __syncthreads();
  }
  return true;
}

}  // namespace

__global__ void __launch_bounds__(kTsThreads, 1) trsm_skinny_kernel(TsParams p) {
  extern __shared__ double sm[];
  double* accS = sm + 2 * kTsStage;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int ntn = (p.nrhs + 7) / 8;
  if (p.status != nullptr && ((volatile DevStatus*)p.status)->code != 0) return;
  for (int s = blockIdx.x; s < p.nblk; s += gridDim.x) {
    const int r = ts_block(p, s);
    const int r0 = r * p.nb, mr = min(p.nb, p.n - r0);
    double acc[8][4];
    // acc = B_r
#pragma unroll
    for (int nt = 0; nt < 8; ++nt)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int row = 16 * warp + g + ((q >= 2) ? 8 : 0), col = 8 * nt + 2 * t + (q & 1);
        acc[nt][q] = (nt < ntn && row < mr && col < p.nrhs) ? __ldcg(&p.X[(r0 + row) + (long long)col * p.ldx]) : 0.0;
      }
    // acc -= T(r, j) X_j for the blocks j solved before r
    for (int sj = 0; sj < s; ++sj) {
      const int j = ts_block(p, sj);
      const int j0 = j * p.nb, mj = min(p.nb, p.n - j0);
      const double* G = p.amode == 0 ? p.L + r0 + (long long)j0 * p.lda   // A(r, j)
                                     : p.L + j0 + (long long)r0 * p.lda;  // A(j, r)^T
      if (!ts_product(acc, -1.0, sm, G, p.lda, p.amode, mr, mj, p.X + j0, p.ldx, p.nrhs, false, &p.flags[j], p.epoch,
                      p.status))
        return;
    }
    if (p.Y != nullptr) {
      // prescaled form: publish z_r = acc first (the others need only z), then Y_r = inv(T_rr) z_r
#pragma unroll
      for (int nt = 0; nt < 8; ++nt)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int row = 16 * warp + g + ((q >= 2) ? 8 : 0), col = 8 * nt + 2 * t + (q & 1);
          if (nt < ntn && row < mr && col < p.nrhs) p.X[(r0 + row) + (long long)col * p.ldx] = acc[nt][q];
        }
      __threadfence();
      __syncthreads();
      if (tid == 0) asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(&p.flags[r]), "r"(p.epoch) : "memory");
    }
    // inv(T_rr) acc  (amode 1: inv(A_rr)^T = Winv_r^T)
#pragma unroll
    for (int nt = 0; nt < 8; ++nt)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int row = 16 * warp + g + ((q >= 2) ? 8 : 0), col = 8 * nt + 2 * t + (q & 1);
        if (nt < ntn) accS[row + col * kTsAccLD] = acc[nt][q];
        acc[nt][q] = 0.0;
      }
    __syncthreads();
    const double* Wr = p.Winv + (long long)r * p.nb * p.nb;
    ts_product(acc, 1.0, sm, Wr, p.nb, p.amode, mr, mr, accS, kTsAccLD, p.nrhs, true);
    double* out = p.Y != nullptr ? p.Y : p.X;
#pragma unroll
    for (int nt = 0; nt < 8; ++nt)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int row = 16 * warp + g + ((q >= 2) ? 8 : 0), col = 8 * nt + 2 * t + (q & 1);
        if (nt < ntn && row < mr && col < p.nrhs) out[(r0 + row) + (long long)col * p.ldx] = acc[nt][q];
      }
    if (p.Y == nullptr) {
      __threadfence();
      __syncthreads();
      if (tid == 0) asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(&p.flags[r]), "r"(p.epoch) : "memory");
    }
  }
}

size_t trsm_skinny_flag_bytes(int n, int nb) { return sizeof(int) * (size_t)((n + nb - 1) / nb) + 256; }

// flags: device array of ceil(n/nb) ints that persists across calls; epoch
// must differ from every value the flags hold (the caller counts calls).
int launch_trsm_skinny(cudaStream_t st, int bwd, int amode, int n, int nrhs, const double* L, long long lda,
                       const double* Winv, int nb, double* X, long long ldx, int* flags, int epoch, int sm_count,
                       DevStatus* status, double* Y) {
  if (n <= 0 || nrhs <= 0) return EGPU_OK;
  if (nrhs > kTsMaxRhs || nb > 128 || nb < 8 || nb % 2 != 0 || ldx % 2 != 0 || lda % 2 != 0 ||
      reinterpret_cast<uintptr_t>(X) % 16 != 0 || reinterpret_cast<uintptr_t>(L) % 16 != 0 ||
      reinterpret_cast<uintptr_t>(Winv) % 16 != 0 || reinterpret_cast<uintptr_t>(Y) % 16 != 0)
    return EGPU_ERR_UNSUPPORTED;
  TsParams p;
  p.L = L; p.lda = lda; p.Winv = Winv; p.X = X; p.ldx = ldx; p.Y = Y;
  p.n = n; p.nrhs = nrhs; p.nb = nb; p.nblk = (n + nb - 1) / nb; p.bwd = bwd; p.amode = amode;
  p.flags = flags; p.epoch = epoch; p.status = status;
  const size_t smem = sizeof(double) * kTsSmemDoubles;
  static bool attr = false;
  if (!attr) {
    if (cudaFuncSetAttribute(trsm_skinny_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess) {
      cudaGetLastError();
      return EGPU_ERR_UNSUPPORTED;
    }
    attr = true;
  }
  const int grid = std::min(p.nblk, sm_count);
  TraceMark tm(st, kTraceSolve, (double)n * n * nrhs, 4.0 * (double)n * n + 16.0 * n * nrhs);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(kTsThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr1[1];
  attr1[0].id = cudaLaunchAttributeCooperative;  // every CTA resident: the flag waits always end
  attr1[0].val.cooperative = 1;
  cfg.attrs = attr1;
  cfg.numAttrs = 1;
  cudaError_t e = cudaLaunchKernelEx(&cfg, trsm_skinny_kernel, p);
  count_launch();
  if (e != cudaSuccess) {
    set_last_error(e, "trsm_skinny launch", __FILE__, __LINE__);
    return EGPU_ERR_CUDA;
  }
  return EGPU_OK;
}

}  // namespace egpu
