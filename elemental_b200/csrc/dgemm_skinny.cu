// C += alpha * A * B for a tall-and-skinny product: A (M x K) column-major,
// B (K x N) column-major with N <= 64, C (M x N).  This is the residual
// r = b - A x of iterative refinement: HBM-bound at the FP64 tensor rate
// (every A element is used N times), so the design goal is to keep enough
// bytes in flight per SM to stream A: a CTA takes a 128-row block and a 1/S
// slice of K (split-K), runs a 4-stage ring of 16-byte cp.async.cg copies
// (128 x 32 of A, 32 x N of B per stage), multiplies with 16 x 8 x 8 DMMA
// fragments, and adds its partial block into C with FP64 atomics.
#include "internal.h"

namespace egpu {

namespace {

constexpr int kSgThreads = 256;
constexpr int kSgKC = 32;
constexpr int kSgLDA = 132;  // sA[a + k * 132]
constexpr int kSgLDB = 36;   // sB[k + c * 36]
constexpr int kSgMaxN = 64;
constexpr int kSgStages = 4;
constexpr int kSgStageA = kSgKC * kSgLDA;
constexpr int kSgStageB = kSgMaxN * kSgLDB;
constexpr int kSgStage = kSgStageA + kSgStageB;
constexpr int kSgSmemDoubles = kSgStages * kSgStage;

struct SgParams {
  const double* A;
  long long lda;
  const double* B;
  long long ldb;
  double* C;
  long long ldc;
  int M, N, K, kslice;
  double alpha;
  DevStatus* status;
};

// chunk [k0, k0 + 32) of the CTA's rows into stage buffers (zero outside)
__device__ __forceinline__ void sg_stage(double* sA, double* sB, const SgParams& p, int m0, int k0, int kend) {
  const int tid = threadIdx.x;
  for (int e = tid; e < 64 * kSgKC; e += kSgThreads) {  // row pairs
    const int a = 2 * (e & 63), k = e >> 6;
    double* d = &sA[a + k * kSgLDA];
    const int r = m0 + a, kk = k0 + k;
    if (kk < kend && r + 1 < p.M) cp_async16_cg(d, &p.A[r + (long long)kk * p.lda]);
    else {
      d[0] = (kk < kend && r < p.M) ? p.A[r + (long long)kk * p.lda] : 0.0;
      d[1] = 0.0;
    }
  }
  for (int e = tid; e < (kSgKC / 2) * p.N; e += kSgThreads) {  // k pairs
    const int k = 2 * (e & 15), c = e >> 4;
    double* d = &sB[k + c * kSgLDB];
    const int kk = k0 + k;
    if (kk + 1 < kend) cp_async16_cg(d, &p.B[kk + (long long)c * p.ldb]);
    else {
      d[0] = (kk < kend) ? p.B[kk + (long long)c * p.ldb] : 0.0;
      d[1] = 0.0;
    }
  }
  asm volatile("cp.async.commit_group;" ::: "memory");
}

}  // namespace

// NT: 8-column tiles of B and C (compile-time: a DMMA skipped under a
// run-time predicate still costs its issue slots).
template <int NT>
__global__ void __launch_bounds__(kSgThreads, 1) dgemm_skinny_kernel(SgParams p) {
  extern __shared__ double sm[];
  if (p.status != nullptr && ((volatile DevStatus*)p.status)->code != 0) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int m0 = blockIdx.x * 128;
  const int kbeg = blockIdx.y * p.kslice, kend = min(p.K, kbeg + p.kslice);
  if (kbeg >= kend) return;
  const int nch = (kend - kbeg + kSgKC - 1) / kSgKC;
  double acc[NT][4];
#pragma unroll
  for (int nt = 0; nt < NT; ++nt)
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[nt][q] = 0.0;
  // prologue: stages 0 .. S-2 in flight
#pragma unroll
  for (int s = 0; s < kSgStages - 1; ++s) {
    if (s < nch) sg_stage(sm + s * kSgStage, sm + s * kSgStage + kSgStageA, p, m0, kbeg + s * kSgKC, kend);
    else asm volatile("cp.async.commit_group;" ::: "memory");
  }
  for (int ch = 0; ch < nch; ++ch) {
    asm volatile("cp.async.wait_group %0;" ::"n"(kSgStages - 2) : "memory");
    __syncthreads();  // chunk ch landed for every thread; stage (ch-1) free for reuse
    const int nx = ch + kSgStages - 1;
    if (nx < nch) {
      double* st = sm + (nx % kSgStages) * kSgStage;
      sg_stage(st, st + kSgStageA, p, m0, kbeg + nx * kSgKC, kend);
    } else {
      asm volatile("cp.async.commit_group;" ::: "memory");
    }
    const double* sA = sm + (ch % kSgStages) * kSgStage;
    const double* sB = sA + kSgStageA;
#pragma unroll
    for (int kk = 0; kk < kSgKC; kk += 8) {
      double a[4];
      const int ra = 16 * warp + g;
      a[0] = sA[ra + (kk + t) * kSgLDA];
      a[1] = sA[ra + 8 + (kk + t) * kSgLDA];
      a[2] = sA[ra + (kk + t + 4) * kSgLDA];
      a[3] = sA[ra + 8 + (kk + t + 4) * kSgLDA];
#pragma unroll
      for (int nt = 0; nt < NT; ++nt) {
        double bf[2];
        bf[0] = sB[(kk + t) + (8 * nt + g) * kSgLDB];
        bf[1] = sB[(kk + t + 4) + (8 * nt + g) * kSgLDB];
        dmma_16x8x8(acc[nt], a, bf);
      }
    }
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");
#pragma unroll
  for (int nt = 0; nt < NT; ++nt)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int row = m0 + 16 * warp + g + ((q >= 2) ? 8 : 0), col = 8 * nt + 2 * t + (q & 1);
      if (row < p.M && col < p.N) atomicAdd(&p.C[row + (long long)col * p.ldc], p.alpha * acc[nt][q]);
    }
}

int launch_dgemm_skinny(cudaStream_t st, int M, int N, int K, double alpha, const double* A, long long lda,
                        const double* B, long long ldb, double* C, long long ldc, int sm_count, DevStatus* status) {
  if (M <= 0 || N <= 0 || K <= 0) return EGPU_OK;
  if (N > kSgMaxN || lda % 2 || ldb % 2 || reinterpret_cast<uintptr_t>(A) % 16 ||
      reinterpret_cast<uintptr_t>(B) % 16)
    return EGPU_ERR_UNSUPPORTED;
  const size_t smem = sizeof(double) * kSgSmemDoubles;
  const int nt = N <= 8 ? 1 : N <= 16 ? 2 : N <= 32 ? 4 : 8;
  const int ai = nt == 1 ? 0 : nt == 2 ? 1 : nt == 4 ? 2 : 3;
  void (*kern)(SgParams) = nt == 1 ? dgemm_skinny_kernel<1>
                           : nt == 2 ? dgemm_skinny_kernel<2>
                           : nt == 4 ? dgemm_skinny_kernel<4> : dgemm_skinny_kernel<8>;
  static bool attr[4] = {false, false, false, false};
  if (!attr[ai]) {
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
      cudaGetLastError();
      return EGPU_ERR_UNSUPPORTED;
    }
    attr[ai] = true;
  }
  const int mt = (M + 127) / 128;
  // about four CTAs per SM in total, K slices a multiple of the chunk
  int splits = std::max(1, (4 * sm_count + mt - 1) / mt);
  int kslice = (K + splits - 1) / splits;
  kslice = std::max(kSgKC * 4, (kslice + kSgKC - 1) / kSgKC * kSgKC);
  splits = (K + kslice - 1) / kslice;
  SgParams p{A, lda, B, ldb, C, ldc, M, N, K, kslice, alpha, status};
  TraceMark tm(st, kTraceUpdate, 2.0 * M * N * K, 8.0 * ((double)M * K + (double)K * N * mt + 2.0 * M * N * splits));
  kern<<<dim3(mt, splits), kSgThreads, smem, st>>>(p);
  count_launch();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_last_error(e, "dgemm_skinny launch", __FILE__, __LINE__);
    return EGPU_ERR_CUDA;
  }
  return EGPU_OK;
}

}  // namespace egpu
