// C += alpha * A * B for a tall-and-skinny product: A (M x K) column-major,
// B (K x N) column-major with N <= 64, C (M x N).  This is the residual
// r = b - A x of iterative refinement: at N = 32 the FP64 tensor rate and
// the HBM stream of A are about balanced, so the design keeps both busy: a
// CTA takes a 128-row block and a 1/S slice of K (split-K), a producer warp
// streams it through a 4-stage ring with one TMA box per operand chunk
// (A: 132 rows x 32, pitch 132; B: 36 x N, pitch 36 -- both 4 mod 16, so
// the 8-byte fragment loads are conflict-free; the extra rows are read and
// ignored, the parts past the matrix arrive as zeros), eight consumer warps
// multiply with 16 x 8 x 8 DMMA fragments and add the partial block into C
// with FP64 atomics.
#include "internal.h"

namespace egpu {

namespace {

constexpr int kSgConsumers = 256;
constexpr int kSgThreads = kSgConsumers + 32;  // + the producer warp
constexpr int kSgKC = 32;
constexpr int kSgLDA = 132;  // sA[a + kl * 132]
constexpr int kSgLDB = 36;   // sB[kl + c * 36]
constexpr int kSgMaxN = 64;
constexpr int kSgStages = 4;
constexpr int kSgStageA = kSgKC * kSgLDA;
constexpr int kSgStageB = kSgMaxN * kSgLDB;
constexpr int kSgStage = kSgStageA + kSgStageB;
constexpr int kSgSmemDoubles = kSgStages * kSgStage;
static_assert((kSgStage * 8) % 128 == 0 && (kSgStageA * 8) % 128 == 0, "stage parts start on 128-byte boundaries");

struct SgParams {
  double* C;
  long long ldc;
  int M, N, K, kslice;
  double alpha;
  DevStatus* status;
};

}  // namespace

// NT: 8-column tiles of B and C (compile-time: a DMMA skipped under a
// run-time predicate still costs its issue slots).
template <int NT>
__global__ void __launch_bounds__(kSgThreads, 1)
    dgemm_skinny_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
                        SgParams p) {
  extern __shared__ __align__(128) double sm[];
  __shared__ __align__(8) uint64_t full[kSgStages], empty[kSgStages];
  __shared__ int s_go;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int m0 = blockIdx.x * 128;
  const int kbeg = blockIdx.y * p.kslice, kend = min(p.K, kbeg + p.kslice);
  const int nch = (kend - kbeg + kSgKC - 1) / kSgKC;
  if (tid == 0) {
    for (int i = 0; i < kSgStages; ++i) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], kSgConsumers / 32);
    }
    fence_mbar_init();
    int go = (p.status == nullptr || ((volatile DevStatus*)p.status)->code == 0) && nch > 0;
    if (go && smem_u32(sm) % 128 != 0) {  // no TMA into a misaligned stage
      set_status(p.status, kTimeout, 204);
      go = 0;
    }
    s_go = go;
  }
  __syncthreads();
  if (!s_go) return;
  if (warp == kSgConsumers / 32) {
    // producer: one lane issues both boxes of each chunk
    if (lane != 0) return;
    tma_prefetch_desc(&mapA);
    tma_prefetch_desc(&mapB);
    const uint32_t bytes = (uint32_t)(8 * (kSgLDA * kSgKC + kSgLDB * p.N));
    for (int ch = 0; ch < nch; ++ch) {
      const int slot = ch % kSgStages;
      if (ch >= kSgStages && !mbar_wait_bounded(&empty[slot], ((uint32_t)(ch / kSgStages) & 1u) ^ 1u)) {
        set_status(p.status, kTimeout, 221);
        return;
      }
      double* st = sm + slot * kSgStage;
      const int k0 = kbeg + ch * kSgKC;
      mbar_expect_tx(&full[slot], bytes);
      tma_load_2d(st, &mapA, &full[slot], m0, k0);
      tma_load_2d(st + kSgStageA, &mapB, &full[slot], k0, 0);
    }
    return;
  }
  const int g = lane >> 2, t = lane & 3;
  double acc[NT][4];
#pragma unroll
  for (int nt = 0; nt < NT; ++nt)
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[nt][q] = 0.0;
  for (int ch = 0; ch < nch; ++ch) {
    const int slot = ch % kSgStages;
    if (!mbar_wait_bounded(&full[slot], (uint32_t)(ch / kSgStages) & 1u)) {
      if (lane == 0) set_status(p.status, kTimeout, 222);
      return;
    }
    const double* sA = sm + slot * kSgStage;
    const double* sB = sA + kSgStageA;
    // the slice's last chunk may reach past kend only at the end of K,
    // where the boxes read zeros
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
    __syncwarp();
    // the slot's refill is a TMA write: order this warp's reads of it first
    if (lane == 0) {
      fence_proxy_async_smem();
      mbar_arrive(&empty[slot]);
    }
  }
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
  CUtensorMap mapA, mapB;
  if (!make_tma_2d(&mapA, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, A, M, K, 8ull * lda, kSgLDA, kSgKC, false) ||
      !make_tma_2d(&mapB, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, B, K, N, 8ull * ldb, kSgLDB, (uint32_t)N, false))
    return EGPU_ERR_UNSUPPORTED;
  const size_t smem = sizeof(double) * kSgSmemDoubles;
  const int nt = N <= 8 ? 1 : N <= 16 ? 2 : N <= 32 ? 4 : 8;
  const int ai = nt == 1 ? 0 : nt == 2 ? 1 : nt == 4 ? 2 : 3;
  void (*kern)(const CUtensorMap, const CUtensorMap, SgParams) = nt == 1   ? dgemm_skinny_kernel<1>
                                                                 : nt == 2 ? dgemm_skinny_kernel<2>
                                                                 : nt == 4 ? dgemm_skinny_kernel<4>
                                                                           : dgemm_skinny_kernel<8>;
  static bool attr[4] = {false, false, false, false};
  if (!attr[ai]) {
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
      cudaGetLastError();
      return EGPU_ERR_UNSUPPORTED;
    }
    attr[ai] = true;
  }
  const int mt = (M + 127) / 128;
  // about four CTAs per SM in total, K slices a multiple of four chunks (a
  // chunk never straddles two slices)
  int splits = std::max(1, (4 * sm_count + mt - 1) / mt);
  int kslice = (K + splits - 1) / splits;
  kslice = std::max(kSgKC * 4, (kslice + kSgKC - 1) / kSgKC * kSgKC);
  splits = (K + kslice - 1) / kslice;
  SgParams p{C, ldc, M, N, K, kslice, alpha, status};
  TraceMark tm(st, kTraceUpdate, 2.0 * M * N * K, 8.0 * ((double)M * K + (double)K * N * mt + 2.0 * M * N * splits));
  kern<<<dim3(mt, splits), kSgThreads, smem, st>>>(mapA, mapB, p);
  count_launch();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_last_error(e, "dgemm_skinny launch", __FILE__, __LINE__);
    return EGPU_ERR_CUDA;
  }
  return EGPU_OK;
}

}  // namespace egpu
