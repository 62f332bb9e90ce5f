// Host side of the FP64 GEMM engine: tensor-map encoding and launch.
#include <cudaTypedefs.h>

#include <mutex>

#include "dgemm.cuh"
#include "internal.h"

namespace egpu {

static PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
static std::once_flag g_encode_once;

static PFN_cuTensorMapEncodeTiled_v12000 encoder() {
  std::call_once(g_encode_once, [] {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  });
  return g_encode;
}

// 2-D tensor map over a column-major FP64 view: `inner` contiguous elements,
// `outer` columns `ld` elements apart.
static bool make_map(CUtensorMap* m, const double* base, uint64_t inner, uint64_t outer, uint64_t ld,
                     uint32_t box_inner, uint32_t box_outer, bool swz128) {
  auto enc = encoder();
  if (!enc) return false;
  cuuint64_t dims[2] = {inner, outer};
  cuuint64_t strides[1] = {ld * sizeof(double)};
  cuuint32_t box[2] = {box_inner, box_outer};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double*>(base), dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE,
                   swz128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

bool make_tma_2d(CUtensorMap* m, int dtype, const void* base, uint64_t inner, uint64_t outer,
                 uint64_t ld_bytes, uint32_t box_inner, uint32_t box_outer, bool swz128) {
  auto enc = encoder();
  if (!enc) return false;
  cuuint64_t dims[2] = {inner, outer};
  cuuint64_t strides[1] = {ld_bytes};
  cuuint32_t box[2] = {box_inner, box_outer};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = enc(m, (CUtensorMapDataType)dtype, 2, const_cast<void*>(base), dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE,
                   swz128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

static int sm_count_of_current_device() {
  static int cache[32] = {0};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 32 && cache[dev] > 0) return cache[dev];
  int n = 0;
  if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
  if (dev >= 0 && dev < 32) cache[dev] = n;
  return n;
}

bool tma_compatible(const void* p, long long ld) {
  return (reinterpret_cast<uintptr_t>(p) % 16 == 0) && (ld % 2 == 0) && ld > 0;
}

template <bool AK, bool BK, int WM, int WN>
static cudaError_t launch_variant(cudaStream_t st, const CUtensorMap& ma, const CUtensorMap& mb,
                                  const GemmParams& p, long long nblocks) {
  using S = GemmShape<WM, WN>;
  auto kern = dgemm_tma_kernel<AK, BK, WM, WN>;
  static unsigned attr_mask = 0;  // per template instance, one bit per device
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 32 || !(attr_mask & (1u << dev))) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, S::kSmemBytes);
    if (e != cudaSuccess) return e;
    if (dev < 32) attr_mask |= (1u << dev);
  }
  kern<<<(unsigned)nblocks, S::kThreads, S::kSmemBytes, st>>>(ma, mb, p);
  count_launch();
  return cudaGetLastError();
}


// ---- small products ------------------------------------------------------
// A product with only a few 128 x 64 tiles (a panel multiply or the next
// block column's update of a small factorization) leaves most of the GPU
// idle and is bound by the per-SM DMMA rate of the few CTAs it has.  This form spreads it over many more warps: each warp computes a
// 32 x 32 tile of C (2 x 4 DMMA m16n8k8 tiles) straight from global memory
// (L2), 16 k at a time with the next 16 in flight, and a CTA of WM x WN
// warps covers a (32 WM) x (32 WN) tile.  All of a CTA's loads come before a
// CTA barrier and its stores after it, so C may alias A when the CTA covers
// every column of C (WN * 32 >= N), or B when it covers every row.
struct SmallParams {
  const double* A;
  const double* B;
  double* C;
  long long lda, ldb, ldc;
  int M, N, K, tri, wm, wn;
  double alpha, beta;
  const DevStatus* status;
};

template <bool AK, bool BK>
__global__ void __launch_bounds__(128) dgemm_small_kernel(const SmallParams p) {
  if (p.status != nullptr && p.status->code != 0) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int row0 = (blockIdx.x * p.wm + warp % p.wm) * 32;
  const int col0 = (blockIdx.y * p.wn + warp / p.wm) * 32;
  // a warp whose tile is wholly outside C or outside the triangle has no work
  // but still meets the CTA barrier
  const bool live = row0 < p.M && col0 < p.N && !(p.tri == 1 && row0 + 31 < col0) && !(p.tri == 2 && row0 > col0 + 31);
  double acc[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int r = 0; r < 4; ++r) acc[i][j][r] = 0.0;
  if (live) {
    // this lane's rows of op(A) and columns of op(B), clamped (a row or column
    // past the edge is read at a valid address and multiplied by zero)
    const double* ar[4];
    const double* bc[4];
    bool am[4], bm[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {  // rows row0 + g + 8 q
      const int m = row0 + g + 8 * q;
      am[q] = m < p.M;
      ar[q] = p.A + (AK ? (long long)min(m, p.M - 1) * p.lda : (long long)min(m, p.M - 1));
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int n = col0 + 8 * j + g;
      bm[j] = n < p.N;
      bc[j] = p.B + (BK ? (long long)min(n, p.N - 1) * p.ldb : (long long)min(n, p.N - 1));
    }
    const long long as = AK ? 1 : p.lda, bs = BK ? 1 : p.ldb;  // k stride
    double af[4][4], bf[4][4];  // [k offset t, t+4, t+8, t+12][row / column slot]
    double an[4][4], bn[4][4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int k = t + 4 * u;
      const bool kin = k < p.K;
#pragma unroll
      for (int q = 0; q < 4; ++q) af[u][q] = (kin && am[q]) ? __ldg(ar[q] + k * as) : 0.0;
#pragma unroll
      for (int j = 0; j < 4; ++j) bf[u][j] = (kin && bm[j]) ? __ldg(bc[j] + k * bs) : 0.0;
    }
    for (int k0 = 0; k0 < p.K; k0 += 16) {
      const bool more = k0 + 16 < p.K;
      if (more) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int k = k0 + 16 + t + 4 * u;
          const bool kin = k < p.K;
#pragma unroll
          for (int q = 0; q < 4; ++q) an[u][q] = (kin && am[q]) ? __ldg(ar[q] + k * as) : 0.0;
#pragma unroll
          for (int j = 0; j < 4; ++j) bn[u][j] = (kin && bm[j]) ? __ldg(bc[j] + k * bs) : 0.0;
        }
      }
      // two k8 steps: k = k0 + {t, t+4} and k0 + 8 + {t, t+4}
#pragma unroll
      for (int s2 = 0; s2 < 2; ++s2) {
#pragma unroll
        for (int i = 0; i < 2; ++i) {
          // rows 16 i + g (slot 2 i) and 16 i + g + 8 (slot 2 i + 1)
          const double a4[4] = {af[2 * s2][2 * i], af[2 * s2][2 * i + 1], af[2 * s2 + 1][2 * i],
                                af[2 * s2 + 1][2 * i + 1]};
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const double b2[2] = {bf[2 * s2][j], bf[2 * s2 + 1][j]};
            dmma_16x8x8(acc[i][j], a4, b2);
          }
        }
      }
      if (more) {
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            af[u][q] = an[u][q];
            bf[u][q] = bn[u][q];
          }
      }
    }
  }
  // every load of the CTA is done before any store (C may alias A or B)
  __syncthreads();
  if (!live) return;
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int m = row0 + 16 * i + g + (r >= 2 ? 8 : 0);
        const int n = col0 + 8 * j + 2 * t + (r & 1);
        if (m >= p.M || n >= p.N) continue;
        if ((p.tri == 1 && m < n) || (p.tri == 2 && m > n)) continue;
        double* c = &p.C[m + (long long)n * p.ldc];
        *c = p.beta == 0.0 ? p.alpha * acc[i][j][r] : fma(p.beta, *c, p.alpha * acc[i][j][r]);
      }
}

// Byte ranges [lo, hi) of a column-major view (rows x cols, ld) in memory.
static bool views_overlap(const double* a, long long rows_a, long long cols_a, long long lda, const double* b,
                          long long rows_b, long long cols_b, long long ldb) {
  const uintptr_t a0 = reinterpret_cast<uintptr_t>(a), a1 = a0 + 8 * ((cols_a - 1) * lda + rows_a);
  const uintptr_t b0 = reinterpret_cast<uintptr_t>(b), b1 = b0 + 8 * ((cols_b - 1) * ldb + rows_b);
  return a0 < b1 && b0 < a1;
}

// The small form when the 128 x 64 tiles would not fill the SMs; returns
// EGPU_ERR_UNSUPPORTED when it does not apply (then the TMA engine runs).
static int launch_dgemm_small(cudaStream_t st, bool a_kmajor, bool b_kmajor, int M, int N, int K, double alpha,
                              const double* A, long long lda, const double* B, long long ldb, double beta, double* C,
                              long long ldc, int tri, DevStatus* status) {
  // only the smallest products (at most 40 of the engine's tiles, K <= 256):
  // between that and a full wave the TMA engine measured as fast or faster
  const long long big_tiles = (long long)((M + 127) / 128) * ((N + 63) / 64);
  if (big_tiles > 40 || K > 256) return EGPU_ERR_UNSUPPORTED;
  const bool alias_a = views_overlap(C, M, N, ldc, A, a_kmajor ? K : M, a_kmajor ? M : K, lda);
  const bool alias_b = views_overlap(C, M, N, ldc, B, b_kmajor ? K : N, b_kmajor ? N : K, ldb);
  int wm = 2, wn = 2;
  if (alias_a && alias_b) return EGPU_ERR_UNSUPPORTED;
  // in place only as the drivers use it: C is A (the same rows) or C is B
  // (column n of C is column n of op(B)^T)
  if (alias_a && !(C == A && ldc == lda && !a_kmajor)) return EGPU_ERR_UNSUPPORTED;
  if (alias_b && !(C == B && ldc == ldb && b_kmajor)) return EGPU_ERR_UNSUPPORTED;
  if (alias_a) {  // every column of C in one CTA
    if (N > 128) return EGPU_ERR_UNSUPPORTED;
    wn = (N + 31) / 32;
    wm = std::max(1, 4 / wn);
  } else if (alias_b) {  // every row of C in one CTA
    if (M > 128) return EGPU_ERR_UNSUPPORTED;
    wm = (M + 31) / 32;
    wn = std::max(1, 4 / wm);
  }
  SmallParams p;
  p.A = A; p.B = B; p.C = C; p.lda = lda; p.ldb = ldb; p.ldc = ldc;
  p.M = M; p.N = N; p.K = K; p.tri = tri; p.wm = wm; p.wn = wn; p.alpha = alpha; p.beta = beta; p.status = status;
  const dim3 grid((M + 32 * wm - 1) / (32 * wm), (N + 32 * wn - 1) / (32 * wn));
  const double lo_n = std::min(M, N), rect = tri == 1 ? std::max(0, M - N) : std::max(0, N - M);
  const double entries = tri == 0 ? (double)M * N : lo_n * (lo_n + 1) / 2 + rect * lo_n;
  TraceMark tm(st, beta == 0.0 ? kTraceTrsm : kTraceUpdate, 2.0 * entries * K,
               8.0 * ((double)M * K + (double)N * K + (beta == 0.0 ? 1.0 : 2.0) * entries));
  if (a_kmajor && b_kmajor) dgemm_small_kernel<true, true><<<grid, 32 * wm * wn, 0, st>>>(p);
  else if (a_kmajor) dgemm_small_kernel<true, false><<<grid, 32 * wm * wn, 0, st>>>(p);
  else if (b_kmajor) dgemm_small_kernel<false, true><<<grid, 32 * wm * wn, 0, st>>>(p);
  else dgemm_small_kernel<false, false><<<grid, 32 * wm * wn, 0, st>>>(p);
  count_launch();
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_last_error(e, "dgemm_small launch", __FILE__, __LINE__);
    return EGPU_ERR_CUDA;
  }
  return EGPU_OK;
}

// C = alpha * op(A) * op(B) + beta * C (tri: 0 full, 1 lower, 2 upper).
//   a_kmajor = false: A stored M x K column-major (op = NORMAL)
//   a_kmajor = true : A stored K x M column-major (op = TRANSPOSE)
//   b_kmajor = true : B stored K x N column-major (op = NORMAL)
//   b_kmajor = false: B stored N x K column-major (op = TRANSPOSE)
// wide = true selects a 128-column tile, which keeps whole 128-wide row panels
// inside one CTA (in-place multiply by an inverted triangle): 128 x 128 (8
// warps), or 64 x 128 (4 warps, 2 CTAs/SM) when A is MN-major and 128-row
// tiles would not fill the SMs twice over.
int launch_dgemm(cudaStream_t st, bool a_kmajor, bool b_kmajor, int M, int N, int K, double alpha,
                 const double* A, long long lda, const double* B, long long ldb, double beta, double* C,
                 long long ldc, int tri, bool wide, DevStatus* status) {
  if (M <= 0 || N <= 0) return EGPU_OK;
  if (K <= 0) return launch_scale(st, M, N, beta, C, ldc, tri);
  if (!tma_compatible(A, lda) || !tma_compatible(B, ldb)) return EGPU_ERR_ALIGN;
  if (tri != 0 && wide) return EGPU_ERR_ARG;
  {
    const int rc = launch_dgemm_small(st, a_kmajor, b_kmajor, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, tri,
                                      status);
    if (rc != EGPU_ERR_UNSUPPORTED) return rc;
  }
  const bool half = wide && !a_kmajor && (M + 127) / 128 < 2 * sm_count_of_current_device();
  const int BM = half ? 64 : 128, BN = wide ? 128 : 64;
  CUtensorMap ma, mb;
  // K-major: one {16 k, BM} box per stage; MN-major: BM / 16 boxes of
  // {16 m, 16 k} (both 128B-swizzled, see dgemm.cuh)
  bool ok = a_kmajor ? make_map(&ma, A, K, M, lda, kBK, BM, true) : make_map(&ma, A, M, K, lda, 16, kBK, true);
  ok = ok && (b_kmajor ? make_map(&mb, B, K, N, ldb, kBK, BN, true) : make_map(&mb, B, N, K, ldb, 16, kBK, true));
  if (!ok) return EGPU_ERR_TMA;
  GemmParams p;
  p.C = C; p.ldc = ldc; p.M = M; p.N = N; p.K = K; p.alpha = alpha; p.beta = beta; p.tri = tri;
  p.tiles_m = (M + BM - 1) / BM;
  p.tiles_n = (N + BN - 1) / BN;
  p.status = status;
  p.cvec = (reinterpret_cast<uintptr_t>(C) % 16 == 0) && (ldc % 2 == 0);
  long long nblocks;
  if (tri == 0) {
    nblocks = (long long)p.tiles_m * p.tiles_n;
  } else {
    nblocks = 0;
    for (int j = 0; j < p.tiles_n; ++j) {
      int lo = tri == 1 ? j / 2 : 0;
      int hi = tri == 1 ? p.tiles_m : std::min(j / 2 + 1, p.tiles_m);
      nblocks += std::max(0, hi - lo);
    }
  }
  // entries of C the product touches: the whole M x N block, or the lower
  // (tri 1) / upper (tri 2) trapezoid -- a launch over rows [c0, n) of block
  // columns [c0, c1) is a triangle on top of a rectangle
  const double lo_n = std::min(M, N), rect = tri == 1 ? std::max(0, M - N) : std::max(0, N - M);
  const double entries = tri == 0 ? (double)M * N : lo_n * (lo_n + 1) / 2 + rect * lo_n;
  const double flops = 2.0 * entries * K;
  const double bytes = 8.0 * ((double)M * K + (double)N * K + (beta == 0.0 ? 1.0 : 2.0) * entries);
  TraceMark tm(st, beta == 0.0 ? kTraceTrsm : kTraceUpdate, flops, bytes);
  cudaError_t e;
  if (half) {
    if (!b_kmajor) e = launch_variant<false, false, 1, 4>(st, ma, mb, p, nblocks);
    else e = launch_variant<false, true, 1, 4>(st, ma, mb, p, nblocks);
  } else if (wide) {
    if (!a_kmajor && !b_kmajor) e = launch_variant<false, false, 2, 4>(st, ma, mb, p, nblocks);
    else if (!a_kmajor && b_kmajor) e = launch_variant<false, true, 2, 4>(st, ma, mb, p, nblocks);
    else if (a_kmajor && !b_kmajor) e = launch_variant<true, false, 2, 4>(st, ma, mb, p, nblocks);
    else e = launch_variant<true, true, 2, 4>(st, ma, mb, p, nblocks);
  } else {
    if (!a_kmajor && !b_kmajor) e = launch_variant<false, false, 2, 2>(st, ma, mb, p, nblocks);
    else if (!a_kmajor && b_kmajor) e = launch_variant<false, true, 2, 2>(st, ma, mb, p, nblocks);
    else if (a_kmajor && !b_kmajor) e = launch_variant<true, false, 2, 2>(st, ma, mb, p, nblocks);
    else e = launch_variant<true, true, 2, 2>(st, ma, mb, p, nblocks);
  }
  if (e != cudaSuccess) {
    set_last_error(e, "dgemm launch", __FILE__, __LINE__);
    return EGPU_ERR_CUDA;
  }
  return EGPU_OK;
}

// C := beta * C on the (tri) region; used for K == 0 products.
__global__ void scale_kernel(int M, int N, double beta, double* C, long long ldc, int tri) {
  const long long total = (long long)M * N;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(idx % M), c = (int)(idx / M);
    if (tri == 1 && r < c) continue;
    if (tri == 2 && r > c) continue;
    double* p = C + (long long)c * ldc + r;
    *p = (beta == 0.0) ? 0.0 : beta * *p;
  }
}

int launch_scale(cudaStream_t st, int M, int N, double beta, double* C, long long ldc, int tri) {
  if (M <= 0 || N <= 0 || beta == 1.0) return EGPU_OK;
  long long total = (long long)M * N;
  int blocks = (int)std::min<long long>((total + 255) / 256, 148 * 16);
  scale_kernel<<<blocks, 256, 0, st>>>(M, N, beta, C, ldc, tri);
  count_launch();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_last_error(e, "scale launch", __FILE__, __LINE__);
    return EGPU_ERR_CUDA;
  }
  return EGPU_OK;
}

}  // namespace egpu
