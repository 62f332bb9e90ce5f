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
