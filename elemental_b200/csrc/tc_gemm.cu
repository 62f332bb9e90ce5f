// tcgen05 (5th-generation tensor core) GEMM for the mixed-precision
// factorizations: C (FP32, column-major) = alpha * sum_t A_t B_t^T + beta * C
// with A_t, B_t TF32 operands in K-major row-major buffers and an FP32
// accumulator in tensor memory (TMEM).
//
// Split precision: an FP32 operand x is carried as x = hi + lo with
// hi = tf32(x) and lo = tf32(x - hi); with terms = 3 the product is
// hi*hi + hi*lo + lo*hi, which keeps ~21 bits of the FP32 product (the
// dropped lo*lo term is 2^-22 relative).  terms = 1 is the plain TF32 product.
//
// Each CTA (one per SM at a time, 320 threads) takes a contiguous run of up
// to 8 output tiles of 128 x 128 (triangular tile lists for the symmetric
// rank-k update of a lower triangle):
//   warp 8 lane 0: TMA producer, 128-byte-swizzled 128 x 32 tiles into a
//                  ring of stages that runs across tile boundaries
//                  (mbarrier full/empty pairs, bounded waits);
//   warp 9 lane 0: MMA issuer, tcgen05.mma.cta_group::1.kind::tf32 128x128x8,
//                  four per 32-wide k tile and term, into one of two TMEM
//                  accumulators (256 columns) so that a tile's epilogue
//                  overlaps the next tile's MMAs;
//   warps 0-7    : epilogue, C rows read into registers before the
//                  accumulator is ready, then tcgen05.ld.32x32b of their 32
//                  TMEM lanes (warp e: lanes 32 (e % 4).., columns 64 (e / 4)..)
//                  and a coalesced store, one output row per thread.
#include <cudaTypedefs.h>

#include "internal.h"

namespace egpu {

namespace {

constexpr int kTcBM = 128, kTcBN = 128, kTcBK = 32;  // BK: 32 TF32 = one 128-byte swizzle row
constexpr int kTcThreads = 320;  // 8 epilogue warps, producer, MMA issuer
constexpr int kTcEpiWarps = 8;
constexpr int kTcProdWarp = 8, kTcMmaWarp = 9;
constexpr int kTcTileBytes = kTcBM * kTcBK * 4;  // 16 KiB per operand tile

template <int NT>
struct TcShape {
  static constexpr int kOps = NT == 1 ? 2 : 4;  // A_hi, B_hi (+ A_lo, B_lo)
  static constexpr int kStages = NT == 1 ? 6 : 3;
  static constexpr int kStageBytes = kOps * kTcTileBytes;
  static constexpr int kSmemBytes = kStages * kStageBytes + 1024 /*align*/ + 256 /*barriers*/;
};

struct TcParams {
  float* C;
  long long ldc;
  int M, N, K;
  float alpha, beta;
  int tri;  // 0 full, 1 lower trapezoid r >= c of C (M >= N; tiles i >= j, diagonal tiles masked)
  int tiles_m, tiles_n;
  DevStatus* status;
  // optional TF32 split of the result (sh == null: none): rows r >= srow0 of
  // C land in K-major rows sh[(r - srow0) * sldk + c], c < swidth (zero past N)
  float* sh;
  float* sl;
  long long sldk;
  int srow0, swidth;
};

__device__ __forceinline__ uint64_t sw128_kmajor_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);  // start address
  d |= (uint64_t)1 << 16;                   // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)(1024 >> 4) << 32;         // stride byte offset: 8 rows x 128 B
  d |= (uint64_t)1 << 46;                   // descriptor version (sm_100)
  d |= (uint64_t)2 << 61;                   // 128-byte swizzle
  return d;
}

// kind::tf32 instruction descriptor: FP32 accumulate, TF32 A/B, both K-major, M=128, N=128
constexpr uint32_t kTcIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(kTcBN >> 3) << 17) |
                              ((uint32_t)(kTcBM >> 4) << 24);

__device__ __forceinline__ void tc_mma(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(dtmem),
      "l"(adesc), "l"(bdesc), "r"(kTcIdesc), "r"(acc)
      : "memory");
}

__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 32 lanes x 32 columns of 32-bit TMEM words: thread i gets lane (base lane + i), columns col..col+31
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// tile index -> (tm, tn); lower-triangular lists enumerate tm >= tn column by column
__device__ __forceinline__ void tc_tile_of(const TcParams& p, int bid, int& tm, int& tn) {
  if (p.tri == 0) {
    tm = bid % p.tiles_m;
    tn = bid / p.tiles_m;
    return;
  }
  int j = 0, rem = bid;
  while (j < p.tiles_n && rem >= p.tiles_m - j) { rem -= p.tiles_m - j; ++j; }
  tn = j;
  tm = j + rem;
}

}  // namespace

template <int NT>
__global__ void __maxnreg__(200) tc_gemm_kernel(const __grid_constant__ CUtensorMap mah,
                                                                 const __grid_constant__ CUtensorMap mbh,
                                                                 const __grid_constant__ CUtensorMap mal,
                                                                 const __grid_constant__ CUtensorMap mbl,
                                                                 TcParams p, int ntiles, int per_cta) {
  using S = TcShape<NT>;
  extern __shared__ unsigned char tc_smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(tc_smem_raw) + 1023) & ~uintptr_t(1023));  // swizzle atoms: 1 KiB aligned
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + S::kStages * S::kStageBytes);
  uint64_t* empty = full + S::kStages;
  uint64_t* tfull = empty + S::kStages;  // [2] accumulator ready
  uint64_t* tempty = tfull + 2;          // [2] accumulator drained (8 epilogue warps arrive)
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tempty + 2);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (p.status != nullptr && ((volatile DevStatus*)p.status)->code != 0) return;  // uniform
  const int KT = (p.K + kTcBK - 1) / kTcBK;
  // a contiguous run of `per_cta` tiles per CTA: CTAs retire every few tiles,
  // so kernels of a higher-priority stream (the look-ahead panel chain) get
  // SMs between them instead of waiting for the whole update
  const int t_first = blockIdx.x * per_cta, t_end = min(ntiles, t_first + per_cta);

  if (tid == 0) {
    for (int s = 0; s < S::kStages; ++s) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
    for (int a = 0; a < 2; ++a) { mbar_init(&tfull[a], 1); mbar_init(&tempty[a], kTcEpiWarps); }
    *abort_flag = 0;
    fence_mbar_init();
  }
  if (warp == kTcMmaWarp) {  // 256 TMEM columns: two 128 x 128 FP32 accumulators
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 256;" ::"r"(smem_u32(tmem_slot))
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == kTcProdWarp) {
    if (lane == 0) {  // ---- TMA producer
      tma_prefetch_desc(&mah);
      tma_prefetch_desc(&mbh);
      if (NT == 3) { tma_prefetch_desc(&mal); tma_prefetch_desc(&mbl); }
      int g = 0;
      for (int t = t_first; t < t_end && !*abort_flag; ++t) {
        int tm, tn;
        tc_tile_of(p, t, tm, tn);
        const int m0 = tm * kTcBM, n0 = tn * kTcBN;
        for (int kt = 0; kt < KT; ++kt, ++g) {
          const int s = g % S::kStages;
          const uint32_t ph = (uint32_t)(g / S::kStages) & 1u;
          if (!mbar_wait_bounded(&empty[s], ph ^ 1u)) { *abort_flag = 1; set_status(p.status, kTimeout, 101); break; }
          unsigned char* st = smem + s * S::kStageBytes;
          mbar_expect_tx(&full[s], S::kStageBytes);
          const int k0 = kt * kTcBK;
          tma_load_2d(st, &mah, &full[s], k0, m0);
          tma_load_2d(st + kTcTileBytes, &mbh, &full[s], k0, n0);
          if (NT == 3) {
            tma_load_2d(st + 2 * kTcTileBytes, &mal, &full[s], k0, m0);
            tma_load_2d(st + 3 * kTcTileBytes, &mbl, &full[s], k0, n0);
          }
        }
      }
    }
  } else if (warp == kTcMmaWarp) {
    if (lane == 0) {  // ---- MMA issuer
      int g = 0, i = 0;
      for (int t = t_first; t < t_end && !*abort_flag; ++t, ++i) {
        const int a = i & 1;
        const uint32_t acc_addr = tmem + (uint32_t)(a * kTcBN);
        if (!mbar_wait_bounded(&tempty[a], ((uint32_t)(i >> 1) & 1u) ^ 1u)) {
          *abort_flag = 1; set_status(p.status, kTimeout, 104); break;
        }
        tc_fence_after();
        for (int kt = 0; kt < KT; ++kt, ++g) {
          const int s = g % S::kStages;
          const uint32_t ph = (uint32_t)(g / S::kStages) & 1u;
          if (!mbar_wait_bounded(&full[s], ph)) { *abort_flag = 1; set_status(p.status, kTimeout, 102); break; }
          tc_fence_after();
          const uint32_t st = smem_u32(smem + s * S::kStageBytes);
          const uint64_t ah = sw128_kmajor_desc(st), bh = sw128_kmajor_desc(st + kTcTileBytes);
          const uint64_t al = sw128_kmajor_desc(st + 2 * kTcTileBytes), bl = sw128_kmajor_desc(st + 3 * kTcTileBytes);
#pragma unroll
          for (int kk = 0; kk < kTcBK / 8; ++kk) {  // 8 TF32 = 32 bytes per MMA along K
            const uint64_t adv = (uint64_t)((kk * 32) >> 4);
            tc_mma(acc_addr, ah + adv, bh + adv, (kt | kk) != 0);
            if (NT == 3) {
              tc_mma(acc_addr, ah + adv, bl + adv, 1u);
              tc_mma(acc_addr, al + adv, bh + adv, 1u);
            }
          }
          tc_commit(&empty[s]);  // stage free once these MMAs have read it
        }
        tc_commit(&tfull[a]);  // accumulator a complete
      }
    }
  } else {
    // ---- epilogue: warp e reads TMEM lanes 32 (e % 4) .. (its quarter) and
    // columns 64 (e / 4) .. of each tile; each thread owns one output row.
    const int q = warp & 3, half = warp >> 2;
    int i = 0;
    for (int t = t_first; t < t_end; ++t, ++i) {
      int tm, tn;
      tc_tile_of(p, t, tm, tn);
      const int m0 = tm * kTcBM, n0 = tn * kTcBN + half * 64;
      const int r = m0 + q * 32 + lane;
      const int a = i & 1;
      // columns n0 + j, j < jmax, of row r are written (bounds, lower triangle)
      int jmax = r < p.M ? min(64, p.N - n0) : 0;
      if (p.tri) jmax = min(jmax, r - n0 + 1);
      float* cbase = p.C + (long long)n0 * p.ldc + (r < p.M ? r : 0);
      // this thread's 64 C entries in flight while the MMAs run
      float cv[64];
      {
        const float* cp = cbase;
#pragma unroll
        for (int j = 0; j < 64; ++j, cp += p.ldc) cv[j] = (p.beta != 0.0f && j < jmax) ? *cp : 0.0f;
      }
      const bool have = __all_sync(0xffffffffu, mbar_wait_bounded(&tfull[a], (uint32_t)(i >> 1) & 1u));
      if (!have) {
        if (lane == 0) { *abort_flag = 1; set_status(p.status, kTimeout, 103); }
        break;
      }
      tc_fence_after();
      const bool split = p.sh != nullptr && r >= p.srow0 && r < p.M;
#pragma unroll
      for (int c0 = 0; c0 < 64; c0 += 32) {
        float v[32];
        tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(a * kTcBN + half * 64 + c0), v);
        float* cp;  // opaque copy of the base: keeps the load addresses from staying live
        asm volatile("mov.b64 %0, %1;" : "=l"(cp) : "l"(cbase + (long long)c0 * p.ldc));
#pragma unroll
        for (int j = 0; j < 32; ++j, cp += p.ldc) {
          v[j] = c0 + j < jmax ? fmaf(p.alpha, v[j], p.beta * cv[c0 + j]) : 0.0f;
          if (c0 + j < jmax) *cp = v[j];
        }
        if (split && n0 + c0 < p.swidth) {  // the result's TF32 hi/lo split, 16-byte stores
          float* sh = p.sh + (long long)(r - p.srow0) * p.sldk + (n0 + c0);
          float* sl = p.sl + (long long)(r - p.srow0) * p.sldk + (n0 + c0);
#pragma unroll
          for (int j4 = 0; j4 < 32; j4 += 4) {
            float4 h4, l4;
            h4.x = tf32_rna(v[j4]);     l4.x = tf32_rna(v[j4] - h4.x);
            h4.y = tf32_rna(v[j4 + 1]); l4.y = tf32_rna(v[j4 + 1] - h4.y);
            h4.z = tf32_rna(v[j4 + 2]); l4.z = tf32_rna(v[j4 + 2] - h4.z);
            h4.w = tf32_rna(v[j4 + 3]); l4.w = tf32_rna(v[j4 + 3] - h4.w);
            *reinterpret_cast<float4*>(sh + j4) = h4;
            *reinterpret_cast<float4*>(sl + j4) = l4;
          }
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&tempty[a])) : "memory");
      if (*abort_flag) break;
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == kTcMmaWarp) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 256;" ::"r"(tmem) : "memory");
  }
}

template <int NT>
static cudaError_t tc_launch_variant(cudaStream_t st, const CUtensorMap& mah, const CUtensorMap& mbh,
                                     const CUtensorMap& mal, const CUtensorMap& mbl, const TcParams& p,
                                     long long nblocks) {
  auto kern = tc_gemm_kernel<NT>;
  static unsigned attr_mask = 0;
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 32 || !(attr_mask & (1u << dev))) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, TcShape<NT>::kSmemBytes);
    if (e != cudaSuccess) return e;
    if (dev < 32) attr_mask |= (1u << dev);
  }
  int dev_sms = 148;
  cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, dev);
  const int per_cta = (int)std::max<long long>(1, std::min<long long>(8, nblocks / (4LL * dev_sms)));
  const unsigned grid = (unsigned)((nblocks + per_cta - 1) / per_cta);
  kern<<<grid, kTcThreads, TcShape<NT>::kSmemBytes, st>>>(mah, mbh, mal, mbl, p, (int)nblocks, per_cta);
  count_launch();
  return cudaGetLastError();
}

int launch_tc_gemm(cudaStream_t st, int M, int N, int K, float alpha, const float* Ahi, const float* Alo,
                   const float* Bhi, const float* Blo, long long ldk, float beta, float* C, long long ldc, int tri,
                   int terms, DevStatus* status, float* Sh, float* Sl, long long sldk, int srow0, int swidth) {
  if (M <= 0 || N <= 0 || K <= 0) return M <= 0 || N <= 0 ? EGPU_OK : EGPU_ERR_ARG;
  if (terms != 1 && terms != 3) return EGPU_ERR_ARG;
  if (Sh != nullptr &&
      (Sl == nullptr || sldk % 32 != 0 || swidth > sldk || swidth < std::min(N, (int)sldk) ||
       reinterpret_cast<uintptr_t>(Sh) % 16 != 0 || reinterpret_cast<uintptr_t>(Sl) % 16 != 0))
    return EGPU_ERR_ARG;
  if (tri == 1 && M < N) return EGPU_ERR_ARG;  // lower trapezoid: rows >= columns
  if (ldk < K || ldk % 4 != 0) return EGPU_ERR_ALIGN;
  for (const float* q : {Ahi, Bhi, terms == 3 ? Alo : Ahi, terms == 3 ? Blo : Bhi})
    if (q == nullptr || reinterpret_cast<uintptr_t>(q) % 16 != 0) return EGPU_ERR_ALIGN;
  CUtensorMap mah, mbh, mal, mbl;
  const uint64_t ldb = (uint64_t)ldk * sizeof(float);
  bool ok = make_tma_2d(&mah, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, Ahi, K, M, ldb, kTcBK, kTcBM, true) &&
            make_tma_2d(&mbh, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, Bhi, K, N, ldb, kTcBK, kTcBN, true);
  if (ok && terms == 3)
    ok = make_tma_2d(&mal, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, Alo, K, M, ldb, kTcBK, kTcBM, true) &&
         make_tma_2d(&mbl, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, Blo, K, N, ldb, kTcBK, kTcBN, true);
  else {
    mal = mah;
    mbl = mbh;
  }
  if (!ok) return EGPU_ERR_TMA;
  TcParams p;
  p.C = C; p.ldc = ldc; p.M = M; p.N = N; p.K = K; p.alpha = alpha; p.beta = beta; p.tri = tri;
  p.tiles_m = (M + kTcBM - 1) / kTcBM;
  p.tiles_n = (N + kTcBN - 1) / kTcBN;
  p.status = status;
  p.sh = Sh; p.sl = Sl; p.sldk = sldk; p.srow0 = srow0; p.swidth = swidth;
  long long nblocks = (long long)p.tiles_m * p.tiles_n;
  if (tri) {  // tiles on or below the diagonal: column j holds tiles j .. tiles_m-1
    nblocks = 0;
    for (int j = 0; j < p.tiles_n; ++j) nblocks += p.tiles_m - j;
  }
  const double flops = (tri ? (double)N * (N + 1) + 2.0 * (double)(M - N) * N : 2.0 * M * N) * K * terms;
  const double bytes = 4.0 * terms * ((double)M * K + (double)N * K) / (terms == 3 ? 1.5 : 1.0) +
                       4.0 * (beta == 0.0f ? 1.0 : 2.0) * M * N * (tri ? 0.5 : 1.0);
  TraceMark tm(st, kTraceTc, flops, bytes);
  cudaError_t e = terms == 1 ? tc_launch_variant<1>(st, mah, mbh, mal, mbl, p, nblocks)
                             : tc_launch_variant<3>(st, mah, mbh, mal, mbl, p, nblocks);
  if (e != cudaSuccess) {
    set_last_error(e, "tc_gemm launch", __FILE__, __LINE__);
    return EGPU_ERR_CUDA;
  }
  return EGPU_OK;
}

}  // namespace egpu
