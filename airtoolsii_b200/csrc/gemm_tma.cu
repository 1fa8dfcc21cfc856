// tcgen05 GEMM with TMA operand loads (K-major A and B).
//
// Two operand sources share one kernel:
//  * MODE_DENSE: A [M][lda] and B [N][ldb] row-major bf16 matrices, 2D
//    tensor maps, box {KS, 128} and {KS, BN};
//  * MODE_CONV: the implicit 3x3 convolution of an NHWC bf16 image X
//    [B][H][W][C]: a 4D tensor map (C, W, H, B) whose box {KS, bw, bh, bb}
//    (bw*bh*bb = 128 pixels, a rectangle of consecutive pixels) is loaded at
//    the tile origin shifted by the tap (dw, dh); out-of-image coordinates
//    read as zero, which is the convolution's zero padding.  Stage k is tap
//    k / (C/KS), channels (k % (C/KS))*KS.. +KS; the weights W[N][ldb] carry
//    the same K index (tap*C + ci).
//
// A stage holds KS = SW/2 K elements (SW = 128, 64 or 32 bytes per row) in
// the canonical K-major swizzled UMMA layout that TMA writes with the
// matching CU_TENSOR_MAP_SWIZZLE_*: rows of SW bytes, 8-row atoms of 8*SW
// bytes (SBO), 16-byte chunks XOR-swizzled by row; each K=16 MMA step
// advances the descriptor start address by 32 bytes.
//
// Roles (128 threads): thread 0 waits for a free stage and issues its two
// TMA loads onto the stage's `full` mbarrier (expect-tx bytes); thread 32
// waits for `full`, issues the tcgen05.mma instructions and commits them to
// the stage's `empty` mbarrier, and after the last stage to `done`; then all
// four warps drain TMEM through gemm_epilogue.  No multicast.
#include <cuda.h>
#include <cudaTypedefs.h>

#include "umma.cuh"

namespace airt {

namespace {

using namespace umma;

enum { MODE_DENSE = 0, MODE_CONV = 1 };

struct ConvGeo {
  int W, H, cchunks;  // image width, height, C / KS
};

constexpr uint32_t stage_bytes(int BN, int SW) {
  return (((uint32_t)(BM + BN) * (uint32_t)SW) + 1023u) & ~1023u;
}

// About 100 KB per CTA (two CTAs per SM), at least 2 and at most 8 stages;
// stages above 40 KB take four stages and one CTA per SM.
constexpr int tma_stages(int BN, int SW) {
  return stage_bytes(BN, SW) > 40960u ? 4
         : (int)(102400u / stage_bytes(BN, SW)) > 8 ? 8
         : (int)(102400u / stage_bytes(BN, SW)) < 2 ? 2
                                                     : (int)(102400u / stage_bytes(BN, SW));
}

__device__ __forceinline__ void expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void tma2d(uint32_t dst, const CUtensorMap *map, int x, int y, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, "
      "%3}], [%4];" ::"r"(dst),
      "l"(map), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void tma4d(uint32_t dst, const CUtensorMap *map, int x, int y, int z, int w,
                                      uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, "
      "%3, %4, %5}], [%6];" ::"r"(dst),
      "l"(map), "r"(x), "r"(y), "r"(z), "r"(w), "r"(bar)
      : "memory");
}

// K-major swizzled shared-memory descriptor: LBO unused (16 B), SBO = one
// 8-row atom, layout type 2 / 4 / 6 for 128 / 64 / 32-byte swizzle.
template <int SW>
__device__ __forceinline__ uint64_t make_desc_sw(uint32_t saddr) {
  constexpr uint64_t layout = SW == 128 ? 2 : SW == 64 ? 4 : 6;
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)1 << 16;
  d |= (uint64_t)(((8u * SW) >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  d |= layout << 61;
  return d;
}

__device__ __forceinline__ void mbar_arrive_plain(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

template <int BN, int EPI, int MODE, int SW>
__global__ void __launch_bounds__(128) k_gemm_tma(const __grid_constant__ CUtensorMap mapA,
                                                  const __grid_constant__ CUtensorMap mapB, GemmArgs g,
                                                  ConvGeo geo) {
  constexpr int KS = SW / 2;
  constexpr uint32_t A_BYTES = BM * SW, B_BYTES = BN * SW;
  constexpr uint32_t ST_BYTES = stage_bytes(BN, SW);
  constexpr int S = tma_stages(BN, SW);
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char *base = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const uint32_t sbase = smem_addr(base);
  __shared__ __align__(8) uint64_t full[S], empty[S], done;
  __shared__ uint32_t s_tmem;
  __shared__ int s_abort;
  volatile int *abort_flag = &s_abort;

  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  int kb = 0, nk;
  if (MODE == MODE_DENSE) {
    kb = blockIdx.z * g.ksplit;
    const int ke = min(g.K, kb + g.ksplit);
    nk = ke > kb ? (ke - kb + KS - 1) / KS : 0;
  } else {
    nk = 9 * geo.cchunks;
  }
  const int warp = threadIdx.x >> 5;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_addr(&s_tmem)),
                 "r"((uint32_t)BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (threadIdx.x == 0) {
    s_abort = 0;
    for (int i = 0; i < S; ++i) {
      mbar_init(smem_addr(&full[i]), 1);
      mbar_init(smem_addr(&empty[i]), 1);
    }
    mbar_init(smem_addr(&done), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(&mapA) : "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(&mapB) : "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = s_tmem;

  if (threadIdx.x == 0) {
    // ---- TMA producer
    int w0 = 0, h0 = 0, b0 = 0;
    if (MODE == MODE_CONV) {
      w0 = m0 % geo.W;
      const int q = m0 / geo.W;
      h0 = q % geo.H;
      b0 = q / geo.H;
    }
    for (int k = 0; k < nk; ++k) {
      const int st = k % S;
      if (k >= S && !mbar_wait(smem_addr(&empty[st]), (uint32_t)((k / S - 1) & 1))) {
        *abort_flag = 1;
        break;
      }
      const uint32_t sa = sbase + st * ST_BYTES, sb = sa + A_BYTES;
      const uint32_t bar = smem_addr(&full[st]);
      expect_tx(bar, A_BYTES + B_BYTES);
      if (MODE == MODE_DENSE) {
        const int kx = kb + k * KS;
        tma2d(sa, &mapA, kx, m0, bar);
        tma2d(sb, &mapB, kx, n0, bar);
      } else {
        const int tap = k / geo.cchunks, cc = k - tap * geo.cchunks;
        tma4d(sa, &mapA, cc * KS, w0 + tap % 3 - 1, h0 + tap / 3 - 1, b0, bar);
        tma2d(sb, &mapB, k * KS, n0, bar);
      }
    }
  } else if (threadIdx.x == 32) {
    // ---- MMA issuer
    constexpr uint32_t idesc = make_idesc<BN, false, false>();
    int issued = 0;
    for (int k = 0; k < nk; ++k) {
      const int st = k % S;
      if (!mbar_wait(smem_addr(&full[st]), (uint32_t)((k / S) & 1))) {
        *abort_flag = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t sa = sbase + st * ST_BYTES, sb = sa + A_BYTES;
#pragma unroll
      for (int kk = 0; kk < KS / 16; ++kk)
        mma_bf16(tmem, make_desc_sw<SW>(sa + kk * 32), make_desc_sw<SW>(sb + kk * 32), idesc,
                 (k > 0 || kk > 0) ? 1u : 0u);
      commit(smem_addr(&empty[st]));
      ++issued;
    }
    if (issued > 0) commit(smem_addr(&done));
    else mbar_arrive_plain(smem_addr(&done));
  }
  if (!mbar_wait(smem_addr(&done), 0u)) *abort_flag = 1;
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  __syncthreads();
  if (s_abort) {
    if (threadIdx.x == 0) atomicExch(g.err, 1);
  } else {
    gemm_epilogue<BN, EPI>(g, tmem, m0, n0, nk > 0);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)BN));
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    AIRT_CHECK_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
    AIRT_REQUIRE(q == cudaDriverEntryPointSuccess && p, "cuTensorMapEncodeTiled is not available");
    fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

CUtensorMapSwizzle swizzle_of(int sw) {
  return sw == 128 ? CU_TENSOR_MAP_SWIZZLE_128B : sw == 64 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_32B;
}

// bf16 tensor map; dims[0] innermost, strides in bytes for dims 1..rank-1.
CUtensorMap make_map(const void *base, int rank, const cuuint64_t *dims, const cuuint64_t *strides,
                     const cuuint32_t *box, int sw) {
  AIRT_REQUIRE(((uintptr_t)base & 15) == 0, "tensor map base must be 16-byte aligned");
  for (int i = 0; i + 1 < rank; ++i) AIRT_REQUIRE(strides[i] % 16 == 0, "tensor map strides must be multiples of 16 bytes");
  CUtensorMap m;
  const cuuint32_t es[5] = {1, 1, 1, 1, 1};
  const CUresult r = encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, (cuuint32_t)rank, const_cast<void *>(base),
                                 dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle_of(sw),
                                 CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  AIRT_REQUIRE(r == CUDA_SUCCESS, "tensor map encoding failed");
  return m;
}

template <int BN, int EPI, int MODE, int SW>
void launch_tma(const CUtensorMap &ma, const CUtensorMap &mb, const GemmArgs &g, ConvGeo geo, dim3 grid,
                cudaStream_t s) {
  const size_t smem = (size_t)tma_stages(BN, SW) * stage_bytes(BN, SW) + 1024;
  auto kern = k_gemm_tma<BN, EPI, MODE, SW>;
  AIRT_CHECK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  kern<<<grid, 128, smem, s>>>(ma, mb, g, geo);
  AIRT_LAUNCH_CHECK();
}

template <int MODE, int SW>
void dispatch_tma(const CUtensorMap &ma, const CUtensorMap &mb, const GemmArgs &g, ConvGeo geo, int bn,
                  int epi, dim3 grid, cudaStream_t s) {
#define AIRT_T(BNV)                                                                                        \
  switch (epi) {                                                                                           \
    case EPI_STORE_F32: launch_tma<BNV, EPI_STORE_F32, MODE, SW>(ma, mb, g, geo, grid, s); break;          \
    case EPI_BIAS_RELU_BF16: launch_tma<BNV, EPI_BIAS_RELU_BF16, MODE, SW>(ma, mb, g, geo, grid, s); break; \
    case EPI_BIAS_BF16: launch_tma<BNV, EPI_BIAS_BF16, MODE, SW>(ma, mb, g, geo, grid, s); break;          \
    case EPI_ADD_F32: launch_tma<BNV, EPI_ADD_F32, MODE, SW>(ma, mb, g, geo, grid, s); break;              \
    default: launch_tma<BNV, EPI_ATOMIC_F32_T, MODE, SW>(ma, mb, g, geo, grid, s); break;                  \
  }
  switch (bn) {
    case 32: AIRT_T(32) break;
    case 64: AIRT_T(64) break;
    case 128: AIRT_T(128) break;
    case 256: AIRT_T(256) break;
    default: AIRT_REQUIRE(false, "gemm: BN must be 32, 64, 128 or 256");
  }
#undef AIRT_T
}

}  // namespace

bool gemm_tma_ok(const GemmArgs &g) {
  return g.lda % 8 == 0 && g.ldb % 8 == 0 && ((uintptr_t)g.A & 15) == 0 && ((uintptr_t)g.B & 15) == 0 &&
         g.K >= 8 && (g.ksplit <= 0 || g.ksplit >= g.K || g.ksplit % 64 == 0);
}

void gemm_bf16_tma(const GemmArgs &g0, int bn, int epi, cudaStream_t s) {
  GemmArgs g = g0;
  if (g.ksplit <= 0 || g.ksplit > g.K) g.ksplit = g.K;
  AIRT_REQUIRE(gemm_tma_ok(g), "gemm: operands unsuitable for TMA");
  const cuuint64_t da[2] = {(cuuint64_t)g.K, (cuuint64_t)g.M}, sa[1] = {(cuuint64_t)g.lda * 2};
  const cuuint64_t db[2] = {(cuuint64_t)g.K, (cuuint64_t)g.N}, sb[1] = {(cuuint64_t)g.ldb * 2};
  const cuuint32_t ba[2] = {64, (cuuint32_t)BM}, bb[2] = {64, (cuuint32_t)bn};
  const CUtensorMap ma = make_map(g.A, 2, da, sa, ba, 128);
  const CUtensorMap mb = make_map(g.B, 2, db, sb, bb, 128);
  const int splits = (g.K + g.ksplit - 1) / g.ksplit;
  const dim3 grid((g.M + BM - 1) / BM, (g.N + bn - 1) / bn, splits);
  dispatch_tma<MODE_DENSE, 128>(ma, mb, g, ConvGeo{}, bn, epi, grid, s);
}

// Pixel box of 128 consecutive NHWC pixels, or false when the image shape
// does not tile that way.
static bool conv_box(int Bimg, int H, int W, int &bw, int &bh, int &bb) {
  (void)Bimg;
  if (W >= 128) {
    if (W % 128) return false;
    bw = 128, bh = 1, bb = 1;
    return true;
  }
  if (128 % W) return false;
  bw = W;
  const int rows = 128 / W;
  if (rows <= H) {
    if (H % rows) return false;
    bh = rows, bb = 1;
    return true;
  }
  if (rows % H) return false;
  bh = H, bb = rows / H;
  return bb <= 256;
}

bool conv3x3_tma_ok(const GemmArgs &g) {
  int bw, bh, bb;
  return g.conv_C % 16 == 0 && ((uintptr_t)g.convX & 15) == 0 && ((uintptr_t)g.B & 15) == 0 &&
         g.ldb % 8 == 0 && g.M % (g.conv_H * g.conv_W) == 0 &&
         conv_box(g.M / (g.conv_H * g.conv_W), g.conv_H, g.conv_W, bw, bh, bb);
}

void conv3x3_bf16_tma(const GemmArgs &g, int bn, int epi, cudaStream_t s) {
  AIRT_REQUIRE(conv3x3_tma_ok(g), "conv3x3: shape unsuitable for TMA");
  const int C = g.conv_C, H = g.conv_H, W = g.conv_W, Bimg = g.M / (H * W);
  const int sw = C % 64 == 0 ? 128 : C % 32 == 0 ? 64 : 32;
  const int ks = sw / 2;
  int bw, bh, bb;
  conv_box(Bimg, H, W, bw, bh, bb);
  const cuuint64_t dx[4] = {(cuuint64_t)C, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)Bimg};
  const cuuint64_t sx[3] = {(cuuint64_t)C * 2, (cuuint64_t)W * C * 2, (cuuint64_t)H * W * C * 2};
  const cuuint32_t bx[4] = {(cuuint32_t)ks, (cuuint32_t)bw, (cuuint32_t)bh, (cuuint32_t)bb};
  const CUtensorMap ma = make_map(g.convX, 4, dx, sx, bx, sw);
  const cuuint64_t dw[2] = {(cuuint64_t)9 * C, (cuuint64_t)g.N}, swt[1] = {(cuuint64_t)g.ldb * 2};
  const cuuint32_t bwt[2] = {(cuuint32_t)ks, (cuuint32_t)bn};
  const CUtensorMap mb = make_map(g.B, 2, dw, swt, bwt, sw);
  const ConvGeo geo{W, H, C / ks};
  const dim3 grid((g.M + BM - 1) / BM, (g.N + bn - 1) / bn, 1);
  if (sw == 128) dispatch_tma<MODE_CONV, 128>(ma, mb, g, geo, bn, epi, grid, s);
  else if (sw == 64) dispatch_tma<MODE_CONV, 64>(ma, mb, g, geo, bn, epi, grid, s);
  else dispatch_tma<MODE_CONV, 32>(ma, mb, g, geo, bn, epi, grid, s);
}

}  // namespace airt
