// tcgen05 GEMM with TMA operand loads, persistent and warp-specialised.
//
// Four operand sources (three in k_gemm_tma, one in k_conv_rows):
//  * MODE_DENSE: A [M][lda] and B [N][ldb] row-major bf16 matrices
//    (K-major), 2D tensor maps, boxes {64, 128} and {64, BN};
//  * MODE_CONV: the implicit 3x3 convolution of an NHWC bf16 image X
//    [B][H][W][C] (K-major): a 4D tensor map (C, W, H, B) whose box
//    {KS, bw, bh, bb} (bw*bh*bb = 128 consecutive pixels) is loaded at the
//    tile origin shifted by the tap (dw, dh); out-of-image coordinates read
//    as zero, which is the convolution's zero padding.  Stage k is tap
//    k / (C/KS), channels (k % (C/KS))*KS.. +KS; the weights W[N][ldb] carry
//    the same K index (tap*C + ci);
//  * MODE_HALO: the same convolution for images whose rows hold whole
//    128-pixel tiles (W % 128 == 0): instead of nine tap boxes per tile,
//    each kernel row dh brings one strip of 130 pixels (the tile and one
//    pixel either side) of image row h + dh - 1, and the three taps of that
//    row read it shifted by 0, 1 and 2 pixel rows through the descriptor's
//    start address (the swizzle pattern follows the shared-memory address,
//    so the descriptor's base offset stays 0).  With 64-byte rows (32
//    channels) a one-row shift is not a whole 128-byte swizzle phase, so a
//    second strip starting one pixel later serves the middle tap.  Per tile
//    3 (or 6) strips replace 9 boxes; a stage carries one kernel row (its
//    strips and the three taps' weight slices);
//  * row runs (k_conv_rows, below): the halo strips of an input row loaded
//    once for the three output rows that read it, weights resident;
//  * MODE_WGRAD: the weight gradient of that convolution, both operands
//    MN-major: A^T[pixel][tap*C + ci] gathered as 64-pixel boxes of X
//    shifted per tap (one box per 64/32/16 channels of the 128-row M tile),
//    B = dY [pixel][N]; K runs over pixels, split across tiles, and the
//    epilogue adds into gw[N][M] atomically.
//
// Shared-memory tiles use the canonical swizzled UMMA layouts that TMA
// writes with the matching CU_TENSOR_MAP_SWIZZLE_* (SW = 128, 64 or 32
// bytes): K-major rows of SW bytes in 8-row atoms (SBO = 8*SW), each K=16
// MMA step 32 bytes further; MN-major rows of SW bytes (SW/2 elements of M
// or N) per K index, 8-row atoms along K (SBO = 8*SW), 64-row boxes per MN
// group (LBO = 64*SW), each K=16 step 16 rows further.
//
// Roles (192 threads, persistent over tiles): warp 0 lane 0 streams the TMA
// loads of every tile's K slices through an S-stage ring (`full` barriers
// with expect-tx bytes, `empty` barriers released by tcgen05.commit); warp 1
// lane 0 issues the tcgen05.mma instructions into one of two TMEM
// accumulators and commits the tile to `acc_full`; warps 2-5 drain the other
// accumulator meanwhile (warp w reads TMEM lanes 32*(w%4)..) and release it
// through `acc_empty`.  All waits are bounded.  No multicast.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>

#include "umma.cuh"

namespace airt {

namespace {

using namespace umma;

enum { MODE_DENSE = 0, MODE_CONV = 1, MODE_WGRAD = 2, MODE_HALO = 3 };

// Halo strips: rows (pixels) per strip, a multiple of 8 covering the 130
// pixels a 128-pixel tile's taps read.
constexpr int kStripRows = 136;
constexpr int kStripBox = 130;

struct TmaGeo {
  int W, H;                      // image width and height (CONV, WGRAD)
  int C;                         // channels of X (WGRAD)
  int cchunks;                   // C / KS (CONV)
  int tiles_m, tiles_n, splits;  // tile grid
  int K, ksplit;                 // K extent and K range per split (DENSE, WGRAD)
};

constexpr uint32_t round1k(uint32_t b) { return (b + 1023u) & ~1023u; }

// Stages: about 104 KB per CTA when two CTAs share an SM, about 200 KB
// when one does; between 2 and 8.
constexpr int ring_stages(uint32_t stage, bool two_per_sm) {
  return (int)((two_per_sm ? 106496u : 204800u) / stage) > 8 ? 8
         : (int)((two_per_sm ? 106496u : 204800u) / stage) < 2 ? 2
                                                                : (int)((two_per_sm ? 106496u : 204800u) / stage);
}

template <int BN, int MODE, int SWA>
struct TmaCfg {
  static constexpr bool MN = MODE == MODE_WGRAD;
  static constexpr int KS = MN ? 64 : SWA / 2;  // K elements per stage (per tap for MODE_HALO)
  static constexpr int STRIPS = SWA == 128 ? 1 : 2;
  static constexpr uint32_t STRIP_BYTES = round1k((uint32_t)kStripRows * SWA);
  static constexpr uint32_t A_BYTES = MODE == MODE_HALO ? STRIPS * STRIP_BYTES : BM * KS * 2;
  static constexpr uint32_t B_BYTES = (MODE == MODE_HALO ? 3 : 1) * BN * KS * 2;
  // bytes the TMA copies of one stage deliver (a halo strip is kStripBox
  // rows of its kStripRows-row slot)
  static constexpr uint32_t TX_BYTES =
      MODE == MODE_HALO ? STRIPS * (uint32_t)kStripBox * SWA + B_BYTES : A_BYTES + B_BYTES;
  static constexpr uint32_t ST = round1k(A_BYTES + B_BYTES);
  static constexpr bool TWO = BN <= 128;  // TMEM: two CTAs x two accumulators x BN columns
  static constexpr int S = ring_stages(ST, TWO);
  // the request never falls below 80 KB (two CTAs) or 120 KB (one CTA), so
  // no third CTA lands on an SM and waits for TMEM columns
  static constexpr size_t SMEM_RING = (size_t)S * ST + 1024;
  static constexpr size_t SMEM = SMEM_RING > (TWO ? 81920u : 122880u) ? SMEM_RING : (TWO ? 81920u : 122880u);
};

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

// Swizzled shared-memory descriptor: layout type 2 / 4 / 6 for 128 / 64 /
// 32-byte swizzle; lbo / sbo in bytes.
template <int SW>
__device__ __forceinline__ uint64_t make_desc_sw(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  constexpr uint64_t layout = SW == 128 ? 2 : SW == 64 ? 4 : 6;
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  d |= layout << 61;
  return d;
}

__device__ __forceinline__ void mbar_arrive_plain(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

struct TileCoord {
  int m0, n0, kb, nk;
};

template <int BN, int MODE, int SWA>
__device__ __forceinline__ TileCoord tile_coord(const TmaGeo &geo, int t) {
  using Cfg = TmaCfg<BN, MODE, SWA>;
  const int mt = t % geo.tiles_m, r = t / geo.tiles_m;
  const int nt = r % geo.tiles_n, z = r / geo.tiles_n;
  TileCoord c;
  c.m0 = mt * BM;
  c.n0 = nt * BN;
  if (MODE == MODE_CONV) {
    c.kb = 0;
    c.nk = 9 * geo.cchunks;
  } else if (MODE == MODE_HALO) {
    c.kb = 0;
    c.nk = 3 * geo.cchunks;  // one stage per kernel row and channel chunk
  } else {
    c.kb = z * geo.ksplit;
    const int ke = min(geo.K, c.kb + geo.ksplit);
    c.nk = ke > c.kb ? (ke - c.kb + Cfg::KS - 1) / Cfg::KS : 0;
  }
  return c;
}

// Pixel p -> box origin (w, h, image) in an H x W image batch.
__device__ __forceinline__ void pixel_whb(int p, int W, int H, int &w, int &h, int &b) {
  w = p % W;
  const int q = p / W;
  h = q % H;
  b = q / H;
}

template <int BN, int EPI, int MODE, int SWA, int SWB>
__global__ void __launch_bounds__(192, 1) k_gemm_tma(const __grid_constant__ CUtensorMap mapA,
                                                     const __grid_constant__ CUtensorMap mapB, GemmArgs g,
                                                     TmaGeo geo) {
  using Cfg = TmaCfg<BN, MODE, SWA>;
  constexpr int S = Cfg::S, KS = Cfg::KS;
  constexpr uint32_t A_BYTES = Cfg::A_BYTES, ST = Cfg::ST;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char *base = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const uint32_t sbase = smem_addr(base);
  __shared__ __align__(8) uint64_t full[S], empty[S], acc_full[2], acc_empty[2];
  __shared__ uint32_t s_tmem;
  __shared__ int s_abort;
  volatile int *abort_flag = &s_abort;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ntiles = geo.tiles_m * geo.tiles_n * geo.splits;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_addr(&s_tmem)),
                 "r"((uint32_t)(2 * BN)));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (threadIdx.x == 0) {
    s_abort = 0;
    for (int i = 0; i < S; ++i) {
      mbar_init(smem_addr(&full[i]), 1);
      mbar_init(smem_addr(&empty[i]), 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(smem_addr(&acc_full[i]), 1);
      mbar_init(smem_addr(&acc_empty[i]), 128);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(&mapA) : "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(&mapB) : "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = s_tmem;

  if (warp == 0) {
    if (lane == 0) {
      // ---- TMA producer
      uint32_t it = 0;
      for (int t = blockIdx.x; t < ntiles && !*abort_flag; t += gridDim.x) {
        const TileCoord tc = tile_coord<BN, MODE, SWA>(geo, t);
        int w0 = 0, h0 = 0, b0 = 0;
        if (MODE == MODE_CONV || MODE == MODE_HALO) pixel_whb(tc.m0, geo.W, geo.H, w0, h0, b0);
        for (int k = 0; k < tc.nk; ++k, ++it) {
          const uint32_t st = it % S;
          if (it >= (uint32_t)S && !mbar_wait(smem_addr(&empty[st]), ((it / S) - 1) & 1u)) {
            *abort_flag = 1;
            break;
          }
          const uint32_t sa = sbase + st * ST, sb = sa + A_BYTES;
          const uint32_t bar = smem_addr(&full[st]);
          expect_tx(bar, Cfg::TX_BYTES);
          if (MODE == MODE_DENSE) {
            const int kx = tc.kb + k * KS;
            tma2d(sa, &mapA, kx, tc.m0, bar);
            tma2d(sb, &mapB, kx, tc.n0, bar);
          } else if (MODE == MODE_CONV) {
            const int tap = k / geo.cchunks, cc = k - tap * geo.cchunks;
            tma4d(sa, &mapA, cc * KS, w0 + tap % 3 - 1, h0 + tap / 3 - 1, b0, bar);
            tma2d(sb, &mapB, k * KS, tc.n0, bar);
          } else if (MODE == MODE_HALO) {
            // kernel row dh, channel chunk cc: strip(s) of image row h0 + dh - 1
            // from pixel w0 - 1 (and w0), then the weights of taps 3dh .. 3dh+2
            const int dh = k / geo.cchunks, cc = k - dh * geo.cchunks;
#pragma unroll
            for (int q = 0; q < Cfg::STRIPS; ++q)
              tma4d(sa + q * Cfg::STRIP_BYTES, &mapA, cc * KS, w0 - 1 + q, h0 + dh - 1, b0, bar);
#pragma unroll
            for (int dw = 0; dw < 3; ++dw)
              tma2d(sb + dw * (BN * KS * 2), &mapB, ((3 * dh + dw) * geo.cchunks + cc) * KS, tc.n0,
                    bar);
          } else {
            constexpr int GA = SWA / 2, GB = SWB / 2;  // M / N elements per box
            const int p0 = tc.kb + k * KS;
            int pw, ph, pb;
            pixel_whb(p0, geo.W, geo.H, pw, ph, pb);
#pragma unroll
            for (int j = 0; j < BM / GA; ++j) {
              const int kk = tc.m0 + j * GA;
              const int tap = kk / geo.C, ci = kk - tap * geo.C;
              // taps past the ninth are the K padding: a box far outside the image reads zeros
              const int dh = tap < 9 ? tap / 3 - 1 : -(1 << 20), dw = tap < 9 ? tap % 3 - 1 : 0;
              tma4d(sa + j * (64 * SWA), &mapA, tap < 9 ? ci : 0, pw + dw, ph + dh, pb, bar);
            }
#pragma unroll
            for (int j = 0; j < BN / GB; ++j) tma2d(sb + j * (64 * SWB), &mapB, tc.n0 + j * GB, p0, bar);
          }
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // ---- MMA issuer
      constexpr bool MN = Cfg::MN;
      constexpr uint32_t idesc = make_idesc<BN, MN, MN>();
      uint32_t it = 0, tl = 0;
      for (int t = blockIdx.x; t < ntiles && !*abort_flag; t += gridDim.x, ++tl) {
        const TileCoord tc = tile_coord<BN, MODE, SWA>(geo, t);
        const uint32_t buf = tl & 1u;
        if (tl >= 2 && !mbar_wait(smem_addr(&acc_empty[buf]), ((tl >> 1) - 1) & 1u)) {
          *abort_flag = 1;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t dtm = tmem + buf * BN;
        bool ok = true;
        for (int k = 0; k < tc.nk; ++k, ++it) {
          const uint32_t st = it % S;
          if (!mbar_wait(smem_addr(&full[st]), (it / S) & 1u)) {
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t sa = sbase + st * ST, sb = sa + A_BYTES;
          if constexpr (MODE == MODE_HALO) {
            // tap dw reads the strip shifted by dw pixel rows: strip 0 at rows
            // 0 and 2 (2-row shifts keep 64-byte rows on a swizzle phase), or,
            // with 128-byte rows, at any row; strip 1 (64-byte rows) at row 0
#pragma unroll
            for (int dw = 0; dw < 3; ++dw) {
              const uint32_t a0 = Cfg::STRIPS == 2 && dw == 1 ? sa + Cfg::STRIP_BYTES
                                                              : sa + (uint32_t)dw * SWA;
#pragma unroll
              for (int kk = 0; kk < KS / 16; ++kk) {
                const uint64_t da = make_desc_sw<SWA>(a0 + kk * 32, 16, 8 * SWA);
                const uint64_t db = make_desc_sw<SWA>(sb + dw * (BN * KS * 2) + kk * 32, 16, 8 * SWA);
                mma_bf16(dtm, da, db, idesc, (k > 0 || dw > 0 || kk > 0) ? 1u : 0u);
              }
            }
            commit(smem_addr(&empty[st]));
          } else {
            // K step kk: the base descriptors plus the step's byte offset / 16
            const uint64_t da0 = MN ? make_desc_sw<SWA>(sa, 64 * SWA, 8 * SWA) : make_desc_sw<SWA>(sa, 16, 8 * SWA);
            const uint64_t db0 = MN ? make_desc_sw<SWB>(sb, 64 * SWB, 8 * SWB) : make_desc_sw<SWA>(sb, 16, 8 * SWA);
#pragma unroll
            for (int kk = 0; kk < KS / 16; ++kk) {
              const uint64_t da = da0 + (MN ? (uint64_t)kk * SWA : (uint64_t)kk * 2);
              const uint64_t db = db0 + (MN ? (uint64_t)kk * SWB : (uint64_t)kk * 2);
              mma_bf16(dtm, da, db, idesc, (k > 0 || kk > 0) ? 1u : 0u);
            }
            commit(smem_addr(&empty[st]));
          }
        }
        if (!ok) {
          *abort_flag = 1;
          break;
        }
        if (tc.nk > 0) commit(smem_addr(&acc_full[buf]));
        else mbar_arrive_plain(smem_addr(&acc_full[buf]));
      }
    }
  } else {
    // ---- epilogue warps 2-5
    const int quad = warp & 3;
    uint32_t tl = 0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++tl) {
      const TileCoord tc = tile_coord<BN, MODE, SWA>(geo, t);
      const uint32_t buf = tl & 1u;
      if (!mbar_wait(smem_addr(&acc_full[buf]), (tl >> 1) & 1u)) {
        *abort_flag = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      gemm_epilogue<BN, EPI>(g, tmem + ((uint32_t)(quad * 32) << 16) + buf * BN, tc.m0 + quad * 32 + lane,
                             tc.n0, tc.nk > 0);
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      mbar_arrive_plain(smem_addr(&acc_empty[buf]));
    }
  }
  __syncthreads();
  if (s_abort && threadIdx.x == 0) atomicExch(g.err, 1);
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)(2 * BN)));
}

// ---------------------------------------------------------------- row runs
// The 3x3 convolution of images whose rows hold whole 128-pixel segments,
// walked as runs of R consecutive output rows of one segment.  Each input
// row of a run is loaded once (as the halo strips of MODE_HALO: 130 pixels,
// one either side; with 64-byte pixel rows a second strip one pixel later),
// so R + 2 input rows serve R output rows where MODE_HALO loads three per
// output row, and the nine taps' weight slices are loaded once per CTA and
// stay resident.  One ring stage holds one input row (all channel chunks);
// output row i of a run reads the stages of input rows i, i+1 and i+2, and
// input row i is released once output row i's MMAs complete (it is the last
// row to read it).  Requires N == BN (one output-channel tile).
struct RowsGeo {
  int W, H, R;             // image width, height; output rows per run
  int segs, hblocks;       // 128-pixel segments per row; runs per column
  int nunits;              // Bimg * segs * hblocks
  int cch;                 // channel chunks, C / KS
  int S;                   // ring stages
  uint32_t stage_bytes;    // one input row: cch * strips strips
  uint32_t w_bytes;        // resident weights: 9 * cch slices of BN x KS
  int tma_out;             // k_conv_stack: BF16 output rows leave by TMA stores
};

constexpr int kRowsMaxStages = 8;

// ONE: a single strip per input row also for 64-byte pixel rows, the middle
// tap reading it one pixel row (64 bytes) further on.
template <int SWA, bool ONE>
struct RowsCfg {
  static constexpr int KS = SWA / 2;
  static constexpr int STRIPS = SWA == 128 || ONE ? 1 : 2;
  static constexpr uint32_t STRIP_BYTES = round1k((uint32_t)kStripRows * SWA);
};

struct RowsUnit {
  int w0, h0, b, rows;
};

__device__ __forceinline__ RowsUnit rows_unit(const RowsGeo &geo, int u) {
  RowsUnit r;
  const int hb = u % geo.hblocks, q = u / geo.hblocks;
  r.w0 = (q % geo.segs) * 128;
  r.b = q / geo.segs;
  r.h0 = hb * geo.R;
  r.rows = min(geo.R, geo.H - r.h0);
  return r;
}

// Epilogue groups of four warps: NE groups drain 2*NE TMEM accumulators in
// turn (output row ol -> accumulator ol % (2 NE), group ol % NE), so two
// warps per SM sub-partition hide each other's TMEM-load and store latency.
template <int BN>
struct RowsRoles {
  static constexpr int NE = BN <= 64 ? 2 : 1;
  static constexpr int NACC = 2 * NE;
  static constexpr int THREADS = 64 + 128 * NE;
  static constexpr uint32_t TMEM_COLS = (uint32_t)(NACC * BN);
};

template <int BN, int EPI, int SWA, bool ONE>
__global__ void __launch_bounds__(RowsRoles<BN>::THREADS, 1)
    k_conv_rows(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB, GemmArgs g,
                RowsGeo geo) {
  using Cfg = RowsCfg<SWA, ONE>;
  using Ro = RowsRoles<BN>;
  constexpr int KS = Cfg::KS, STRIPS = Cfg::STRIPS, NACC = Ro::NACC, NE = Ro::NE;
  constexpr uint32_t STRIP = Cfg::STRIP_BYTES;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char *base = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const uint32_t wbase = smem_addr(base);  // resident weights (w_bytes, a multiple of 1 KB)
  const uint32_t rbase = wbase + geo.w_bytes;
  __shared__ __align__(8) uint64_t full[kRowsMaxStages], empty[kRowsMaxStages], acc_full[NACC],
      acc_empty[NACC], wfull;
  __shared__ uint32_t s_tmem;
  __shared__ int s_abort;
  volatile int *abort_flag = &s_abort;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int S = geo.S;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_addr(&s_tmem)),
                 "r"(Ro::TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (threadIdx.x == 0) {
    s_abort = 0;
    for (int i = 0; i < S; ++i) {
      mbar_init(smem_addr(&full[i]), 1);
      mbar_init(smem_addr(&empty[i]), 1);
    }
    for (int i = 0; i < NACC; ++i) {
      mbar_init(smem_addr(&acc_full[i]), 1);
      mbar_init(smem_addr(&acc_empty[i]), 128);
    }
    mbar_init(smem_addr(&wfull), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(&mapA) : "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(&mapB) : "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = s_tmem;

  if (warp == 0) {
    if (lane == 0) {
      // ---- TMA producer: the weights once, then one stage per input row
      const uint32_t wb = smem_addr(&wfull);
      expect_tx(wb, geo.w_bytes);
      for (int j = 0; j < 9 * geo.cch; ++j) tma2d(wbase + (uint32_t)j * (BN * SWA), &mapB, j * KS, 0, wb);
      const uint32_t tx = (uint32_t)(geo.cch * STRIPS * kStripBox * SWA);
      uint32_t it = 0;
      for (int u = blockIdx.x; u < geo.nunits && !*abort_flag; u += gridDim.x) {
        const RowsUnit ru = rows_unit(geo, u);
        bool ok = true;
        for (int r = 0; r < ru.rows + 2; ++r, ++it) {
          const uint32_t st = it % S;
          if (it >= (uint32_t)S && !mbar_wait(smem_addr(&empty[st]), ((it / S) - 1) & 1u)) {
            ok = false;
            break;
          }
          const uint32_t sa = rbase + st * geo.stage_bytes, bar = smem_addr(&full[st]);
          expect_tx(bar, tx);
          for (int cc = 0; cc < geo.cch; ++cc)
#pragma unroll
            for (int q = 0; q < STRIPS; ++q)
              tma4d(sa + (uint32_t)(cc * STRIPS + q) * STRIP, &mapA, cc * KS, ru.w0 - 1 + q, ru.h0 - 1 + r, ru.b,
                    bar);
        }
        if (!ok) {
          *abort_flag = 1;
          break;
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // ---- MMA issuer.  A descriptor's start-address field is the byte
      // address / 16 in its low bits, so the descriptors of the taps, chunks
      // and K steps are the stage's (or the weights') base descriptor plus a
      // constant: one 64-bit add per operand per MMA.
      constexpr uint32_t idesc = make_idesc<BN, false, false>();
      const uint64_t wdesc = make_desc_sw<SWA>(wbase, 16, 8 * SWA);
      bool ok = mbar_wait(smem_addr(&wfull), 0);
      uint32_t it = 0, ol = 0;
      for (int u = blockIdx.x; ok && u < geo.nunits && !*abort_flag; u += gridDim.x) {
        const RowsUnit ru = rows_unit(geo, u);
        for (int r = 0; r < 2 && ok; ++r) ok = mbar_wait(smem_addr(&full[(it + r) % S]), ((it + r) / S) & 1u);
        for (int i = 0; ok && i < ru.rows; ++i, ++ol) {
          const uint32_t sr = it + i + 2;
          const uint32_t buf = ol % NACC;
          if (!mbar_wait(smem_addr(&full[sr % S]), (sr / S) & 1u) ||
              (ol >= (uint32_t)NACC && !mbar_wait(smem_addr(&acc_empty[buf]), ((ol / NACC) - 1) & 1u))) {
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t dtm = tmem + buf * BN;
          uint32_t acc = 0;
          for (int dh = 0; dh < 3; ++dh) {
            const uint64_t sdesc = make_desc_sw<SWA>(rbase + ((it + i + dh) % S) * geo.stage_bytes, 16, 8 * SWA);
            for (int cc = 0; cc < geo.cch; ++cc) {
              const uint64_t cdesc = sdesc + ((uint64_t)(cc * STRIPS) * STRIP >> 4);
              // tap dw reads the strip shifted by dw pixel rows (strip 1 for
              // the middle tap when pixel rows are 64 bytes: see MODE_HALO)
#pragma unroll
              for (int dw = 0; dw < 3; ++dw) {
                const uint64_t da = cdesc + ((STRIPS == 2 && dw == 1 ? STRIP : (uint32_t)dw * SWA) >> 4);
                const uint64_t db = wdesc + ((uint64_t)((3 * dh + dw) * geo.cch + cc) * (BN * SWA) >> 4);
#pragma unroll
                for (int kk = 0; kk < KS / 16; ++kk) {
                  mma_bf16(dtm, da + 2 * kk, db + 2 * kk, idesc, acc);
                  acc = 1;
                }
              }
            }
          }
          commit(smem_addr(&acc_full[buf]));
          commit(smem_addr(&empty[(it + i) % S]));  // input row i: output row i was its last reader
        }
        if (!ok) break;
        commit(smem_addr(&empty[(it + ru.rows) % S]));
        commit(smem_addr(&empty[(it + ru.rows + 1) % S]));
        it += ru.rows + 2;
      }
      if (!ok) *abort_flag = 1;
    }
  } else {
    // ---- epilogue groups: warps 2 + 4e .. 5 + 4e; warp w reads TMEM lanes
    // 32 * (w % 4) ..; group e takes the output rows ol with ol % NE == e
    const int quad = warp & 3, grp = (warp - 2) >> 2;
    uint32_t ol = 0;
    bool ok = true;
    for (int u = blockIdx.x; ok && u < geo.nunits; u += gridDim.x) {
      const RowsUnit ru = rows_unit(geo, u);
      for (int i = 0; i < ru.rows; ++i, ++ol) {
        if ((int)(ol % NE) != grp) continue;
        const uint32_t buf = ol % NACC;
        if (!mbar_wait(smem_addr(&acc_full[buf]), (ol / NACC) & 1u)) {
          *abort_flag = 1;
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const int m0 = ((ru.b * geo.H + ru.h0 + i) * geo.W) + ru.w0;
        gemm_epilogue<BN, EPI>(g, tmem + ((uint32_t)(quad * 32) << 16) + buf * BN, m0 + quad * 32 + lane, 0,
                               true);
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        mbar_arrive_plain(smem_addr(&acc_empty[buf]));
      }
    }
  }
  __syncthreads();
  if (s_abort && threadIdx.x == 0) atomicExch(g.err, 1);
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(Ro::TMEM_COLS));
}

// ---------------------------------------------------------------- stacked rows
// Row runs with the three kernel rows stacked along N.  An input row r of a
// run feeds output rows r-2, r-1 and r (kernel rows 2, 1, 0); with the
// weights of one tap column laid out as [W(dh=2); W(dh=1); W(dh=0)] (3 BN
// rows) one MMA of N = 3 BN multiplies the input row's strip once into the
// accumulators of all three output rows, which sit side by side in a ring
// of RB TMEM blocks (output row ol in block ol % RB).  The A tile (128
// pixels x 16 channels, 4 KB) is read from shared memory once per three
// kernel rows instead of once per kernel row, so the MMAs are no longer
// bound by shared-memory operand bandwidth at small BN.  All MMAs
// accumulate: the epilogue zeroes a block after draining it (and every block
// once at the start) before handing it back.  An input row's stage is free
// as soon as its own MMAs complete; output row i is complete after input row
// i + 2.  At the run's ends and where the three blocks wrap around the ring
// the MMA covers fewer rows (N = BN or 2 BN) or splits in two.
__device__ __forceinline__ uint32_t idesc_n(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}

__device__ __forceinline__ void tmem_zero32(uint32_t taddr) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, "
      "%1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1};" ::"r"(taddr),
      "r"(0u)
      : "memory");
}

template <int BN>
struct StackRoles {
  static constexpr int NE = 2;                   // epilogue groups of four warps
  static constexpr int RB = 256 / BN;            // TMEM blocks (256 columns: two CTAs per SM)
  static constexpr int THREADS = 64 + 128 * NE;
  static constexpr uint32_t TMEM_COLS = 256;
  // BN = 32: two CTAs per SM (their shared memory fits), so the registers
  // of two 320-thread CTAs must fit as well
  static constexpr int MIN_CTAS = BN == 32 ? 2 : 1;
};

__device__ __forceinline__ void named_sync(int id, int count) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

__device__ __forceinline__ void tma_store4d(const CUtensorMap *map, uint32_t src, int x, int y, int z, int w) {
  asm volatile(
      "cp.async.bulk.tensor.4d.global.shared::cta.bulk_group [%0, {%1, %2, %3, %4}], [%5];" ::"l"(map), "r"(x),
      "r"(y), "r"(z), "r"(w), "r"(src)
      : "memory");
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}

template <int BN, int EPI, int SWA, bool ONE>
__global__ void __launch_bounds__(StackRoles<BN>::THREADS, StackRoles<BN>::MIN_CTAS)
    k_conv_stack(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
                 const __grid_constant__ CUtensorMap mapD, GemmArgs g, RowsGeo geo) {
  using Cfg = RowsCfg<SWA, ONE>;
  using Ro = StackRoles<BN>;
  constexpr int KS = Cfg::KS, STRIPS = Cfg::STRIPS, RB = Ro::RB, NE = Ro::NE;
  constexpr uint32_t STRIP = Cfg::STRIP_BYTES;
  static_assert(3 * BN <= 256, "N = 3 BN must fit one MMA");
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char *base = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const uint32_t wbase = smem_addr(base);
  const uint32_t rbase = wbase + geo.w_bytes;
  __shared__ __align__(8) uint64_t full[kRowsMaxStages], empty[kRowsMaxStages], acc_full[RB], acc_empty[RB],
      wfull, stg_free[NE], stg_full[NE];
  __shared__ uint32_t s_tmem;
  __shared__ int s_abort;
  volatile int *abort_flag = &s_abort;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int S = geo.S;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_addr(&s_tmem)),
                 "r"(Ro::TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (threadIdx.x == 0) {
    s_abort = 0;
    for (int i = 0; i < S; ++i) {
      mbar_init(smem_addr(&full[i]), 1);
      mbar_init(smem_addr(&empty[i]), 1);
    }
    for (int i = 0; i < RB; ++i) {
      mbar_init(smem_addr(&acc_full[i]), 1);
      mbar_init(smem_addr(&acc_empty[i]), 128);
    }
    mbar_init(smem_addr(&wfull), 1);
    for (int e = 0; e < NE; ++e) {
      mbar_init(smem_addr(&stg_free[e]), 1);
      mbar_init(smem_addr(&stg_full[e]), 128);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(&mapA) : "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(&mapB) : "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = s_tmem;

  if (warp == 0) {
    if (lane == 0) {
      // ---- TMA producer: weight slabs [dw][cc][dh = 2, 1, 0], then one
      // stage per input row
      const uint32_t wb = smem_addr(&wfull);
      expect_tx(wb, geo.w_bytes);
      for (int dw = 0; dw < 3; ++dw)
        for (int cc = 0; cc < geo.cch; ++cc)
          for (int dh = 0; dh < 3; ++dh)
            tma2d(wbase + (uint32_t)((dw * geo.cch + cc) * 3 + (2 - dh)) * (BN * SWA), &mapB,
                  ((3 * dh + dw) * geo.cch + cc) * KS, 0, wb);
      const uint32_t tx = (uint32_t)(geo.cch * STRIPS * kStripBox * SWA);
      uint32_t it = 0;
      for (int u = blockIdx.x; u < geo.nunits && !*abort_flag; u += gridDim.x) {
        const RowsUnit ru = rows_unit(geo, u);
        bool ok = true;
        for (int r = 0; r < ru.rows + 2; ++r, ++it) {
          const uint32_t st = it % S;
          if (it >= (uint32_t)S && !mbar_wait(smem_addr(&empty[st]), ((it / S) - 1) & 1u)) {
            ok = false;
            break;
          }
          const uint32_t sa = rbase + st * geo.stage_bytes, bar = smem_addr(&full[st]);
          expect_tx(bar, tx);
          for (int cc = 0; cc < geo.cch; ++cc)
#pragma unroll
            for (int q = 0; q < STRIPS; ++q)
              tma4d(sa + (uint32_t)(cc * STRIPS + q) * STRIP, &mapA, cc * KS, ru.w0 - 1 + q, ru.h0 - 1 + r, ru.b,
                    bar);
        }
        if (!ok) {
          *abort_flag = 1;
          break;
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // ---- MMA issuer: one step per input row r of a run
      const uint64_t wdesc = make_desc_sw<SWA>(wbase, 16, 8 * SWA);
      bool ok = mbar_wait(smem_addr(&wfull), 0);
      uint32_t it = 0, ol0 = 0;  // stage counter; sequence number of the run's first output row
      for (int u = blockIdx.x; ok && u < geo.nunits && !*abort_flag; u += gridDim.x) {
        const RowsUnit ru = rows_unit(geo, u);
        for (int r = 0; ok && r < ru.rows + 2; ++r, ++it) {
          // a new output row (r) starts here: its block must be drained and zeroed
          if (r < ru.rows) {
            const uint32_t ol = ol0 + r;
            if (!mbar_wait(smem_addr(&acc_empty[ol % RB]), (ol / RB) & 1u)) {
              ok = false;
              break;
            }
          }
          if (!mbar_wait(smem_addr(&full[it % S]), (it / S) & 1u)) {
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const int lo = max(0, r - 2), hi = min(ru.rows - 1, r);
          const uint64_t sdesc = make_desc_sw<SWA>(rbase + (it % S) * geo.stage_bytes, 16, 8 * SWA);
          // the covered blocks, split where they wrap around the ring
          const int b_lo = (int)((ol0 + lo) % RB);
          const int n1 = min(hi - lo + 1, RB - b_lo);  // rows before the wrap
          for (int part = 0; part < 2; ++part) {
            const int first = part == 0 ? lo : lo + n1;
            const int cnt = part == 0 ? n1 : hi - lo + 1 - n1;
            if (cnt <= 0) continue;
            const uint32_t dtm = tmem + (uint32_t)((ol0 + first) % RB) * BN;
            const uint32_t idesc = idesc_n(cnt * BN);
            const int s0 = first - r + 2;  // slab block of output row `first`
            for (int cc = 0; cc < geo.cch; ++cc) {
              const uint64_t cdesc = sdesc + ((uint64_t)(cc * STRIPS) * STRIP >> 4);
#pragma unroll
              for (int dw = 0; dw < 3; ++dw) {
                const uint64_t da = cdesc + ((STRIPS == 2 && dw == 1 ? STRIP : (uint32_t)dw * SWA) >> 4);
                const uint64_t db =
                    wdesc + ((uint64_t)((dw * geo.cch + cc) * 3 + s0) * (BN * SWA) >> 4);
#pragma unroll
                for (int kk = 0; kk < KS / 16; ++kk) mma_bf16(dtm, da + 2 * kk, db + 2 * kk, idesc, 1u);
              }
            }
          }
          commit(smem_addr(&empty[it % S]));  // this input row has no other reader
          if (r >= 2) commit(smem_addr(&acc_full[(ol0 + r - 2) % RB]));  // output row r - 2 is complete
        }
        ol0 += ru.rows;
      }
      if (!ok) *abort_flag = 1;
    }
  } else {
    // ---- epilogue groups: group e drains the output rows ol with
    // ol % NE == e, i.e. the blocks b with b % NE == e (RB is a multiple of
    // NE); warp w reads and zeroes TMEM lanes 32 * (w % 4) ..  With tma_out
    // a row's BF16 result is written to the group's staging tile in the
    // output map's swizzled layout and leaves by one TMA store (the bias
    // comes from shared memory), instead of 16-byte stores per thread.
    constexpr bool BF = EPI == EPI_BIAS_RELU_BF16 || EPI == EPI_BIAS_BF16;
    constexpr int ROWB = BN * 2;  // bytes of one output pixel row
    const int quad = warp & 3, grp = (warp - 2) >> 2, gtid = threadIdx.x - 64 - 128 * grp;
    const uint32_t lane_base = tmem + ((uint32_t)(quad * 32) << 16);
    const bool tma_out = BF && geo.tma_out;
    const uint32_t stg = rbase + (uint32_t)S * geo.stage_bytes + (uint32_t)grp * (128u * ROWB);
    __shared__ __align__(16) float s_bias[64];
    if (tma_out) {
      if (threadIdx.x - 64 < BN) s_bias[threadIdx.x - 64] = g.bias ? g.bias[threadIdx.x - 64] : 0.f;
      named_sync(3, 128 * NE);
    }
    auto zero_block = [&](int b) {
#pragma unroll
      for (int c = 0; c < BN; c += 32) tmem_zero32(lane_base + (uint32_t)(b * BN + c));
      asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    };
    for (int b = grp; b < RB; b += NE) {
      zero_block(b);
      mbar_arrive_plain(smem_addr(&acc_empty[b]));
    }
    uint32_t ol = 0, nst = 0;
    bool ok = true;
    for (int u = blockIdx.x; ok && u < geo.nunits; u += gridDim.x) {
      const RowsUnit ru = rows_unit(geo, u);
      for (int i = 0; i < ru.rows; ++i, ++ol) {
        if ((int)(ol % NE) != grp) continue;
        const int b = (int)(ol % RB);
        if (!mbar_wait(smem_addr(&acc_full[b]), (ol / RB) & 1u)) {
          *abort_flag = 1;
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (!tma_out) {
          const int m0 = ((ru.b * geo.H + ru.h0 + i) * geo.W) + ru.w0;
          gemm_epilogue<BN, EPI>(g, lane_base + (uint32_t)(b * BN), m0 + quad * 32 + lane, 0, true);
          zero_block(b);
          mbar_arrive_plain(smem_addr(&acc_empty[b]));
          continue;
        }
        if constexpr (BF) {
        // drain and pack: pk[k] holds channels 2k, 2k+1 of this pixel
        uint32_t pk[BN / 2];
#pragma unroll
        for (int c = 0; c < BN; c += 32) {
          float v[32];
          tmem_ld32(lane_base + (uint32_t)(b * BN + c), v);
#pragma unroll
          for (int q = 0; q < 16; ++q) {
            float lo = v[2 * q] + s_bias[c + 2 * q], hi = v[2 * q + 1] + s_bias[c + 2 * q + 1];
            if (EPI == EPI_BIAS_RELU_BF16) {
              lo = fmaxf(lo, 0.f);
              hi = fmaxf(hi, 0.f);
            }
            const __nv_bfloat162 h2 = __floats2bfloat162_rn(lo, hi);
            pk[c / 2 + q] = *reinterpret_cast<const uint32_t *>(&h2);
          }
        }
        zero_block(b);
        mbar_arrive_plain(smem_addr(&acc_empty[b]));
        // the staging tile is free once the group's previous store has read
        // it (the leader waits for that and opens stg_free); bounded waits
        const uint32_t k = nst++;
        if (gtid == 0) {
          asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
          mbar_arrive_plain(smem_addr(&stg_free[grp]));
        }
        if (!mbar_wait(smem_addr(&stg_free[grp]), k & 1u)) {
          *abort_flag = 1;
          ok = false;
          break;
        }
        const int p = quad * 32 + lane;  // pixel row of the tile
#pragma unroll
        for (int j = 0; j < ROWB / 16; ++j) {
          const int sj = ROWB == 128 ? (j ^ (p & 7)) : (j ^ ((p >> 1) & 3));
          const uint32_t dst = stg + (uint32_t)(p * ROWB + sj * 16);
          asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(dst), "r"(pk[4 * j]), "r"(pk[4 * j + 1]),
                       "r"(pk[4 * j + 2]), "r"(pk[4 * j + 3])
                       : "memory");
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_arrive_plain(smem_addr(&stg_full[grp]));
        if (gtid == 0) {
          if (!mbar_wait(smem_addr(&stg_full[grp]), k & 1u)) {
            *abort_flag = 1;
            ok = false;
            break;
          }
          tma_store4d(&mapD, stg, 0, ru.w0, ru.h0 + i, ru.b);
        }
        }  // BF
      }
    }
    if (tma_out && gtid == 0) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
  }
  __syncthreads();
  if (s_abort && threadIdx.x == 0) atomicExch(g.err, 1);
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(Ro::TMEM_COLS));
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

int sm_count() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    AIRT_CHECK_CUDA(cudaGetDevice(&dev));
    AIRT_CHECK_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
  }
  return n;
}

template <int BN, int MODE, int SWA>
int persistent_ctas(int ntiles) {
  using Cfg = TmaCfg<BN, MODE, SWA>;
  return std::max(1, std::min(ntiles, sm_count() * (Cfg::TWO ? 2 : 1)));
}

template <int BN, int EPI, int MODE, int SWA, int SWB>
void launch_tma(const CUtensorMap &ma, const CUtensorMap &mb, const GemmArgs &g, const TmaGeo &geo,
                cudaStream_t s) {
  using Cfg = TmaCfg<BN, MODE, SWA>;
  auto kern = k_gemm_tma<BN, EPI, MODE, SWA, SWB>;
  AIRT_CHECK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Cfg::SMEM));
  const int ntiles = geo.tiles_m * geo.tiles_n * geo.splits;
  kern<<<persistent_ctas<BN, MODE, SWA>(ntiles), 192, Cfg::SMEM, s>>>(ma, mb, g, geo);
  AIRT_LAUNCH_CHECK();
}

template <int MODE, int SWA, int SWB>
void dispatch_tma(const CUtensorMap &ma, const CUtensorMap &mb, const GemmArgs &g, const TmaGeo &geo, int bn,
                  int epi, cudaStream_t s) {
#define AIRT_T(BNV)                                                                                     \
  switch (epi) {                                                                                        \
    case EPI_STORE_F32: launch_tma<BNV, EPI_STORE_F32, MODE, SWA, SWB>(ma, mb, g, geo, s); break;       \
    case EPI_BIAS_RELU_BF16: launch_tma<BNV, EPI_BIAS_RELU_BF16, MODE, SWA, SWB>(ma, mb, g, geo, s); break; \
    case EPI_BIAS_BF16: launch_tma<BNV, EPI_BIAS_BF16, MODE, SWA, SWB>(ma, mb, g, geo, s); break;       \
    case EPI_ADD_F32: launch_tma<BNV, EPI_ADD_F32, MODE, SWA, SWB>(ma, mb, g, geo, s); break;           \
    default: launch_tma<BNV, EPI_ATOMIC_F32_T, MODE, SWA, SWB>(ma, mb, g, geo, s); break;               \
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

int swizzle_for(int c) { return c % 64 == 0 ? 128 : c % 32 == 0 ? 64 : 32; }

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
  TmaGeo geo{};
  geo.tiles_m = (g.M + BM - 1) / BM;
  geo.tiles_n = (g.N + bn - 1) / bn;
  geo.splits = (g.K + g.ksplit - 1) / g.ksplit;
  geo.K = g.K;
  geo.ksplit = g.ksplit;
  dispatch_tma<MODE_DENSE, 128, 128>(ma, mb, g, geo, bn, epi, s);
}

// Box of `pix` consecutive NHWC pixels as a (bw, bh, bb) rectangle, or false
// when the image shape does not tile that way.
static bool pixel_box(int pix, int H, int W, int &bw, int &bh, int &bb) {
  if (W >= pix) {
    if (W % pix) return false;
    bw = pix, bh = 1, bb = 1;
    return true;
  }
  if (pix % W) return false;
  bw = W;
  const int rows = pix / W;
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
         g.ldb % 8 == 0 && g.M % (g.conv_H * g.conv_W) == 0 && pixel_box(128, g.conv_H, g.conv_W, bw, bh, bb);
}

int g_conv_halo = 3;
int g_conv_one_strip = 0;

// MODE_HALO launch: tiles lie within one image row (W % 128 == 0) and the
// channels fill whole 64- or 128-byte rows.
static bool conv3x3_halo(const GemmArgs &g, int bn, int epi, cudaStream_t s) {
  const int C = g.conv_C, H = g.conv_H, W = g.conv_W, Bimg = g.M / (H * W);
  const int sw = swizzle_for(C), ks = sw / 2;
  // the three taps' weight slices of a stage stay within 24 KB, so that two
  // CTAs per SM keep at least two stages each
  if (!g_conv_halo || W % 128 != 0 || sw < 64 || W > 4096 || 3 * bn * sw > 24576) return false;
  const cuuint64_t dx[4] = {(cuuint64_t)C, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)Bimg};
  const cuuint64_t sx[3] = {(cuuint64_t)C * 2, (cuuint64_t)W * C * 2, (cuuint64_t)H * W * C * 2};
  const cuuint32_t bx[4] = {(cuuint32_t)ks, (cuuint32_t)kStripBox, 1, 1};
  const CUtensorMap ma = make_map(g.convX, 4, dx, sx, bx, sw);
  const cuuint64_t dw[2] = {(cuuint64_t)9 * C, (cuuint64_t)g.N}, swt[1] = {(cuuint64_t)g.ldb * 2};
  const cuuint32_t bwt[2] = {(cuuint32_t)ks, (cuuint32_t)bn};
  const CUtensorMap mb = make_map(g.B, 2, dw, swt, bwt, sw);
  TmaGeo geo{};
  geo.W = W;
  geo.H = H;
  geo.C = C;
  geo.cchunks = C / ks;
  geo.tiles_m = (g.M + BM - 1) / BM;
  geo.tiles_n = (g.N + bn - 1) / bn;
  geo.splits = 1;
  if (sw == 128) dispatch_tma<MODE_HALO, 128, 128>(ma, mb, g, geo, bn, epi, s);
  else dispatch_tma<MODE_HALO, 64, 64>(ma, mb, g, geo, bn, epi, s);
  return true;
}

template <int BN, int EPI, int SWA, bool ONE>
static void launch_rows(const CUtensorMap &ma, const CUtensorMap &mb, const GemmArgs &g, const RowsGeo &geo,
                        size_t smem, int ctas, cudaStream_t s) {
  auto kern = k_conv_rows<BN, EPI, SWA, ONE>;
  AIRT_CHECK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  kern<<<ctas, RowsRoles<BN>::THREADS, smem, s>>>(ma, mb, g, geo);
  AIRT_LAUNCH_CHECK();
}

// Row-run launch (k_conv_rows): W % 128 == 0, 64- or 128-byte pixel rows, one
// output-channel tile, and the resident weights plus four ring stages within
// the shared memory of one CTA (two per SM when that fits in half).
static bool conv3x3_rows(const GemmArgs &g, int bn, int epi, cudaStream_t s) {
  const int C = g.conv_C, H = g.conv_H, W = g.conv_W, Bimg = g.M / (H * W);
  const int sw = swizzle_for(C), ks = sw / 2;
  if (g_conv_halo < 2 || W % 128 != 0 || sw < 64 || W > 4096 || g.N != bn || bn > 128) return false;
  RowsGeo geo{};
  geo.W = W;
  geo.H = H;
  geo.cch = C / ks;
  const uint32_t strip = round1k((uint32_t)kStripRows * sw);
  const bool one = sw == 64 && g_conv_one_strip;
  geo.stage_bytes = (uint32_t)geo.cch * (sw == 128 || one ? 1u : 2u) * strip;
  geo.w_bytes = (uint32_t)(9 * geo.cch) * (uint32_t)bn * (uint32_t)sw;
  const uint32_t half = 112640u, whole = 225280u;  // per-CTA budgets: two CTAs or one per SM
  int per_sm = 2;
  uint32_t budget = half;
  if (geo.w_bytes + 4 * geo.stage_bytes + 1024 > half) {
    per_sm = 1;
    budget = whole;
  }
  if (geo.w_bytes + 4 * geo.stage_bytes + 1024 > budget) return false;
  geo.S = std::min<int>(kRowsMaxStages, (int)((budget - 1024 - geo.w_bytes) / geo.stage_bytes));
  const size_t smem = (size_t)geo.w_bytes + (size_t)geo.S * geo.stage_bytes + 1024;
  geo.segs = W / 128;
  const int ctas = sm_count() * per_sm;
  // rows per run (any R up to H; the last run of a column may be shorter):
  // the fewest input rows on the busiest CTA, ceil(units/ctas) * (R + 2)
  long best = -1;
  for (int R = 1; R <= H; ++R) {
    const long units = (long)Bimg * geo.segs * ((H + R - 1) / R);
    const long cost = ((units + ctas - 1) / ctas) * (R + 2);
    if (best < 0 || cost < best) {
      best = cost;
      geo.R = R;
    }
  }
  geo.hblocks = (H + geo.R - 1) / geo.R;
  geo.nunits = Bimg * geo.segs * geo.hblocks;
  const cuuint64_t dx[4] = {(cuuint64_t)C, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)Bimg};
  const cuuint64_t sx[3] = {(cuuint64_t)C * 2, (cuuint64_t)W * C * 2, (cuuint64_t)H * W * C * 2};
  const cuuint32_t bx[4] = {(cuuint32_t)ks, (cuuint32_t)kStripBox, 1, 1};
  const CUtensorMap ma = make_map(g.convX, 4, dx, sx, bx, sw);
  const cuuint64_t dw[2] = {(cuuint64_t)9 * C, (cuuint64_t)g.N}, swt[1] = {(cuuint64_t)g.ldb * 2};
  const cuuint32_t bwt[2] = {(cuuint32_t)ks, (cuuint32_t)bn};
  const CUtensorMap mb = make_map(g.B, 2, dw, swt, bwt, sw);
  const int grid = std::max(1, std::min(geo.nunits, ctas));
#define AIRT_R(BNV, SWV, ONEV)                                                                            \
  switch (epi) {                                                                                          \
    case EPI_STORE_F32: launch_rows<BNV, EPI_STORE_F32, SWV, ONEV>(ma, mb, g, geo, smem, grid, s); break; \
    case EPI_BIAS_RELU_BF16:                                                                              \
      launch_rows<BNV, EPI_BIAS_RELU_BF16, SWV, ONEV>(ma, mb, g, geo, smem, grid, s);                     \
      break;                                                                                              \
    case EPI_BIAS_BF16: launch_rows<BNV, EPI_BIAS_BF16, SWV, ONEV>(ma, mb, g, geo, smem, grid, s); break; \
    case EPI_ADD_F32: launch_rows<BNV, EPI_ADD_F32, SWV, ONEV>(ma, mb, g, geo, smem, grid, s); break;     \
    default: return false;                                                                                \
  }
  if (sw == 128) {
    switch (bn) {
      case 32: AIRT_R(32, 128, false) break;
      case 64: AIRT_R(64, 128, false) break;
      default: AIRT_R(128, 128, false) break;
    }
  } else if (one) {
    switch (bn) {
      case 32: AIRT_R(32, 64, true) break;
      case 64: AIRT_R(64, 64, true) break;
      default: AIRT_R(128, 64, true) break;
    }
  } else {
    switch (bn) {
      case 32: AIRT_R(32, 64, false) break;
      case 64: AIRT_R(64, 64, false) break;
      default: AIRT_R(128, 64, false) break;
    }
  }
#undef AIRT_R
  return true;
}

template <int BN, int EPI, int SWA, bool ONE>
static void launch_stack(const CUtensorMap &ma, const CUtensorMap &mb, const CUtensorMap &md, const GemmArgs &g,
                         const RowsGeo &geo, size_t smem, int ctas, cudaStream_t s) {
  auto kern = k_conv_stack<BN, EPI, SWA, ONE>;
  AIRT_CHECK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  kern<<<ctas, StackRoles<BN>::THREADS, smem, s>>>(ma, mb, md, g, geo);
  AIRT_LAUNCH_CHECK();
}

// Stacked row-run launch (k_conv_stack): as the row runs, with BN = 32 or 64
// (N = 3 BN <= 256) and 256 TMEM columns per CTA.
static bool conv3x3_stack(const GemmArgs &g, int bn, int epi, cudaStream_t s) {
  const int C = g.conv_C, H = g.conv_H, W = g.conv_W, Bimg = g.M / (H * W);
  const int sw = swizzle_for(C), ks = sw / 2;
  if (g_conv_halo != 3 || W % 128 != 0 || sw < 64 || W > 4096 || g.N != bn || (bn != 32 && bn != 64))
    return false;
  RowsGeo geo{};
  geo.W = W;
  geo.H = H;
  geo.cch = C / ks;
  const uint32_t strip = round1k((uint32_t)kStripRows * sw);
  geo.stage_bytes = (uint32_t)geo.cch * (sw == 128 ? 1u : 2u) * strip;
  geo.w_bytes = (uint32_t)(9 * geo.cch) * (uint32_t)bn * (uint32_t)sw;
  // with 64-byte pixel rows the middle tap reads a second strip one pixel
  // later; where four stages of two strips do not fit, one strip serves all
  // three taps (shifted by 64 bytes)
  bool one = false;
  geo.tma_out = (epi == EPI_BIAS_RELU_BF16 || epi == EPI_BIAS_BF16) && g.ldd == g.N &&
                ((uintptr_t)g.D & 15) == 0;
  const uint32_t fixed = geo.w_bytes + (geo.tma_out ? 2u * 128u * (uint32_t)bn * 2u : 0u) + 1024u;
  const uint32_t half = 112640u, whole = 225280u;
  if (sw == 64 && fixed + 4 * geo.stage_bytes > whole) {
    one = true;
    geo.stage_bytes /= 2;
  }
  int per_sm = 2;
  uint32_t budget = half;
  if (fixed + 4 * geo.stage_bytes > half) {
    per_sm = 1;
    budget = whole;
  }
  if (fixed + 4 * geo.stage_bytes > budget) return false;
  geo.S = std::min<int>(kRowsMaxStages, (int)((budget - fixed) / geo.stage_bytes));
  const size_t smem = (size_t)fixed + (size_t)geo.S * geo.stage_bytes;
  geo.segs = W / 128;
  const int ctas = sm_count() * per_sm;
  long best = -1;
  for (int R = 1; R <= H; ++R) {
    const long units = (long)Bimg * geo.segs * ((H + R - 1) / R);
    const long cost = ((units + ctas - 1) / ctas) * (R + 2);
    if (best < 0 || cost < best) {
      best = cost;
      geo.R = R;
    }
  }
  geo.hblocks = (H + geo.R - 1) / geo.R;
  geo.nunits = Bimg * geo.segs * geo.hblocks;
  const cuuint64_t dx[4] = {(cuuint64_t)C, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)Bimg};
  const cuuint64_t sx[3] = {(cuuint64_t)C * 2, (cuuint64_t)W * C * 2, (cuuint64_t)H * W * C * 2};
  const cuuint32_t bx[4] = {(cuuint32_t)ks, (cuuint32_t)kStripBox, 1, 1};
  const CUtensorMap ma = make_map(g.convX, 4, dx, sx, bx, sw);
  const cuuint64_t dw[2] = {(cuuint64_t)9 * C, (cuuint64_t)g.N}, swt[1] = {(cuuint64_t)g.ldb * 2};
  const cuuint32_t bwt[2] = {(cuuint32_t)ks, (cuuint32_t)bn};
  const CUtensorMap mb = make_map(g.B, 2, dw, swt, bwt, sw);
  CUtensorMap md = ma;  // unused without tma_out
  if (geo.tma_out) {
    const cuuint64_t dd[4] = {(cuuint64_t)g.N, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)Bimg};
    const cuuint64_t sd[3] = {(cuuint64_t)g.N * 2, (cuuint64_t)W * g.N * 2, (cuuint64_t)H * W * g.N * 2};
    const cuuint32_t bd[4] = {(cuuint32_t)bn, 128, 1, 1};
    md = make_map(g.D, 4, dd, sd, bd, bn * 2);
  }
  const int grid = std::max(1, std::min(geo.nunits, ctas));
#define AIRT_S(BNV, SWV, ONEV)                                                                            \
  switch (epi) {                                                                                          \
    case EPI_STORE_F32: launch_stack<BNV, EPI_STORE_F32, SWV, ONEV>(ma, mb, md, g, geo, smem, grid, s); break; \
    case EPI_BIAS_RELU_BF16:                                                                              \
      launch_stack<BNV, EPI_BIAS_RELU_BF16, SWV, ONEV>(ma, mb, md, g, geo, smem, grid, s);                \
      break;                                                                                              \
    case EPI_BIAS_BF16: launch_stack<BNV, EPI_BIAS_BF16, SWV, ONEV>(ma, mb, md, g, geo, smem, grid, s); break; \
    case EPI_ADD_F32: launch_stack<BNV, EPI_ADD_F32, SWV, ONEV>(ma, mb, md, g, geo, smem, grid, s); break; \
    default: return false;                                                                                \
  }
  if (sw == 128) {
    if (bn == 32) { AIRT_S(32, 128, false) } else { AIRT_S(64, 128, false) }
  } else if (one) {
    if (bn == 32) { AIRT_S(32, 64, true) } else { AIRT_S(64, 64, true) }
  } else {
    if (bn == 32) { AIRT_S(32, 64, false) } else { AIRT_S(64, 64, false) }
  }
#undef AIRT_S
  return true;
}

void conv3x3_bf16_tma(const GemmArgs &g, int bn, int epi, cudaStream_t s) {
  AIRT_REQUIRE(conv3x3_tma_ok(g), "conv3x3: shape unsuitable for TMA");
  if (conv3x3_stack(g, bn, epi, s)) return;
  if (conv3x3_rows(g, bn, epi, s)) return;
  if (conv3x3_halo(g, bn, epi, s)) return;
  const int C = g.conv_C, H = g.conv_H, W = g.conv_W, Bimg = g.M / (H * W);
  const int sw = swizzle_for(C), ks = sw / 2;
  int bw, bh, bb;
  pixel_box(128, H, W, bw, bh, bb);
  const cuuint64_t dx[4] = {(cuuint64_t)C, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)Bimg};
  const cuuint64_t sx[3] = {(cuuint64_t)C * 2, (cuuint64_t)W * C * 2, (cuuint64_t)H * W * C * 2};
  const cuuint32_t bx[4] = {(cuuint32_t)ks, (cuuint32_t)bw, (cuuint32_t)bh, (cuuint32_t)bb};
  const CUtensorMap ma = make_map(g.convX, 4, dx, sx, bx, sw);
  const cuuint64_t dw[2] = {(cuuint64_t)9 * C, (cuuint64_t)g.N}, swt[1] = {(cuuint64_t)g.ldb * 2};
  const cuuint32_t bwt[2] = {(cuuint32_t)ks, (cuuint32_t)bn};
  const CUtensorMap mb = make_map(g.B, 2, dw, swt, bwt, sw);
  TmaGeo geo{};
  geo.W = W;
  geo.H = H;
  geo.C = C;
  geo.cchunks = C / ks;
  geo.tiles_m = (g.M + BM - 1) / BM;
  geo.tiles_n = (g.N + bn - 1) / bn;
  geo.splits = 1;
  if (sw == 128) dispatch_tma<MODE_CONV, 128, 128>(ma, mb, g, geo, bn, epi, s);
  else if (sw == 64) dispatch_tma<MODE_CONV, 64, 64>(ma, mb, g, geo, bn, epi, s);
  else dispatch_tma<MODE_CONV, 32, 32>(ma, mb, g, geo, bn, epi, s);
}

bool conv3x3_wgrad_tma_ok(const GemmArgs &g) {
  int bw, bh, bb;
  return g.conv_C % 16 == 0 && g.N % 16 == 0 && ((uintptr_t)g.convX & 15) == 0 &&
         ((uintptr_t)g.B & 15) == 0 && g.ldb == g.N && g.K % (g.conv_H * g.conv_W) == 0 &&
         pixel_box(64, g.conv_H, g.conv_W, bw, bh, bb);
}

void conv3x3_wgrad_bf16_tma(const GemmArgs &g, int bn, cudaStream_t s) {
  AIRT_REQUIRE(conv3x3_wgrad_tma_ok(g), "conv3x3: shape unsuitable for TMA");
  const int C = g.conv_C, H = g.conv_H, W = g.conv_W, P = g.K, Bimg = P / (H * W);
  const int swa = swizzle_for(C), swb = swizzle_for(g.N);
  int bw, bh, bb;
  pixel_box(64, H, W, bw, bh, bb);
  const cuuint64_t dx[4] = {(cuuint64_t)C, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)Bimg};
  const cuuint64_t sx[3] = {(cuuint64_t)C * 2, (cuuint64_t)W * C * 2, (cuuint64_t)H * W * C * 2};
  const cuuint32_t bx[4] = {(cuuint32_t)(swa / 2), (cuuint32_t)bw, (cuuint32_t)bh, (cuuint32_t)bb};
  const CUtensorMap ma = make_map(g.convX, 4, dx, sx, bx, swa);
  const cuuint64_t dy[2] = {(cuuint64_t)g.N, (cuuint64_t)P}, sy[1] = {(cuuint64_t)g.ldb * 2};
  const cuuint32_t by[2] = {(cuuint32_t)(swb / 2), 64};
  const CUtensorMap mb = make_map(g.B, 2, dy, sy, by, swb);
  TmaGeo geo{};
  geo.W = W;
  geo.H = H;
  geo.C = C;
  geo.tiles_m = (g.M + BM - 1) / BM;
  geo.tiles_n = (g.N + bn - 1) / bn;
  // split the pixels so that about two tiles fall to each CTA
  const int ctas = sm_count() * (bn <= 128 ? 2 : 1);
  const int want = std::max(1, (2 * ctas + geo.tiles_m * geo.tiles_n - 1) / (geo.tiles_m * geo.tiles_n));
  geo.ksplit = std::max(64, (((P + want - 1) / want) + 63) / 64 * 64);
  geo.splits = (P + geo.ksplit - 1) / geo.ksplit;
  geo.K = P;
#define AIRT_W(SA, SB) dispatch_tma<MODE_WGRAD, SA, SB>(ma, mb, g, geo, bn, EPI_ATOMIC_F32_T, s)
  if (swa == 128) {
    if (swb == 128) AIRT_W(128, 128); else if (swb == 64) AIRT_W(128, 64); else AIRT_W(128, 32);
  } else if (swa == 64) {
    if (swb == 128) AIRT_W(64, 128); else if (swb == 64) AIRT_W(64, 64); else AIRT_W(64, 32);
  } else {
    if (swb == 128) AIRT_W(32, 128); else if (swb == 64) AIRT_W(32, 64); else AIRT_W(32, 32);
  }
#undef AIRT_W
}

}  // namespace airt
