// tcgen05 BF16 GEMM kernel (see umma.cuh for the scheme).
#include "umma.cuh"

namespace airt {

namespace {

using namespace umma;

__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src, bool valid) {
  const int n = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(n) : "memory");
}

// Stage one operand tile (R rows of the M or N dimension, BK of K) into the
// canonical layout.  k0: first K index of the slice; kend: end of this
// CTA's K range; rows: extent of the M/N dimension.
template <int R, bool MN>
__device__ __forceinline__ void stage_tile(uint32_t sbase, const __nv_bfloat16 *G, int ld, int r0,
                                           int rows, int k0, int kend) {
  constexpr int CHUNKS = R * BK / 8;
  for (int c = threadIdx.x; c < CHUNKS; c += kProducers) {
    if (!MN) {
      // K-major: thread -> row (fastest), then K chunk
      const int r = c % R, kc = c / R;
      const int gr = r0 + r, gk = k0 + kc * 8;
      const bool ok = gr < rows && gk < kend;
      const __nv_bfloat16 *src = ok ? G + (size_t)gr * ld + gk : G;
      cp_async16(sbase + kmaj_off<R>(r, kc), src, ok);
    } else {
      // MN-major: 8 consecutive K rows per 8 threads, then MN chunk, then K group
      const int k8 = c & 7, rc = (c >> 3) % (R / 8), kg = c / R;
      const int k = kg * 8 + k8;
      const int gk = k0 + k, gr = r0 + rc * 8;
      const bool ok = gr < rows && gk < kend;
      const __nv_bfloat16 *src = ok ? G + (size_t)gk * ld + gr : G;
      cp_async16(sbase + mnmaj_off<R>(rc, k), src, ok);
    }
  }
}

// Implicit 3x3 convolution operand gathers.  kProducers == BM, so in the
// K-major A tile every thread owns one pixel row (threadIdx.x) for the whole
// CTA; its coordinates and the 9-bit mask of in-image taps are decoded once.
struct ConvRow {
  const __nv_bfloat16 *px;  // this pixel's channel vector
  uint32_t taps;            // bit t: tap t lies inside the image
};

__device__ __forceinline__ uint32_t tap_mask(int h, int w, int H, int W) {
  uint32_t m = 0;
#pragma unroll
  for (int t = 0; t < 9; ++t) {
    const int hh = h + t / 3 - 1, ww = w + t % 3 - 1;
    if (hh >= 0 && hh < H && ww >= 0 && ww < W) m |= 1u << t;
  }
  return m;
}

__device__ __forceinline__ ConvRow conv_row(const GemmArgs &g, int p) {
  ConvRow r{g.convX, 0u};
  if (p < g.M) {
    const int w = p % g.conv_W, q = p / g.conv_W, h = q % g.conv_H;
    r.px = g.convX + (size_t)p * g.conv_C;
    r.taps = tap_mask(h, w, g.conv_H, g.conv_W);
  }
  return r;
}

// A tile of a K slice starting at k0: chunk kc = 8 channels of one tap.
__device__ __forceinline__ void stage_conv_tile(uint32_t sbase, const GemmArgs &g, const ConvRow &row,
                                                int k0) {
  const int C = g.conv_C, W = g.conv_W;
  int tap = k0 / C, ci = k0 - tap * C;
#pragma unroll
  for (int kc = 0; kc < BK / 8; ++kc) {
    const bool ok = tap < 9 && ((row.taps >> tap) & 1u);
    const __nv_bfloat16 *src =
        ok ? row.px + ((tap / 3 - 1) * W + (tap % 3 - 1)) * C + ci : g.convX;
    cp_async16(sbase + kmaj_off<BM>(threadIdx.x, kc), src, ok);
    ci += 8;
    if (ci == C) {
      ci = 0;
      ++tap;
    }
  }
}

// A^T tile for the weight gradient (MN-major: M = convolution K index, K =
// pixel).  Thread -> (pixel k8 = tid % 8 of each group of 8, M chunk
// rc = (tid / 8) % 16), so its tap and channel offset are fixed for the CTA;
// the pixels it visits are k0 + 8*i + k8, i = 0..7, walked incrementally.
struct ConvCol {
  int tap, ci;  // convolution K index m0 + rc*8 -> (tap, ci); tap >= 9: padding
};

__device__ __forceinline__ ConvCol conv_col(const GemmArgs &g, int m0) {
  const int kk = m0 + ((threadIdx.x >> 3) % (BM / 8)) * 8;
  const int tap = kk / g.conv_C;
  return ConvCol{tap, kk - tap * g.conv_C};
}

__device__ __forceinline__ void stage_conv_tile_mn(uint32_t sbase, const GemmArgs &g, const ConvCol &col,
                                                   int k0, int kend) {
  const int C = g.conv_C, H = g.conv_H, W = g.conv_W;
  const int k8 = threadIdx.x & 7, rc = (threadIdx.x >> 3) % (BM / 8);
  const int dh = col.tap / 3 - 1, dw = col.tap % 3 - 1;
  int p = k0 + k8;
  int w = p % W, q = p / W, h = q % H;
  const ptrdiff_t shift = ((ptrdiff_t)dh * W + dw) * C + col.ci;
#pragma unroll
  for (int i = 0; i < BK / 8; ++i) {
    const int hh = h + dh, ww = w + dw;
    const bool ok = col.tap < 9 && p < kend && hh >= 0 && hh < H && ww >= 0 && ww < W;
    const __nv_bfloat16 *src = ok ? g.convX + ((ptrdiff_t)p * C + shift) : g.convX;
    cp_async16(sbase + mnmaj_off<BM>(rc, i * 8 + k8), src, ok);
    p += 8;
    w += 8;
    while (w >= W) {
      w -= W;
      if (++h == H) h = 0;
    }
  }
}

// Pipeline depth per N tile width: two CTAs per SM (about 100 KB of shared
// memory each) up to BN = 128, one CTA with four stages at BN = 256.
template <int BN>
struct Stages {
  static constexpr int value = BN == 32 ? 5 : BN == 64 ? 4 : BN == 128 ? 3 : 4;
};

__device__ __forceinline__ void cp_async_arrive(uint32_t bar) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// Warp-specialised tile: warps 0-3 gather operand slices into an S-stage
// shared-memory ring with cp.async (each thread's copies complete onto the
// stage's `full` barrier), warp 4 lane 0 issues the tcgen05 MMAs of a stage
// once it is full and commits them to the stage's `empty` barrier, and after
// the last stage to `done`; warps 0-3 then drain TMEM in the epilogue.
// Every wait is bounded; a wait that gives up sets g.err and the tile is
// skipped.
template <int BN, bool A_MN, bool B_MN, int EPI, int CONV = 0>
__global__ void __launch_bounds__(kGemmThreads) k_gemm(GemmArgs g) {
  constexpr int S = Stages<BN>::value;
  constexpr uint32_t A_BYTES = BM * BK * 2, B_BYTES = BN * BK * 2, ST_BYTES = A_BYTES + B_BYTES;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char *base = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const uint32_t sbase = smem_addr(base);
  __shared__ __align__(8) uint64_t full[S], empty[S], done;
  __shared__ uint32_t s_tmem;
  __shared__ int s_abort;
  volatile int *abort_flag = &s_abort;

  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  const int kb = blockIdx.z * g.ksplit;
  const int ke = min(g.K, kb + g.ksplit);
  const int nk = ke > kb ? (ke - kb + BK - 1) / BK : 0;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_addr(&s_tmem)),
                 "r"((uint32_t)BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (threadIdx.x == 0) {
    s_abort = 0;
    for (int i = 0; i < S; ++i) {
      mbar_init(smem_addr(&full[i]), kProducers);
      mbar_init(smem_addr(&empty[i]), 1);
    }
    mbar_init(smem_addr(&done), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = s_tmem;

  if (threadIdx.x < kProducers) {
    // ---- producers
    ConvRow crow{};
    ConvCol ccol{};
    if (CONV == 1) crow = conv_row(g, m0 + threadIdx.x);
    if (CONV == 2) ccol = conv_col(g, m0);
    for (int k = 0; k < nk; ++k) {
      const int st = k % S;
      if (k >= S && !mbar_wait(smem_addr(&empty[st]), (uint32_t)((k / S - 1) & 1))) {
        *abort_flag = 1;
        break;
      }
      if (*abort_flag) break;
      const uint32_t sa = sbase + st * ST_BYTES, sb = sa + A_BYTES;
      const int k0 = kb + k * BK;
      if (CONV == 1) stage_conv_tile(sa, g, crow, k0);
      else if (CONV == 2) stage_conv_tile_mn(sa, g, ccol, k0, ke);
      else stage_tile<BM, A_MN>(sa, g.A, g.lda, m0, g.M, k0, ke);
      stage_tile<BN, B_MN>(sb, g.B, g.ldb, n0, g.N, k0, ke);
      cp_async_arrive(smem_addr(&full[st]));
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
  } else if (lane == 0) {
    // ---- MMA issuer (warp 4, one thread)
    constexpr uint32_t idesc = make_idesc<BN, A_MN, B_MN>();
    int issued = 0;
    for (int k = 0; k < nk; ++k) {
      const int st = k % S;
      if (!mbar_wait(smem_addr(&full[st]), (uint32_t)((k / S) & 1))) {
        *abort_flag = 1;
        break;
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t sa = sbase + st * ST_BYTES, sb = sa + A_BYTES;
#pragma unroll
      for (int kk = 0; kk < BK / 16; ++kk) {
        const uint64_t da = make_desc(sa + kk * 2 * (BM * 16), BM * 16, 128);
        const uint64_t db = make_desc(sb + kk * 2 * (BN * 16), BN * 16, 128);
        mma_bf16(tmem, da, db, idesc, (k > 0 || kk > 0) ? 1u : 0u);
      }
      commit(smem_addr(&empty[st]));
      ++issued;
    }
    if (issued > 0) commit(smem_addr(&done));  // arrives when every issued MMA has completed
    else mbar_arrive(smem_addr(&done));
  }
  // ---- epilogue: warps 0-3 wait for the accumulator
  if (threadIdx.x < kProducers && !mbar_wait(smem_addr(&done), 0u)) *abort_flag = 1;
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  __syncthreads();
  if (s_abort) {
    if (threadIdx.x == 0) atomicExch(g.err, 1);
  } else if (threadIdx.x < kProducers) {
    gemm_epilogue<BN, EPI>(g, tmem + ((uint32_t)(warp * 32) << 16), m0 + warp * 32 + lane, n0, nk > 0);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)BN));
}

template <int BN, bool A_MN, bool B_MN, int EPI, int CONV = 0>
void launch(const GemmArgs &g, cudaStream_t s) {
  const size_t smem = Stages<BN>::value * (size_t)(BM * BK * 2 + BN * BK * 2) + 1024;
  auto kern = k_gemm<BN, A_MN, B_MN, EPI, CONV>;
  AIRT_CHECK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int splits = g.ksplit > 0 ? (g.K + g.ksplit - 1) / g.ksplit : 1;
  dim3 grid((g.M + BM - 1) / BM, (g.N + BN - 1) / BN, splits > 0 ? splits : 1);
  kern<<<grid, kGemmThreads, smem, s>>>(g);
  AIRT_LAUNCH_CHECK();
}

template <int BN>
void dispatch_epi(const GemmArgs &g, bool a_mn, bool b_mn, int epi, cudaStream_t s) {
#define AIRT_G(AM, BMJ)                                                           \
  switch (epi) {                                                                  \
    case EPI_STORE_F32: launch<BN, AM, BMJ, EPI_STORE_F32>(g, s); break;          \
    case EPI_BIAS_RELU_BF16: launch<BN, AM, BMJ, EPI_BIAS_RELU_BF16>(g, s); break; \
    case EPI_BIAS_BF16: launch<BN, AM, BMJ, EPI_BIAS_BF16>(g, s); break;          \
    default: launch<BN, AM, BMJ, EPI_ATOMIC_F32_T>(g, s); break;                  \
  }
  if (!a_mn && !b_mn) { AIRT_G(false, false) }
  else if (!a_mn && b_mn) { AIRT_G(false, true) }
  else if (a_mn && !b_mn) { AIRT_G(true, false) }
  else { AIRT_G(true, true) }
#undef AIRT_G
}

}  // namespace

int g_gemm_path = 0;

void conv3x3_bf16(const GemmArgs &g0, int bn, int epi, cudaStream_t s) {
  if (g_gemm_path == 0 && conv3x3_tma_ok(g0)) {
    conv3x3_bf16_tma(g0, bn, epi, s);
    return;
  }
  GemmArgs g = g0;
  AIRT_REQUIRE(g.convX && g.conv_C % 8 == 0 && g.conv_C > 0, "conv3x3: channels must be a multiple of 8");
  AIRT_REQUIRE(((uintptr_t)g.convX & 15) == 0 && ((uintptr_t)g.B & 15) == 0 && g.ldb % 8 == 0,
               "conv3x3: operands must be 16-byte aligned");
  AIRT_REQUIRE(g.K % BK == 0, "conv3x3: K must be padded to a multiple of 64");
  AIRT_REQUIRE(epi == EPI_BIAS_RELU_BF16 || epi == EPI_BIAS_BF16 || epi == EPI_ADD_F32,
               "conv3x3: unsupported epilogue");
  g.ksplit = g.K;
#define AIRT_C(BNV)                                                                     \
  if (epi == EPI_BIAS_RELU_BF16) launch<BNV, false, false, EPI_BIAS_RELU_BF16, 1>(g, s); \
  else if (epi == EPI_BIAS_BF16) launch<BNV, false, false, EPI_BIAS_BF16, 1>(g, s);      \
  else launch<BNV, false, false, EPI_ADD_F32, 1>(g, s);
  switch (bn) {
    case 32: AIRT_C(32) break;
    case 64: AIRT_C(64) break;
    case 128: AIRT_C(128) break;
    case 256: AIRT_C(256) break;
    default: AIRT_REQUIRE(false, "conv3x3: BN must be 32, 64, 128 or 256");
  }
#undef AIRT_C
}

void conv3x3_wgrad_bf16(const GemmArgs &g0, int bn, cudaStream_t s) {
  if (g_gemm_path == 0 && conv3x3_wgrad_tma_ok(g0)) {
    conv3x3_wgrad_bf16_tma(g0, bn, s);
    return;
  }
  GemmArgs g = g0;
  AIRT_REQUIRE(g.convX && g.conv_C % 8 == 0 && g.conv_C > 0, "conv3x3: channels must be a multiple of 8");
  AIRT_REQUIRE(((uintptr_t)g.convX & 15) == 0 && ((uintptr_t)g.B & 15) == 0 && g.ldb % 8 == 0,
               "conv3x3: operands must be 16-byte aligned");
  AIRT_REQUIRE(g.M % 8 == 0 && g.N % 8 == 0 && g.M > 0 && g.N > 0 && g.K > 0, "conv3x3: bad sizes");
  if (g.ksplit <= 0) g.ksplit = g.K;
  AIRT_REQUIRE(g.ksplit % BK == 0 || g.ksplit >= g.K, "conv3x3: ksplit must be a multiple of 64");
  switch (bn) {
    case 32: launch<32, true, true, EPI_ATOMIC_F32_T, 2>(g, s); break;
    case 64: launch<64, true, true, EPI_ATOMIC_F32_T, 2>(g, s); break;
    case 128: launch<128, true, true, EPI_ATOMIC_F32_T, 2>(g, s); break;
    case 256: launch<256, true, true, EPI_ATOMIC_F32_T, 2>(g, s); break;
    default: AIRT_REQUIRE(false, "conv3x3: BN must be 32, 64, 128 or 256");
  }
}

void gemm_bf16(const GemmArgs &g0, int bn, bool a_mn, bool b_mn, int epi, cudaStream_t s) {
  GemmArgs g = g0;
  AIRT_REQUIRE(g.M > 0 && g.N > 0 && g.K >= 0, "gemm: bad sizes");
  AIRT_REQUIRE(g.lda % 8 == 0 && g.ldb % 8 == 0, "gemm: leading dimensions must be multiples of 8");
  AIRT_REQUIRE(((uintptr_t)g.A & 15) == 0 && ((uintptr_t)g.B & 15) == 0,
               "gemm: operands must be 16-byte aligned");
  AIRT_REQUIRE(!a_mn || g.M % 8 == 0, "gemm: MN-major A needs M % 8 == 0");
  AIRT_REQUIRE(!b_mn || g.N % 8 == 0, "gemm: MN-major B needs N % 8 == 0");
  AIRT_REQUIRE(g.K % 8 == 0, "gemm: K must be a multiple of 8 (zero-padded)");
  if (g.ksplit <= 0) g.ksplit = g.K > 0 ? g.K : BK;
  AIRT_REQUIRE(g.ksplit % BK == 0 || g.ksplit >= g.K, "gemm: ksplit must be a multiple of 64");
  if (g_gemm_path == 0 && !a_mn && !b_mn && gemm_tma_ok(g)) {
    gemm_bf16_tma(g, bn, epi, s);
    return;
  }
  switch (bn) {
    case 32: dispatch_epi<32>(g, a_mn, b_mn, epi, s); break;
    case 64: dispatch_epi<64>(g, a_mn, b_mn, epi, s); break;
    case 128: dispatch_epi<128>(g, a_mn, b_mn, epi, s); break;
    case 256: dispatch_epi<256>(g, a_mn, b_mn, epi, s); break;
    default: AIRT_REQUIRE(false, "gemm: BN must be 32, 64, 128 or 256");
  }
}

}  // namespace airt

// Test hook: operand path of the GEMM kernels (0 = TMA where possible,
// 1 = cp.async only).
extern "C" int airt_test_gemm_path(int path) {
  if (path < 0 || path > 1) return AIRT_ERR_ARG;
  airt::g_gemm_path = path;
  return AIRT_OK;
}

// Test hook: operand form of the TMA 3x3 convolution (see g_conv_halo).
// mode 0-3: g_conv_halo; + 4: one strip per input row in the row runs.
extern "C" int airt_test_conv_halo(int mode) {
  if (mode < 0 || mode > 7) return AIRT_ERR_ARG;
  airt::g_conv_halo = mode & 3;
  airt::g_conv_one_strip = (mode & 4) ? 1 : 0;
  return AIRT_OK;
}

// Test hook: D = A * B^T through the tcgen05 kernel, device pointers.
extern "C" int airt_test_gemm_bf16(int M, int N, int K, const void *A, int lda, int a_mn, const void *B,
                                   int ldb, int b_mn, float *D, int ldd, int bn, int ksplit,
                                   int atomic_t, void *stream) {
  try {
    airt::DevBuf<int> err;
    err.ensure(1);
    AIRT_CHECK_CUDA(cudaMemsetAsync(err.p, 0, sizeof(int), (cudaStream_t)stream));
    airt::GemmArgs g{};
    g.M = M;
    g.N = N;
    g.K = K;
    g.A = (const __nv_bfloat16 *)A;
    g.B = (const __nv_bfloat16 *)B;
    g.lda = lda;
    g.ldb = ldb;
    g.D = D;
    g.ldd = ldd;
    g.ksplit = ksplit;
    g.err = err.p;
    airt::gemm_bf16(g, bn, a_mn != 0, b_mn != 0,
                    atomic_t ? airt::EPI_ATOMIC_F32_T : airt::EPI_STORE_F32, (cudaStream_t)stream);
    int h = 0;
    AIRT_CHECK_CUDA(cudaMemcpyAsync(&h, err.p, sizeof(int), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    AIRT_CHECK_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    if (h) {
      airt::set_error("gemm: a bounded wait gave up");
      return AIRT_ERR_TIMEOUT;
    }
  } catch (const airt::Status &st) {
    return st.code;
  }
  return AIRT_OK;
}
