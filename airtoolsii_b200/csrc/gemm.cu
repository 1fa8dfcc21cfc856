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
  for (int c = threadIdx.x; c < CHUNKS; c += kThreads) {
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
  asm volatile("cp.async.commit_group;" ::: "memory");
}

template <int BN, bool A_MN, bool B_MN, int EPI>
__global__ void __launch_bounds__(kThreads) k_gemm(GemmArgs g) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char *base = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  constexpr uint32_t A_BYTES = BM * BK * 2, B_BYTES = BN * BK * 2;
  const uint32_t sA[2] = {smem_addr(base), smem_addr(base + A_BYTES + B_BYTES)};
  const uint32_t sB[2] = {smem_addr(base + A_BYTES), smem_addr(base + 2 * A_BYTES + B_BYTES)};
  __shared__ __align__(8) uint64_t bars[2];
  __shared__ uint32_t s_tmem;
  __shared__ int s_abort;

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
    mbar_init(smem_addr(&bars[0]), 1);
    mbar_init(smem_addr(&bars[1]), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = s_tmem;
  constexpr uint32_t idesc = make_idesc<BN, A_MN, B_MN>();

  if (nk > 0) {
    stage_tile<BM, A_MN>(sA[0], g.A, g.lda, m0, g.M, kb, ke);
    stage_tile<BN, B_MN>(sB[0], g.B, g.ldb, n0, g.N, kb, ke);
  }
  for (int it = 0; it < nk; ++it) {
    const int s = it & 1;
    if (it + 1 < nk) {
      const int s2 = (it + 1) & 1;
      if (it + 1 >= 2 && !mbar_wait(smem_addr(&bars[s2]), (uint32_t)(((it - 1) >> 1) & 1)))
        s_abort = 1;
      stage_tile<BM, A_MN>(sA[s2], g.A, g.lda, m0, g.M, kb + (it + 1) * BK, ke);
      stage_tile<BN, B_MN>(sB[s2], g.B, g.ldb, n0, g.N, kb + (it + 1) * BK, ke);
      asm volatile("cp.async.wait_group 2;" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (s_abort) break;
    if (threadIdx.x == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
      for (int kk = 0; kk < BK / 16; ++kk) {
        const uint64_t da = make_desc(sA[s] + kk * 2 * (BM * 16), BM * 16, 128);
        const uint64_t db = make_desc(sB[s] + kk * 2 * (BN * 16), BN * 16, 128);
        mma_bf16(tmem, da, db, idesc, (it > 0 || kk > 0) ? 1u : 0u);
      }
      commit(smem_addr(&bars[s]));
    }
  }
  // wait for the last slice's MMAs (the commit covers every earlier MMA)
  if (nk > 0) {
    const int last = nk - 1;
    if (!mbar_wait(smem_addr(&bars[last & 1]), (uint32_t)((last >> 1) & 1))) s_abort = 1;
  }
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  __syncthreads();
  if (s_abort) {
    if (threadIdx.x == 0) atomicExch(g.err, 1);
  } else {
    const int row = m0 + warp * 32 + lane;
#pragma unroll 1
    for (int c = 0; c < BN; c += 8) {
      float v[8];
      if (nk > 0) {
        tmem_ld8(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
      } else {
#pragma unroll
        for (int i = 0; i < 8; ++i) v[i] = 0.f;
      }
      if (row < g.M) {
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const int col = n0 + c + i;
          if (col >= g.N) continue;
          float y = v[i];
          if (EPI == EPI_STORE_F32) {
            ((float *)g.D)[(size_t)row * g.ldd + col] = y;
          } else if (EPI == EPI_BIAS_RELU_BF16 || EPI == EPI_BIAS_BF16) {
            y += g.bias ? g.bias[col] : 0.f;
            if (EPI == EPI_BIAS_RELU_BF16) y = fmaxf(y, 0.f);
            ((__nv_bfloat16 *)g.D)[(size_t)row * g.ldd + col] = __float2bfloat16(y);
          } else {
            atomicAdd((float *)g.D + (size_t)col * g.ldd + row, y);
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)BN));
}

template <int BN, bool A_MN, bool B_MN, int EPI>
void launch(const GemmArgs &g, cudaStream_t s) {
  const size_t smem = 2 * (size_t)(BM * BK * 2 + BN * BK * 2) + 1024;
  auto kern = k_gemm<BN, A_MN, B_MN, EPI>;
  AIRT_CHECK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int splits = g.ksplit > 0 ? (g.K + g.ksplit - 1) / g.ksplit : 1;
  dim3 grid((g.M + BM - 1) / BM, (g.N + BN - 1) / BN, splits > 0 ? splits : 1);
  kern<<<grid, kThreads, smem, s>>>(g);
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
  switch (bn) {
    case 32: dispatch_epi<32>(g, a_mn, b_mn, epi, s); break;
    case 64: dispatch_epi<64>(g, a_mn, b_mn, epi, s); break;
    case 128: dispatch_epi<128>(g, a_mn, b_mn, epi, s); break;
    case 256: dispatch_epi<256>(g, a_mn, b_mn, epi, s); break;
    default: AIRT_REQUIRE(false, "gemm: BN must be 32, 64, 128 or 256");
  }
}

}  // namespace airt

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
