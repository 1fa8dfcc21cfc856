// tcgen05 (5th-generation tensor core) GEMM for sm_100a, BF16 inputs, FP32
// accumulation in tensor memory.
//
//   D[M x N] (+)= A[M x K] * B[N x K]^T
//
// One CTA computes a 128 x BN tile with 5 warps:
//  * warps 0-3 stage the A and B tiles of 64-wide K slices from global
//    memory into an S-stage shared-memory ring in the canonical no-swizzle
//    UMMA layout (8 x 16-byte core matrices) with cp.async, zero-filling
//    outside the matrix; each thread's copies complete onto the stage's
//    `full` mbarrier (cp.async.mbarrier.arrive);
//  * one thread of warp 4 waits for a full stage, issues four
//    tcgen05.mma.kind::f16 (K = 16 each) and commits them to the stage's
//    `empty` mbarrier, which releases the stage to the producers;
//  * the accumulator lives in TMEM (128 lanes x BN FP32 columns); after the
//    last slice warps 0-3 read their 32 lanes each with tcgen05.ld and run
//    the epilogue (store, bias + ReLU, accumulate, or split-K atomics).
//
// Operand "majorness": K-major means the K index is contiguous in global
// memory (row-major [rows][K]); MN-major means the M (or N) index is
// contiguous (row-major [K][rows]).  Both map onto the descriptor's canonical
// layouts, so the convolution GEMMs need no transposed copies.
//
// Descriptor layouts follow the sm_100 UMMA shared-memory and instruction
// descriptors (start address, leading/stride byte offsets in 16-byte units,
// version 1, no swizzle; c=F32, a=b=BF16, N>>3, M>>4).
#pragma once

#include <cuda_bf16.h>

#include "common.cuh"

namespace airt {

namespace umma {

constexpr int BM = 128;
constexpr int BK = 64;
constexpr int kProducers = 128;                // operand-gathering and epilogue threads
constexpr int kGemmThreads = kProducers + 32;  // plus one MMA-issuing warp
constexpr long long kWaitBudget = 4000000000ll;  // ~2 s of SM clocks

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory descriptor, no swizzle.
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for sm_100
  return d;                // base offset 0, layout type 0 (no swizzle)
}

// Instruction descriptor: D = F32, A = B = BF16, M = 128, N = BN.
template <int BN, bool A_MN, bool B_MN>
__host__ __device__ constexpr uint32_t make_idesc() {
  return (1u << 4)                      // c_format F32
         | (1u << 7)                    // a_format BF16
         | (1u << 10)                   // b_format BF16
         | ((A_MN ? 1u : 0u) << 15)     // a_major
         | ((B_MN ? 1u : 0u) << 16)     // b_major
         | ((uint32_t)(BN >> 3) << 17)  // n_dim
         | ((uint32_t)(BM >> 4) << 24); // m_dim
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  const long long t0 = clock64();
  while (true) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    if (ok) return true;
    if (clock64() - t0 > kWaitBudget) return false;
  }
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
      "%13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, "
      "[%32];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
        "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
        "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
        "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8]) {
  uint32_t r[8];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

// Canonical no-swizzle K-major tile of R rows x BK: 16-byte chunk (row r,
// K chunk kc) at kc*(R*16) + (r/8)*128 + (r%8)*16.  LBO = R*16, SBO = 128.
template <int R>
__device__ __forceinline__ uint32_t kmaj_off(int r, int kc) {
  return (uint32_t)(kc * (R * 16) + (r >> 3) * 128 + (r & 7) * 16);
}

// Canonical no-swizzle MN-major tile of R (MN) x BK (K): 16-byte chunk
// (MN chunk rc = 8 consecutive MN entries, K index k) at
// (k/8)*(R*16) + rc*128 + (k%8)*16.  LBO = 128 ... see make_mn_desc.
template <int R>
__device__ __forceinline__ uint32_t mnmaj_off(int rc, int k) {
  return (uint32_t)((k >> 3) * (R * 16) + rc * 128 + (k & 7) * 16);
}

}  // namespace umma

// Epilogue kinds of the GEMM.
enum GemmEpi {
  EPI_STORE_F32 = 0,      // D -> fp32 [M][ldd]
  EPI_BIAS_RELU_BF16 = 1, // relu(D + bias[n]) -> bf16 [M][ldd]
  EPI_BIAS_BF16 = 2,      // D + bias[n] -> bf16
  EPI_ATOMIC_F32_T = 3,   // atomicAdd(D) into fp32 stored transposed [N][ldd] (split-K)
  EPI_ADD_F32 = 4,        // D += result, fp32 [M][ldd] (no split-K)
};

struct GemmArgs {
  int M, N, K;
  const __nv_bfloat16 *A;  // K-major: [M][lda]; MN-major: [K][lda]
  const __nv_bfloat16 *B;  // K-major: [N][ldb]; MN-major: [K][ldb]
  int lda, ldb;
  void *D;
  int ldd;
  const float *bias;
  int ksplit;              // K range per blockIdx.z
  int *err;
  // implicit 3x3 convolution: A is gathered from an NHWC image X (conv_C
  // channels, conv_C % 8 == 0) instead of a materialised im2col matrix;
  // K index (kh*3 + kw)*conv_C + ci, zero outside the image and for K >= 9C.
  const __nv_bfloat16 *convX;
  int conv_H, conv_W, conv_C;
};

// Epilogue of one 32-row slice of a 128 x BN tile held in TMEM, run by a
// whole warp: lane i owns tile row `row` (TMEM lane (taddr >> 16) + i); taddr
// carries the warp's lane quadrant and the accumulator's first column.
// 32 columns are read per tcgen05.ld; full, aligned 32-column slices leave
// as 16-byte vector accesses, the rest element by element.  have_acc =
// false: the tile's K range was empty and the result is zero.
template <int BN, int EPI>
__device__ __forceinline__ void gemm_epilogue(const GemmArgs &g, uint32_t taddr, int row, int n0,
                                              bool have_acc) {
  using namespace umma;
  static_assert(BN % 32 == 0, "BN must be a multiple of 32");
  const bool vec_ok = (g.ldd & 7) == 0 && ((uintptr_t)g.D & 15) == 0 &&
                      (g.bias == nullptr || ((uintptr_t)g.bias & 15) == 0);
#pragma unroll 1
  for (int c = 0; c < BN; c += 32) {
    float v[32];
    if (have_acc) {
      tmem_ld32(taddr + (uint32_t)c, v);
    } else {
#pragma unroll
      for (int i = 0; i < 32; ++i) v[i] = 0.f;
    }
    const int col0 = n0 + c;
    if (EPI != EPI_ATOMIC_F32_T && vec_ok && row < g.M && col0 + 32 <= g.N) {
      if (EPI == EPI_STORE_F32 || EPI == EPI_ADD_F32) {
        float4 *d = reinterpret_cast<float4 *>((float *)g.D + (size_t)row * g.ldd + col0);
        if (EPI == EPI_ADD_F32) {
          float4 o[8];
#pragma unroll
          for (int j = 0; j < 8; ++j) o[j] = d[j];
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            v[4 * j] += o[j].x;
            v[4 * j + 1] += o[j].y;
            v[4 * j + 2] += o[j].z;
            v[4 * j + 3] += o[j].w;
          }
        }
#pragma unroll
        for (int j = 0; j < 8; ++j) d[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
      } else {
        if (g.bias) {
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            const float4 b = __ldg(reinterpret_cast<const float4 *>(g.bias + col0) + j);
            v[4 * j] += b.x;
            v[4 * j + 1] += b.y;
            v[4 * j + 2] += b.z;
            v[4 * j + 3] += b.w;
          }
        }
        uint4 *d = reinterpret_cast<uint4 *>((__nv_bfloat16 *)g.D + (size_t)row * g.ldd + col0);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          uint4 pk;
          uint32_t *pw = reinterpret_cast<uint32_t *>(&pk);
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            float lo = v[8 * q + 2 * i], hi = v[8 * q + 2 * i + 1];
            if (EPI == EPI_BIAS_RELU_BF16) {
              lo = fmaxf(lo, 0.f);
              hi = fmaxf(hi, 0.f);
            }
            const __nv_bfloat162 h2 = __floats2bfloat162_rn(lo, hi);
            pw[i] = *reinterpret_cast<const uint32_t *>(&h2);
          }
          d[q] = pk;
        }
      }
      continue;
    }
    if (row < g.M) {
#pragma unroll
      for (int i = 0; i < 32; ++i) {
        const int col = col0 + i;
        if (col >= g.N) continue;
        float y = v[i];
        if (EPI == EPI_STORE_F32) {
          ((float *)g.D)[(size_t)row * g.ldd + col] = y;
        } else if (EPI == EPI_BIAS_RELU_BF16 || EPI == EPI_BIAS_BF16) {
          y += g.bias ? g.bias[col] : 0.f;
          if (EPI == EPI_BIAS_RELU_BF16) y = fmaxf(y, 0.f);
          ((__nv_bfloat16 *)g.D)[(size_t)row * g.ldd + col] = __float2bfloat16(y);
        } else if (EPI == EPI_ADD_F32) {
          ((float *)g.D)[(size_t)row * g.ldd + col] += y;
        } else {
          atomicAdd((float *)g.D + (size_t)col * g.ldd + row, y);
        }
      }
    }
  }
}

void gemm_bf16(const GemmArgs &g, int bn, bool a_mn, bool b_mn, int epi, cudaStream_t s);
// Implicit-GEMM 3x3 convolution forward: D = act(conv(X) + bias), A gathered
// from g.convX, B = weights [N][ldb] K-major.
void conv3x3_bf16(const GemmArgs &g, int bn, int epi, cudaStream_t s);
// Implicit-GEMM weight gradient of a 3x3 convolution: gw[N][ldd] +=
// (col(X)^T[M][K] * dY[K][N])^T with M = padded 9*conv_C, K = pixels (split
// by ksplit), B = dY MN-major [pixels][ldb], A^T gathered from g.convX.
void conv3x3_wgrad_bf16(const GemmArgs &g, int bn, cudaStream_t s);

// TMA-fed variants (gemm_tma.cu) for K-major operands; the *_ok predicates
// say whether the operands' alignment and shape allow them.
bool gemm_tma_ok(const GemmArgs &g);
void gemm_bf16_tma(const GemmArgs &g, int bn, int epi, cudaStream_t s);
bool conv3x3_tma_ok(const GemmArgs &g);
void conv3x3_bf16_tma(const GemmArgs &g, int bn, int epi, cudaStream_t s);
bool conv3x3_wgrad_tma_ok(const GemmArgs &g);
void conv3x3_wgrad_bf16_tma(const GemmArgs &g, int bn, cudaStream_t s);
// Operand path: 0 = TMA where possible, 1 = always cp.async (a test switch).
extern int g_gemm_path;
// 3x3 convolution operand form on the TMA path: 0 = nine tap boxes per
// tile; 1 = halo strips where W % 128 == 0 (else tap boxes); 2 = row runs
// with resident weights where they fit (else halo strips, else tap boxes);
// 3 = row runs with the kernel rows stacked along N where BN is 32 or 64
// (else as 2).
extern int g_conv_halo;
// Row runs with 64-byte pixel rows: 1 = one strip per input row (the middle
// tap one pixel row into it), 0 = a second strip one pixel later.
extern int g_conv_one_strip;

}  // namespace airt
