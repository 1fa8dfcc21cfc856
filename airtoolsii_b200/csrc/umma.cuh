// tcgen05 (5th-generation tensor core) GEMM for sm_100a, BF16 inputs, FP32
// accumulation in tensor memory.
//
//   D[M x N] (+)= A[M x K] * B[N x K]^T
//
// One CTA computes a 128 x BN tile with 128 threads (4 warps):
//  * all threads stage the A and B tiles of a 64-wide K slice from global
//    memory into shared memory in the canonical no-swizzle UMMA layout
//    (8 x 16-byte core matrices), zero-filling outside the matrix;
//  * one thread issues four tcgen05.mma.kind::f16 (K = 16 each) per slice,
//    and tcgen05.commit signals an mbarrier when they have read the stage;
//  * two stages alternate, so the next slice is staged while the tensor core
//    works on the current one;
//  * the accumulator lives in TMEM (128 lanes x BN FP32 columns); after the
//    last slice each warp reads its 32 lanes with tcgen05.ld and runs the
//    epilogue (store, bias + ReLU, or split-K atomic accumulation).
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
constexpr int kThreads = 128;
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
};

void gemm_bf16(const GemmArgs &g, int bn, bool a_mn, bool b_mn, int epi, cudaStream_t s);

}  // namespace airt
