// Bulk-async streamed segment SpMV (CSR rows or CSC columns).
//
// The nonzeros are cut (on the host, once per matrix) into tiles of whole
// segments holding at most kTileNnz nonzeros and kTileSeg segments.  Each
// persistent CTA owns a contiguous run of tiles and streams them through a
// kStages-deep ring of shared-memory stages with cp.async.bulk (global ->
// shared; the FP32 values, the int32 indices and the tile's int64 segment
// starts, completion counted on one mbarrier per stage).  Up to kStages-1
// tiles per CTA are in flight while one is consumed, so HBM streaming does
// not wait on the dependent gathers of the vector.
//
// The consumer is element-parallel (merge-path style): thread t takes the
// kElems contiguous nonzeros [e0 + kElems*t, ...) of the tile, issues all of
// their vector gathers at once, forms FP64 products, and the per-segment sums
// come from a block-wide segmented scan keyed by segment (fixed partition
// and fixed scan tree, so results are deterministic).  One thread per
// segment then runs the epilogue.  Utilisation is independent of segment
// lengths (rays of ~460 nonzeros and short rows alike).
//
// Bulk copies need 16-byte aligned global and shared addresses and sizes in
// multiples of 16 bytes: copied ranges are widened (4 index/value elements,
// 2 segment starts) and the arrays are padded (kPad elements, kPtrPad starts).
// Every mbarrier wait is bounded by a clock64 budget; on expiry the kernel
// records an error flag, drains its outstanding copies (again bounded) and
// returns.
#pragma once

#include <climits>

#include "common.cuh"

namespace airt {

constexpr int kStreamThreads = 256;
constexpr int kStreamCtasPerSm = 3;
constexpr int kElems = 8;                           // nonzeros per thread per tile
constexpr int kTileNnz = kStreamThreads * kElems;   // 2048
constexpr int kTileSeg = 256;                       // segments per tile (max)
constexpr int kStages = 3;
constexpr int kPad = 8;                             // padding elements after idx/val
constexpr int kPtrPad = 4;                          // padding entries after ptr
constexpr int kValCap = kTileNnz + 8;               // widened value/index copy
constexpr int kPtrCap = kTileSeg + 4;               // widened segment-start copy
constexpr size_t kStageBytes = (size_t)kValCap * 8 + (size_t)kPtrCap * 8;
constexpr long long kWaitBudget = 4000000000ll;     // ~2 s of SM clocks

__host__ __device__ constexpr size_t stream_smem_bytes() {
  return (size_t)kStages * kStageBytes + kStages * 8 + 128;
}

struct StreamArgs {
  int64_t nseg;
  const int64_t *ptr;
  const int *idx;
  const float *val;
  const float *gvec;
  const int *tile_seg;  // ntiles+1 segment starts of the tiles
  int ntiles;
  int *err;             // set to 1 on a wait timeout
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
      "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}

// Bounded wait for the phase with the given parity; false on timeout.
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

struct StageView {
  float *val;
  int *idx;
  int64_t *ptr;
};

__device__ __forceinline__ StageView stage_view(unsigned char *base, int s) {
  unsigned char *p = base + (size_t)s * kStageBytes;
  StageView v;
  v.val = (float *)p;
  v.idx = (int *)(p + (size_t)kValCap * 4);
  v.ptr = (int64_t *)(p + (size_t)kValCap * 8);
  return v;
}

// Issue the bulk copies of tile t into a stage (one thread).  Records the
// first copied element (ebase) and segment start index (pbase).
__device__ __forceinline__ void stream_issue(const StreamArgs &a, int t, const StageView &sv,
                                             uint32_t bar, int64_t *ebase, int64_t *pbase) {
  const int64_t seg0 = a.tile_seg[t], seg1 = a.tile_seg[t + 1];
  const int64_t e0 = a.ptr[seg0];
  const int64_t e1 = a.ptr[seg1];
  const int64_t a0 = e0 & ~(int64_t)3;
  const int64_t a1 = (e1 + 3) & ~(int64_t)3;
  const int64_t p0 = seg0 & ~(int64_t)1;
  const int64_t p1 = (seg1 + 2) & ~(int64_t)1;  // covers ptr[seg0 .. seg1]
  const uint32_t vb = (uint32_t)((a1 - a0) * 4);
  const uint32_t pb = (uint32_t)((p1 - p0) * 8);
  *ebase = a0;
  *pbase = p0;
  mbar_expect_tx(bar, 2 * vb + pb);
  if (vb) {
    bulk_g2s(smem_u32(sv.val), a.val + a0, vb, bar);
    bulk_g2s(smem_u32(sv.idx), a.idx + a0, vb, bar);
  }
  bulk_g2s(smem_u32(sv.ptr), a.ptr + p0, pb, bar);
}

// Inclusive segmented sum over the block for non-decreasing keys: on return
// val = sum of the vals of all threads t' <= t with key[t'] == key[t].
// s_wkey/s_wval end up holding each warp's inclusive total at its last lane.
__device__ __forceinline__ double block_segscan(int key, double val, int *s_wkey, double *s_wval) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int k2 = __shfl_up_sync(0xffffffffu, key, o);
    const double v2 = __shfl_up_sync(0xffffffffu, val, o);
    if (lane >= o && k2 == key) val += v2;
  }
  if (lane == 31) {
    s_wkey[w] = key;
    s_wval[w] = val;
  }
  __syncthreads();
  constexpr int W = kStreamThreads / 32;
  if (w == 0) {
    int k = lane < W ? s_wkey[lane] : INT_MAX - lane;
    double v = lane < W ? s_wval[lane] : 0.0;
#pragma unroll
    for (int o = 1; o < W; o <<= 1) {
      const int k2 = __shfl_up_sync(0xffffffffu, k, o);
      const double v2 = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o && k2 == k) v += v2;
    }
    if (lane < W) s_wval[lane] = v;
  }
  __syncthreads();
  if (w > 0 && key == s_wkey[w - 1]) val += s_wval[w - 1];
  return val;
}

// Epi: void(int64_t seg, double sum, bool lead)
template <class Epi>
__device__ __forceinline__ void stream_segments(const StreamArgs &a, Epi &&epi) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char *base = (unsigned char *)(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
  uint64_t *bars = (uint64_t *)(base + (size_t)kStages * kStageBytes);
  __shared__ int64_t s_ebase[kStages], s_pbase[kStages];
  __shared__ double s_row[kTileSeg];
  __shared__ int s_wkey[kStreamThreads / 32];
  __shared__ double s_wval[kStreamThreads / 32];
  __shared__ int s_abort, s_abort_t;

  const int G = gridDim.x;
  const int per = a.ntiles / G, rem = a.ntiles % G;
  const int t0 = blockIdx.x * per + min((int)blockIdx.x, rem);
  const int t1 = t0 + per + ((int)blockIdx.x < rem ? 1 : 0);
  const int tid = threadIdx.x;

  if (tid == 0) {
    s_abort = 0;
    for (int s = 0; s < kStages; ++s) mbar_init(smem_u32(&bars[s]), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    for (int k = 0; k < kStages && t0 + k < t1; ++k)
      stream_issue(a, t0 + k, stage_view(base, k), smem_u32(&bars[k]), &s_ebase[k], &s_pbase[k]);
  }
  __syncthreads();

  for (int t = t0; t < t1; ++t) {
    const int k = t - t0;
    const int s = k % kStages;
    if (!mbar_wait(smem_u32(&bars[s]), (uint32_t)((k / kStages) & 1))) {
      s_abort = 1;
      s_abort_t = t;
    }
    const int seg0 = a.tile_seg[t], seg1 = a.tile_seg[t + 1];
    const int nseg = seg1 - seg0;
    for (int i = tid; i < nseg; i += kStreamThreads) s_row[i] = 0.0;
    __syncthreads();
    if (s_abort) break;
    const StageView sv = stage_view(base, s);
    const int64_t eb = s_ebase[s], pbs = s_pbase[s];
    const int64_t *sp = sv.ptr + (seg0 - pbs);  // sp[j] = ptr[seg0 + j], j = 0..nseg
    const int64_t e0 = sp[0], e1 = sp[nseg];
    const int64_t q0 = e0 + (int64_t)kElems * tid;

    // products of this thread's nonzeros (all gathers issued together)
    double pv[kElems];
    int cnt = 0;
    if (q0 < e1) cnt = (int)min((int64_t)kElems, e1 - q0);
#pragma unroll
    for (int j = 0; j < kElems; ++j) {
      pv[j] = 0.0;
      if (j < cnt) {
        const int off = (int)(q0 + j - eb);
        pv[j] = (double)sv.val[off] * (double)__ldg(a.gvec + sv.idx[off]);
      }
    }
    // segment holding q0: the last j with sp[j] <= q0 (empty segments skipped)
    int cs = nseg;
    if (cnt > 0) {
      int lo = 0, hi = nseg;  // invariant: sp[lo] <= q0 < sp[hi]
      while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (sp[mid] <= q0) lo = mid;
        else hi = mid;
      }
      cs = lo;
    }
    // tail partial: the sum over this thread's nonzeros of its last segment
    int tail_seg = nseg;
    double tail = 0.0;
    if (cnt > 0) {
      int c = cs;
      int64_t nb = sp[c + 1];
#pragma unroll
      for (int j = 0; j < kElems; ++j) {
        if (j < cnt) {
          const int64_t q = q0 + j;
          while (q >= nb) {  // crossed into the next nonempty segment
            ++c;
            nb = sp[c + 1];
            tail = 0.0;
          }
          tail += pv[j];
        }
      }
      tail_seg = c;
    }
    const double incl = block_segscan(tail_seg, tail, s_wkey, s_wval);
    // carry into this thread's first segment from the threads before it
    const int lane = tid & 31, w = tid >> 5;
    int pkey = __shfl_up_sync(0xffffffffu, tail_seg, 1);
    double pval = __shfl_up_sync(0xffffffffu, incl, 1);
    if (lane == 0) {
      pkey = w > 0 ? s_wkey[w - 1] : -1;
      pval = w > 0 ? s_wval[w - 1] : 0.0;
    }
    if (cnt > 0) {
      double run = (tid > 0 && pkey == cs) ? pval : 0.0;
      int c = cs;
      int64_t nb = sp[c + 1];
#pragma unroll
      for (int j = 0; j < kElems; ++j) {
        if (j < cnt) {
          run += pv[j];
          const int64_t q = q0 + j;
          if (q + 1 == nb) {  // segment c ends here: complete sum
            s_row[c] = run;
            run = 0.0;
            ++c;
            while (c < nseg && sp[c + 1] == q + 1) ++c;  // empty segments
            nb = c < nseg ? sp[c + 1] : LLONG_MAX;
          }
        }
      }
    }
    __syncthreads();
    for (int i = tid; i < nseg; i += kStreamThreads) epi((int64_t)(seg0 + i), s_row[i], true);
    __syncthreads();  // stage s and s_row consumed
    if (tid == 0 && t + kStages < t1)
      stream_issue(a, t + kStages, sv, smem_u32(&bars[s]), &s_ebase[s], &s_pbase[s]);
  }
  if (s_abort) {
    if (tid == 0) {
      atomicExch(a.err, 1);
      // drain the copies still in flight (tiles abort_t .. abort_t+kStages-1)
      // before the CTA's shared memory goes away
      for (int t = s_abort_t; t < t1 && t < s_abort_t + kStages; ++t) {
        const int k = t - t0;
        (void)mbar_wait(smem_u32(&bars[k % kStages]), (uint32_t)((k / kStages) & 1));
      }
    }
    __syncthreads();
  }
}

// Host helper (sparse.cu): greedy tile table of a CSR/CSC; false when a
// segment does not fit a tile (the gather kernels are used instead).
bool build_tiles(Problem &P, const int64_t *d_ptr, int64_t nseg, DevBuf<int> &tiles, int &ntiles);

}  // namespace airt
