// Row-segment SpMV building blocks shared by the operator and the solvers.
//
// A "segment" is a CSR row or a CSC column.  A group of LANES consecutive
// threads walks one segment with coalesced loads of the FP32 values and int32
// indices, gathers the (L2-resident) vector, accumulates in FP64 and reduces
// with warp shuffles.  The group width is chosen from the mean segment length.
#pragma once

#include "common.cuh"

namespace airt {

// Visit every segment with a LANES-wide group; the functor gets the segment
// index, the group's FP64 partial sum (already reduced: valid on lane 0 of
// the group) and whether this lane is the group leader.  All lanes of a warp
// run the same number of trips so that shuffles stay converged.
template <int LANES, typename TX, class Epi>
__device__ __forceinline__ void for_each_segment(int64_t nseg, const int64_t *__restrict__ ptr,
                                                 const int *__restrict__ idx,
                                                 const float *__restrict__ val,
                                                 const TX *__restrict__ x, Epi &&epi) {
  const int lane = threadIdx.x % LANES;
  const int64_t gid = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / LANES;
  const int64_t ng = (int64_t)gridDim.x * blockDim.x / LANES;
  const int64_t trips = (nseg + ng - 1) / ng;
  for (int64_t t = 0; t < trips; ++t) {
    const int64_t i = gid + t * ng;
    double acc = 0.0;
    if (i < nseg) {
      const int64_t q1 = ptr[i + 1];
      int64_t q = ptr[i] + lane;
      // two independent accumulators for memory-level parallelism
      double acc2 = 0.0;
      for (; q + LANES < q1; q += 2 * LANES) {
        const float v0 = __ldg(val + q), v1 = __ldg(val + q + LANES);
        const int c0 = __ldg(idx + q), c1 = __ldg(idx + q + LANES);
        acc = fma((double)v0, (double)__ldg(x + c0), acc);
        acc2 = fma((double)v1, (double)__ldg(x + c1), acc2);
      }
      if (q < q1) acc = fma((double)__ldg(val + q), (double)__ldg(x + __ldg(idx + q)), acc);
      acc += acc2;
    }
    acc = group_sum<LANES>(acc);
    epi(i, acc, lane == 0 && i < nseg);
  }
}

// Vectorised variant: the 4-aligned body of each segment is read with 16-byte
// loads (float4 values, int4 indices; the arrays are padded and 16-byte
// aligned), one vector per lane per round, and a warp carries 32/LANES
// segments at once so that many independent loads and gathers are in flight
// per SM (narrow groups measured best on B200: 8 lanes per ~460-entry ray).
// The unaligned head and tail (< 4 elements each) are read element-wise.
template <int LANES, typename TX, class Epi>
__device__ __forceinline__ void for_each_segment_v(int64_t nseg, const int64_t *__restrict__ ptr,
                                                   const int *__restrict__ idx,
                                                   const float *__restrict__ val,
                                                   const TX *__restrict__ x, Epi &&epi) {
  const int lane = threadIdx.x % LANES;
  const int64_t gid = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / LANES;
  const int64_t ng = (int64_t)gridDim.x * blockDim.x / LANES;
  const int64_t trips = (nseg + ng - 1) / ng;
  const float4 *__restrict__ V4 = reinterpret_cast<const float4 *>(val);
  const int4 *__restrict__ I4 = reinterpret_cast<const int4 *>(idx);
  for (int64_t t = 0; t < trips; ++t) {
    const int64_t i = gid + t * ng;
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    if (i < nseg) {
      const int64_t q0 = __ldg(ptr + i), q1 = __ldg(ptr + i + 1);
      int64_t qa = (q0 + 3) & ~(int64_t)3;
      if (qa > q1) qa = q1;
      int64_t qb = q1 & ~(int64_t)3;
      if (qb < qa) qb = qa;
      for (int64_t q = q0 + lane; q < qa; q += LANES)
        a0 = fma((double)__ldg(val + q), (double)__ldg(x + __ldg(idx + q)), a0);
      for (int64_t q = qb + lane; q < q1; q += LANES)
        a1 = fma((double)__ldg(val + q), (double)__ldg(x + __ldg(idx + q)), a1);
      const int64_t ve = qb >> 2;
      int64_t v = (qa >> 2) + lane;
      // two vectors per lane per round (both loads issued before the
      // gathers), accumulated in the order of the one-vector loop
      for (; v + LANES < ve; v += 2 * LANES) {
        const float4 f = __ldg(V4 + v), h = __ldg(V4 + v + LANES);
        const int4 c = __ldg(I4 + v), d = __ldg(I4 + v + LANES);
        const TX g0 = __ldg(x + c.x), g1 = __ldg(x + c.y), g2 = __ldg(x + c.z), g3 = __ldg(x + c.w);
        const TX k0 = __ldg(x + d.x), k1 = __ldg(x + d.y), k2 = __ldg(x + d.z), k3 = __ldg(x + d.w);
        a0 = fma((double)f.x, (double)g0, a0);
        a1 = fma((double)f.y, (double)g1, a1);
        a2 = fma((double)f.z, (double)g2, a2);
        a3 = fma((double)f.w, (double)g3, a3);
        a0 = fma((double)h.x, (double)k0, a0);
        a1 = fma((double)h.y, (double)k1, a1);
        a2 = fma((double)h.z, (double)k2, a2);
        a3 = fma((double)h.w, (double)k3, a3);
      }
      if (v < ve) {
        const float4 f = __ldg(V4 + v);
        const int4 c = __ldg(I4 + v);
        const TX g0 = __ldg(x + c.x), g1 = __ldg(x + c.y), g2 = __ldg(x + c.z), g3 = __ldg(x + c.w);
        a0 = fma((double)f.x, (double)g0, a0);
        a1 = fma((double)f.y, (double)g1, a1);
        a2 = fma((double)f.z, (double)g2, a2);
        a3 = fma((double)f.w, (double)g3, a3);
      }
    }
    double acc = (a0 + a1) + (a2 + a3);
    acc = group_sum<LANES>(acc);
    epi(i, acc, lane == 0 && i < nseg);
  }
}

// for_each_segment_v with a prefetch: the leader's pre(i) runs at the start
// of each trip, before the segment's loads, and its value reaches
// epi(i, sum, lead, pre_value), so per-segment operands of the epilogue are
// in flight together with the segment's own loads.
//
// Vectorised variant: the 4-aligned body of each segment is read with 16-byte
// loads (float4 values, int4 indices; the arrays are padded and 16-byte
// aligned), one vector per lane per round, and a warp carries 32/LANES
// segments at once so that many independent loads and gathers are in flight
// per SM (narrow groups measured best on B200: 8 lanes per ~460-entry ray).
// The unaligned head and tail (< 4 elements each) are read element-wise.
template <int LANES, typename TX, class Pre, class Epi>
__device__ __forceinline__ void for_each_segment_vpre(int64_t nseg, const int64_t *__restrict__ ptr,
                                                   const int *__restrict__ idx,
                                                   const float *__restrict__ val,
                                                   const TX *__restrict__ x, Pre &&pre, Epi &&epi) {
  const int lane = threadIdx.x % LANES;
  const int64_t gid = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / LANES;
  const int64_t ng = (int64_t)gridDim.x * blockDim.x / LANES;
  const int64_t trips = (nseg + ng - 1) / ng;
  const float4 *__restrict__ V4 = reinterpret_cast<const float4 *>(val);
  const int4 *__restrict__ I4 = reinterpret_cast<const int4 *>(idx);
  for (int64_t t = 0; t < trips; ++t) {
    const int64_t i = gid + t * ng;
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    decltype(pre(i)) pv{};
    if (i < nseg && lane == 0) pv = pre(i);
    if (i < nseg) {
      const int64_t q0 = __ldg(ptr + i), q1 = __ldg(ptr + i + 1);
      int64_t qa = (q0 + 3) & ~(int64_t)3;
      if (qa > q1) qa = q1;
      int64_t qb = q1 & ~(int64_t)3;
      if (qb < qa) qb = qa;
      for (int64_t q = q0 + lane; q < qa; q += LANES)
        a0 = fma((double)__ldg(val + q), (double)__ldg(x + __ldg(idx + q)), a0);
      for (int64_t q = qb + lane; q < q1; q += LANES)
        a1 = fma((double)__ldg(val + q), (double)__ldg(x + __ldg(idx + q)), a1);
      const int64_t ve = qb >> 2;
      int64_t v = (qa >> 2) + lane;
      // two vectors per lane per round (both loads issued before the
      // gathers), accumulated in the order of the one-vector loop
      for (; v + LANES < ve; v += 2 * LANES) {
        const float4 f = __ldg(V4 + v), h = __ldg(V4 + v + LANES);
        const int4 c = __ldg(I4 + v), d = __ldg(I4 + v + LANES);
        const TX g0 = __ldg(x + c.x), g1 = __ldg(x + c.y), g2 = __ldg(x + c.z), g3 = __ldg(x + c.w);
        const TX k0 = __ldg(x + d.x), k1 = __ldg(x + d.y), k2 = __ldg(x + d.z), k3 = __ldg(x + d.w);
        a0 = fma((double)f.x, (double)g0, a0);
        a1 = fma((double)f.y, (double)g1, a1);
        a2 = fma((double)f.z, (double)g2, a2);
        a3 = fma((double)f.w, (double)g3, a3);
        a0 = fma((double)h.x, (double)k0, a0);
        a1 = fma((double)h.y, (double)k1, a1);
        a2 = fma((double)h.z, (double)k2, a2);
        a3 = fma((double)h.w, (double)k3, a3);
      }
      if (v < ve) {
        const float4 f = __ldg(V4 + v);
        const int4 c = __ldg(I4 + v);
        const TX g0 = __ldg(x + c.x), g1 = __ldg(x + c.y), g2 = __ldg(x + c.z), g3 = __ldg(x + c.w);
        a0 = fma((double)f.x, (double)g0, a0);
        a1 = fma((double)f.y, (double)g1, a1);
        a2 = fma((double)f.z, (double)g2, a2);
        a3 = fma((double)f.w, (double)g3, a3);
      }
    }
    double acc = (a0 + a1) + (a2 + a3);
    acc = group_sum<LANES>(acc);
    epi(i, acc, lane == 0 && i < nseg, pv);
  }
}

// for_each_segment_v over a list of segment tiles, with a per-segment
// predicate.  Tile t covers segments t << tshift .. +(1 << tshift); the
// groups walk the *ntiles listed tiles (tiles[0 .. *ntiles)), so ranges left
// out of the list cost nothing, and segments for which active(i) is false
// are skipped without touching their nonzeros (all lanes of a group evaluate
// it, so the group stays converged).  The segment bounds are loaded
// together with the predicate's operands, not after them, and the leader's
// pre(i) (the epilogue's per-segment operands) is issued before the
// segment's loads; epi(i, sum, lead, pre_value) sees lead = false for
// skipped segments.
template <int LANES, typename TX, class Act, class Pre, class Epi>
__device__ __forceinline__ void for_each_segment_vt(int64_t nseg, const int *__restrict__ tiles,
                                                    const int *__restrict__ ntiles, int tshift,
                                                    const int64_t *__restrict__ ptr,
                                                    const int *__restrict__ idx,
                                                    const float *__restrict__ val,
                                                    const TX *__restrict__ x, Act &&active,
                                                    Pre &&pre, Epi &&epi) {
  const int lane = threadIdx.x % LANES;
  const int64_t gid = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / LANES;
  const int64_t ng = (int64_t)gridDim.x * blockDim.x / LANES;
  const int64_t total = (int64_t)__ldg(ntiles) << tshift;
  const int64_t tmask = ((int64_t)1 << tshift) - 1;
  const int64_t trips = (total + ng - 1) / ng;
  const float4 *__restrict__ V4 = reinterpret_cast<const float4 *>(val);
  const int4 *__restrict__ I4 = reinterpret_cast<const int4 *>(idx);
  for (int64_t t = 0; t < trips; ++t) {
    const int64_t u = gid + t * ng;
    const int64_t i = u < total ? ((int64_t)__ldg(tiles + (u >> tshift)) << tshift) + (u & tmask) : nseg;
    bool on = false;
    int64_t q0 = 0, q1 = 0;
    decltype(pre(i)) pv{};
    if (i < nseg) {
      q0 = __ldg(ptr + i);
      q1 = __ldg(ptr + i + 1);
      on = active(i);
      if (on && lane == 0) pv = pre(i);
    }
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    if (on) {
      // every aligned 16-byte group that overlaps [q0, q1), its elements
      // outside the segment masked out (they belong to the neighbouring
      // segments or the zero padding, so the loads stay inside the arrays):
      // no element-wise head or tail loop, which on short segments (tens of
      // nonzeros) would hold a large share of the loads in serial chains
      const int64_t ve = (q1 + 3) >> 2;
      int64_t v = (q0 >> 2) + lane;
      for (; v + LANES < ve; v += 2 * LANES) {
        const float4 f = __ldg(V4 + v), h = __ldg(V4 + v + LANES);
        const int4 c = __ldg(I4 + v), d = __ldg(I4 + v + LANES);
        const TX g0 = __ldg(x + c.x), g1 = __ldg(x + c.y), g2 = __ldg(x + c.z), g3 = __ldg(x + c.w);
        const TX k0 = __ldg(x + d.x), k1 = __ldg(x + d.y), k2 = __ldg(x + d.z), k3 = __ldg(x + d.w);
        const int64_t e = v << 2, e2 = (v + LANES) << 2;
        if (e >= q0 && e < q1) a0 = fma((double)f.x, (double)g0, a0);
        if (e + 1 >= q0 && e + 1 < q1) a1 = fma((double)f.y, (double)g1, a1);
        if (e + 2 >= q0 && e + 2 < q1) a2 = fma((double)f.z, (double)g2, a2);
        if (e + 3 >= q0 && e + 3 < q1) a3 = fma((double)f.w, (double)g3, a3);
        if (e2 < q1) a0 = fma((double)h.x, (double)k0, a0);
        if (e2 + 1 < q1) a1 = fma((double)h.y, (double)k1, a1);
        if (e2 + 2 < q1) a2 = fma((double)h.z, (double)k2, a2);
        if (e2 + 3 < q1) a3 = fma((double)h.w, (double)k3, a3);
      }
      if (v < ve) {
        const float4 f = __ldg(V4 + v);
        const int4 c = __ldg(I4 + v);
        const TX g0 = __ldg(x + c.x), g1 = __ldg(x + c.y), g2 = __ldg(x + c.z), g3 = __ldg(x + c.w);
        const int64_t e = v << 2;
        if (e >= q0 && e < q1) a0 = fma((double)f.x, (double)g0, a0);
        if (e + 1 >= q0 && e + 1 < q1) a1 = fma((double)f.y, (double)g1, a1);
        if (e + 2 >= q0 && e + 2 < q1) a2 = fma((double)f.z, (double)g2, a2);
        if (e + 3 >= q0 && e + 3 < q1) a3 = fma((double)f.w, (double)g3, a3);
      }
    }
    double acc = (a0 + a1) + (a2 + a3);
    acc = group_sum<LANES>(acc);
    epi(i, acc, lane == 0 && on, pv);
  }
}

// for_each_segment_vt over a block-diagonal matrix whose indices are stored
// as 16-bit offsets within each segment's instance: segment i belongs to
// instance inst_of[i], runs when stop[that] == 0, and gathers x[voff[that] +
// local index].  A lane reads 8 nonzeros per 16-byte index load (two float4
// value loads), two such groups per round, so the streamed bytes per
// nonzero drop from 8 to 6.  The 8-aligned body is vectorised, the head and
// tail (< 8 elements each) are read element-wise; segment sums run in a
// fixed order (per lane four accumulators, then the group's shuffle tree).
template <int LANES, typename TX, class Pre, class Epi>
__device__ __forceinline__ void for_each_segment_vt16(int64_t nseg, const int *__restrict__ tiles,
                                                      const int *__restrict__ ntiles, int tshift,
                                                      const int64_t *__restrict__ ptr,
                                                      const uint16_t *__restrict__ idx,
                                                      const float *__restrict__ val,
                                                      const TX *__restrict__ x,
                                                      const int *__restrict__ inst_of,
                                                      const int *__restrict__ stop,
                                                      const int64_t *__restrict__ voff, Pre &&pre,
                                                      Epi &&epi) {
  const int lane = threadIdx.x % LANES;
  const int64_t gid = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / LANES;
  const int64_t ng = (int64_t)gridDim.x * blockDim.x / LANES;
  const int64_t total = (int64_t)__ldg(ntiles) << tshift;
  const int64_t tmask = ((int64_t)1 << tshift) - 1;
  const int64_t trips = (total + ng - 1) / ng;
  const float4 *__restrict__ V4 = reinterpret_cast<const float4 *>(val);
  const uint4 *__restrict__ I8 = reinterpret_cast<const uint4 *>(idx);
  for (int64_t t = 0; t < trips; ++t) {
    const int64_t u = gid + t * ng;
    const int64_t i = u < total ? ((int64_t)__ldg(tiles + (u >> tshift)) << tshift) + (u & tmask) : nseg;
    bool on = false;
    int64_t q0 = 0, q1 = 0;
    const TX *xb = x;
    decltype(pre(i)) pv{};
    if (i < nseg) {
      q0 = __ldg(ptr + i);
      q1 = __ldg(ptr + i + 1);
      const int k = __ldg(inst_of + i);
      on = __ldg(stop + k) == 0;
      xb = x + __ldg(voff + k);
      if (on && lane == 0) pv = pre(i);
    }
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    if (on) {
      int64_t qa = (q0 + 7) & ~(int64_t)7;
      if (qa > q1) qa = q1;
      int64_t qb = q1 & ~(int64_t)7;
      if (qb < qa) qb = qa;
      for (int64_t q = q0 + lane; q < qa; q += LANES)
        a0 = fma((double)__ldg(val + q), (double)__ldg(xb + __ldg(idx + q)), a0);
      for (int64_t q = qb + lane; q < q1; q += LANES)
        a1 = fma((double)__ldg(val + q), (double)__ldg(xb + __ldg(idx + q)), a1);
      const int64_t ge = qb >> 3;
      int64_t gq = (qa >> 3) + lane;
      for (; gq < ge; gq += LANES) {
        const uint4 c = __ldg(I8 + gq);
        const float4 f = __ldg(V4 + 2 * gq), h = __ldg(V4 + 2 * gq + 1);
        const TX g0 = __ldg(xb + (c.x & 0xFFFFu)), g1 = __ldg(xb + (c.x >> 16));
        const TX g2 = __ldg(xb + (c.y & 0xFFFFu)), g3 = __ldg(xb + (c.y >> 16));
        const TX g4 = __ldg(xb + (c.z & 0xFFFFu)), g5 = __ldg(xb + (c.z >> 16));
        const TX g6 = __ldg(xb + (c.w & 0xFFFFu)), g7 = __ldg(xb + (c.w >> 16));
        a0 = fma((double)f.x, (double)g0, a0);
        a1 = fma((double)f.y, (double)g1, a1);
        a2 = fma((double)f.z, (double)g2, a2);
        a3 = fma((double)f.w, (double)g3, a3);
        a0 = fma((double)h.x, (double)g4, a0);
        a1 = fma((double)h.y, (double)g5, a1);
        a2 = fma((double)h.z, (double)g6, a2);
        a3 = fma((double)h.w, (double)g7, a3);
      }
    }
    double acc = (a0 + a1) + (a2 + a3);
    acc = group_sum<LANES>(acc);
    epi(i, acc, lane == 0 && on, pv);
  }
}

// Lanes per segment of the vectorised kernels from the mean segment length.
inline int vec_lanes_for(int64_t nnz, int64_t nseg) {
  const double avg = nseg ? (double)nnz / (double)nseg : 0.0;
  if (avg > 128) return 8;
  if (avg > 16) return 4;
  return 2;
}

template <int LANES>
__global__ void __launch_bounds__(256, 4) k_spmv_plain(int64_t nseg, const int64_t *__restrict__ ptr,
                                                       const int *__restrict__ idx,
                                                       const float *__restrict__ val,
                                                       const double *__restrict__ x,
                                                       double *__restrict__ y) {
  for_each_segment_v<LANES>(nseg, ptr, idx, val, x, [&](int64_t i, double s, bool lead) {
    if (lead) y[i] = s;
  });
}

inline int lanes_for(int64_t nnz, int64_t nseg) {
  const double avg = nseg ? (double)nnz / (double)nseg : 0.0;
  if (avg >= 48) return 32;
  if (avg >= 20) return 16;
  if (avg >= 8) return 8;
  return 4;
}

inline void spmv_plain(int64_t nseg, const int64_t *ptr, const int *idx, const float *val,
                       const double *x, double *y, cudaStream_t s) {
  if (nseg == 0) return;
  int64_t nnz = 0;
  AIRT_CHECK_CUDA(cudaMemcpyAsync(&nnz, ptr + nseg, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  AIRT_CHECK_CUDA(cudaStreamSynchronize(s));
  const int L = vec_lanes_for(nnz, nseg);
  const unsigned g = grid_for(nseg * L, 256, 4);
  switch (L) {
    case 8: k_spmv_plain<8><<<g, 256, 0, s>>>(nseg, ptr, idx, val, x, y); break;
    case 4: k_spmv_plain<4><<<g, 256, 0, s>>>(nseg, ptr, idx, val, x, y); break;
    default: k_spmv_plain<2><<<g, 256, 0, s>>>(nseg, ptr, idx, val, x, y); break;
  }
  AIRT_LAUNCH_CHECK();
}

void apply_matrix_free(Problem &P, const double *d_in, double *d_out, int transp);

}  // namespace airt
