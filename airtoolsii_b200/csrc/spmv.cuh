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

template <int LANES>
__global__ void __launch_bounds__(256) k_spmv_plain(int64_t nseg, const int64_t *__restrict__ ptr,
                                                    const int *__restrict__ idx,
                                                    const float *__restrict__ val,
                                                    const double *__restrict__ x,
                                                    double *__restrict__ y) {
  for_each_segment<LANES>(nseg, ptr, idx, val, x, [&](int64_t i, double s, bool lead) {
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
  const int L = lanes_for(nnz, nseg);
  const unsigned g = grid_for(nseg * L, 256);
  switch (L) {
    case 32: k_spmv_plain<32><<<g, 256, 0, s>>>(nseg, ptr, idx, val, x, y); break;
    case 16: k_spmv_plain<16><<<g, 256, 0, s>>>(nseg, ptr, idx, val, x, y); break;
    case 8: k_spmv_plain<8><<<g, 256, 0, s>>>(nseg, ptr, idx, val, x, y); break;
    default: k_spmv_plain<4><<<g, 256, 0, s>>>(nseg, ptr, idx, val, x, y); break;
  }
  AIRT_LAUNCH_CHECK();
}

void apply_matrix_free(Problem &P, const double *d_in, double *d_out, int transp);

}  // namespace airt
