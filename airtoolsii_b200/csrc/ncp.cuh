// Normalized cumulative periodogram stopping rule (auxil/check_stoprules.m:
// 97-150) on the device: periodograms of the residual's columns and each
// column's distance to the white-noise cumulative line.  Shared by the SIRT
// loop (decision in its control kernel) and ART (decision on the host).
#pragma once

#include <cmath>
#include <vector>

#include "common.cuh"

namespace airt {
namespace {  // internal linkage: included by more than one translation unit

// NCP (check_stoprules.m:97-150), part 1: periodogram of every residual
// column.  Block row j = column j of the residual reshaped to L x ncols
// (column-major), thread -> frequency f = 1..q (q = floor(L/2)); |sum_n
// r[n] exp(-2 pi i f n / L)|^2 by direct summation with a twiddle table
// (tw[2k], tw[2k+1] = cos, sin of 2 pi k / L).  The residual of the ME
// variant of the forward kernel (rprev holds r after it), or of ART.
__global__ void __launch_bounds__(256) k_ncp_power(int L, int q, const double *__restrict__ r,
                                                   const double *__restrict__ tw, double *__restrict__ pk,
                                                   const int *stop_flag) {
  if (stop_flag && *(volatile const int *)stop_flag) return;
  const int j = blockIdx.x;
  const int f = blockIdx.y * blockDim.x + threadIdx.x + 1;
  if (f > q) return;
  const double *rc = r + (int64_t)j * L;
  double re = 0.0, im = 0.0;
  int idx = 0;  // (f * n) mod L
  for (int n = 0; n < L; ++n) {
    const double v = __ldg(rc + n);
    re = fma(v, __ldg(tw + 2 * idx), re);
    im = fma(v, __ldg(tw + 2 * idx + 1), im);
    idx += f;
    if (idx >= L) idx -= L;
  }
  pk[(int64_t)j * q + (f - 1)] = re * re + im * im;
}

// NCP part 2 for one column (the calling block): c = cumsum(pk)/sum(pk) of
// the q periodogram values p[0..q) and the distance
// sqrt(sum((c - (1:q)/q).^2)) to the white-noise line, returned on thread 0.
// 256 threads own contiguous chunks of the q values; chunk sums meet in a
// block scan.
__device__ __forceinline__ double ncp_distance(int q, const double *__restrict__ p) {
  __shared__ double sh[256];
  __shared__ double tot_sh;
  const int t = threadIdx.x;
  const int per = (q + 255) / 256, f0 = min(q, t * per), f1 = min(q, f0 + per);
  double loc = 0.0;
  for (int f = f0; f < f1; ++f) loc += p[f];
  sh[t] = loc;
  __syncthreads();
  if (t == 0) {  // exclusive prefix of the chunk sums; the total
    double run = 0.0;
    for (int i = 0; i < 256; ++i) {
      const double v = sh[i];
      sh[i] = run;
      run += v;
    }
    tot_sh = run;
  }
  __syncthreads();
  const double tot = tot_sh;
  double c = sh[t], acc = 0.0;
  for (int f = f0; f < f1; ++f) {
    c += p[f];
    const double d = c / tot - (double)(f + 1) / (double)q;
    acc += d * d;
  }
  acc = block_sum<256>(acc);
  return sqrt(acc);
}

// NCP part 2: the distance of every column (block j = column j).
__global__ void __launch_bounds__(256) k_ncp_col(int q, const double *__restrict__ pk,
                                                 double *__restrict__ ncc_col, const int *stop_flag) {
  if (stop_flag && *(volatile const int *)stop_flag) return;
  const int j = blockIdx.x;
  const double d = ncp_distance(q, pk + (int64_t)j * q);
  if (threadIdx.x == 0) ncc_col[j] = d;
}

}  // namespace

// cos, sin of 2 pi k / L, k = 0..L-1, interleaved.
inline std::vector<double> ncp_twiddles(int L) {
  std::vector<double> tw(2 * (size_t)L);
  const double two_pi = 6.283185307179586476925286766559;
  for (int k = 0; k < L; ++k) {
    tw[2 * k] = std::cos(two_pi * k / L);
    tw[2 * k + 1] = std::sin(two_pi * k / L);
  }
  return tw;
}

}  // namespace airt
