// Filtered back projection (auxil/fbp.m:40-79) on the GPU.
//
// fbp.m zero-pads every projection (one column of the nr x na sinogram) to
// `order` samples, multiplies its FFT by a real even filter, and keeps the
// first nr samples of the inverse FFT: a circular convolution of the padded
// column with h = real(ifft(filter)).  The host supplies h (order entries,
// FP64); here every output sample is the direct FP64 sum
// sum_j h[(i - j) mod order] * b[j] over the nr input samples, one CTA per
// column with the column and the 2*nr - 1 kernel taps it needs in shared
// memory.  The filtered sinogram, scaled by pi/(2*na), is back-projected
// with the problem's (or batch's) transpose operator.
#include <algorithm>

#include "common.cuh"

namespace airt {

namespace {

__global__ void __launch_bounds__(256)
    k_fbp_filter(const double *__restrict__ in, double *__restrict__ out, int nr, int64_t ncols,
                 const double *__restrict__ h, int order, const double *__restrict__ col_scale,
                 double scale) {
  extern __shared__ double sm[];
  double *col = sm;        // nr samples of the current column
  double *taps = sm + nr;  // taps[d + nr - 1] = h[d mod order], -nr < d < nr
  for (int d = threadIdx.x; d < 2 * nr - 1; d += blockDim.x) {
    const int dd = d - (nr - 1);
    taps[d] = h[dd >= 0 ? dd : dd + order];
  }
  for (int64_t c = blockIdx.x; c < ncols; c += gridDim.x) {
    __syncthreads();
    for (int j = threadIdx.x; j < nr; j += blockDim.x) col[j] = in[c * nr + j];
    __syncthreads();
    const double sc = col_scale ? col_scale[c] : scale;
    for (int i = threadIdx.x; i < nr; i += blockDim.x) {
      const double *t = taps + i + nr - 1;  // t[-j] = h[(i - j) mod order]
      double acc = 0.0;
      for (int j = 0; j < nr; ++j) acc = fma(t[-j], col[j], acc);
      out[c * nr + i] = acc * sc;
    }
  }
}

}  // namespace

void fbp_filter(const double *d_in, double *d_out, int nr, int64_t ncols, const double *d_h,
                int order, const double *d_col_scale, double scale, cudaStream_t s) {
  AIRT_REQUIRE(nr >= 1 && order >= 2 * nr - 1, "fbp: order must be at least 2*nr - 1");
  const size_t smem = (size_t)(3 * nr - 1) * sizeof(double);
  AIRT_REQUIRE(smem <= 200 * 1024, "fbp: projections too long for the shared-memory filter");
  if (smem > 48 * 1024)
    AIRT_CHECK_CUDA(cudaFuncSetAttribute(k_fbp_filter, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem));
  if (ncols == 0) return;
  const unsigned grid = (unsigned)std::min<int64_t>(ncols, (int64_t)num_sms() * 8);
  k_fbp_filter<<<grid, 256, smem, s>>>(d_in, d_out, nr, ncols, d_h, order, d_col_scale, scale);
  AIRT_LAUNCH_CHECK();
}

}  // namespace airt
