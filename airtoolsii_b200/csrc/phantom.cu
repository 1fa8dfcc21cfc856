// Batched random-ellipse phantoms on the GPU (training data of the learned
// warm start).  Same grid convention as the phantom gallery's ellipse
// rasterisation (testprobs/phantomgallery.m:188-214): xn = ((0:N-1) -
// (N-1)/2) / ((N-1)/2), X along columns, Y = rot90(X) along rows; an
// ellipse (amplitude, a, b, x0, y0, phi) adds its amplitude where
// ((x cos + y sin)^2 / a^2 + (y cos - x sin)^2 / b^2) <= 1; the sum is
// clipped to [lo, hi].  Images are written as x(:) (column-major).
#include "common.cuh"

namespace airt {
namespace {

// params: per image `nell` records of 7 doubles (amp, a, b, x0, y0, cos phi, sin phi)
__global__ void k_ellipses(int N, int nimg, int nell, const double *__restrict__ prm, double lo,
                           double hi, double *__restrict__ out) {
  const int64_t total = (int64_t)nimg * N * N;
  const double c = (N - 1) / 2.0;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t img = t / ((int64_t)N * N);
    const int64_t pix = t - img * N * N;
    const int j = (int)(pix / N), i = (int)(pix % N);  // column-major: pix = j*N + i
    const double X = ((double)j - c) / c;
    const double Y = ((double)(N - 1 - i) - c) / c;
    double v = 0.0;
    const double *pp = prm + img * nell * 7;
    for (int e = 0; e < nell; ++e) {
      const double amp = pp[7 * e], ea = pp[7 * e + 1], eb = pp[7 * e + 2];
      const double x = X - pp[7 * e + 3], y = Y - pp[7 * e + 4];
      const double cs = pp[7 * e + 5], sn = pp[7 * e + 6];
      const double u = __dadd_rn(__dmul_rn(x, cs), __dmul_rn(y, sn));
      const double w = __dsub_rn(__dmul_rn(y, cs), __dmul_rn(x, sn));
      const double q = __dadd_rn(__ddiv_rn(__dmul_rn(u, u), __dmul_rn(ea, ea)),
                                 __ddiv_rn(__dmul_rn(w, w), __dmul_rn(eb, eb)));
      if (q <= 1.0) v += amp;
    }
    v = v < lo ? lo : v;
    v = v > hi ? hi : v;
    out[t] = v;
  }
}

}  // namespace
}  // namespace airt

using namespace airt;

extern "C" int airt_phantom_ellipses(int N, int nimg, int nell, const double *params, double lo,
                                     double hi, double *d_out, void *cuda_stream) {
  try {
    AIRT_REQUIRE(N >= 2 && nimg >= 0 && nell >= 0 && params && d_out, "invalid argument");
    cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
    DevBuf<double> prm;
    prm.upload(params, (size_t)nimg * nell * 7, s);
    const int64_t total = (int64_t)nimg * N * N;
    k_ellipses<<<grid_for(total > 0 ? total : 1, 256), 256, 0, s>>>(N, nimg, nell, prm.p, lo, hi, d_out);
    AIRT_LAUNCH_CHECK();
    AIRT_CHECK_CUDA(cudaStreamSynchronize(s));
  } catch (const Status &st) {
    return st.code;
  }
  return AIRT_OK;
}
