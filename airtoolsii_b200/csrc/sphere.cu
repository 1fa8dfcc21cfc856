// sphericaltomo on the GPU: the system matrix (testprobs/sphericaltomo.m:
// 108-270, isMatrix = 1) and the exact row/column statistics its matrix-free
// operator needs for the SIRT weights.
//
// Row i*p + n samples circle n about the point at angle i at nPhi(n) + 1
// angles; each sample inside the image hits one pixel J; the row holds
// (unique(J), 2*pi*r/nPhi * histc(J, unique(J))).  On the device every sample
// becomes a 64-bit key (row in the high word, J in the low word; samples
// outside the image get a key above every row), one radix sort per chunk of
// angles orders the keys by (row, J), and a run-length encoding gives each
// distinct (row, J) with its hit count w -- MATLAB's unique/histc pair.  The
// chunks run in row order, so their runs concatenate into the CSR directly.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_run_length_encode.cuh>

#include <vector>

#include "common.cuh"
#include "stream.cuh"
#include "trace.cuh"

namespace airt {

namespace {

// One CTA per row of the chunk [row0, row0 + rows); row0 is a multiple of p,
// so local row rl belongs to local angle rl / p and its samples start at
// (rl / p) * S + koff[n].
__global__ void k_sph_keys(RayGeom g, int64_t row0, int rows, int64_t S,
                           unsigned long long *__restrict__ keys) {
  const unsigned long long outside = (unsigned long long)rows << 32;
  for (int rl = blockIdx.x; rl < rows; rl += gridDim.x) {
    const int64_t r = row0 + rl;
    const int i = (int)(r / g.p);
    const int n = (int)(r - (int64_t)i * g.p);
    const double xix = g.cos_t[i], xiy = g.sin_t[i], rad = g.radius[n];
    const int64_t k0 = g.koff[n], k1 = g.koff[n + 1];
    unsigned long long *out = keys + (int64_t)(rl / g.p) * S + k0;
    for (int64_t k = k0 + threadIdx.x; k < k1; k += blockDim.x) {
      const int J = sphere_pixel(g, xix, xiy, rad, k);
      out[k - k0] = J >= 0 ? (((unsigned long long)rl << 32) | (unsigned)J) : outside;
    }
  }
}

__global__ void k_sph_count(const unsigned long long *__restrict__ uk, int64_t nruns, int64_t row0,
                            unsigned long long *__restrict__ counts) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nruns;
       e += (int64_t)gridDim.x * blockDim.x)
    atomicAdd(counts + row0 + (int64_t)(uk[e] >> 32), 1ull);
}

// Entry value: (2*pi*radii(n)/nPhi(n)) * w, sphericaltomo.m:234.
__device__ __forceinline__ double sph_value(const RayGeom &g, int64_t r, int w) {
  const int n = (int)(r % g.p);
  return __dmul_rn(g.cscale[n], (double)w);
}

__global__ void k_sph_fill(RayGeom g, const unsigned long long *__restrict__ uk,
                           const int *__restrict__ cnt, int64_t nruns, int64_t row0,
                           int64_t base, int *__restrict__ ci, float *__restrict__ rv) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nruns;
       e += (int64_t)gridDim.x * blockDim.x) {
    const unsigned long long key = uk[e];
    const int64_t r = row0 + (int64_t)(key >> 32);
    ci[base + e] = (int)(key & 0xffffffffull);
    rv[base + e] = (float)sph_value(g, r, cnt[e]);
  }
}

// Row sums of v^2, |v| and v^2*colw[J]; per-column counts and |v| sums, with
// v the FP32-rounded entry, as k_mf_stats gives them for a straight ray.
__global__ void k_sph_stats(RayGeom g, const unsigned long long *__restrict__ uk,
                            const int *__restrict__ cnt, int64_t nruns, int64_t row0,
                            double *__restrict__ s2, double *__restrict__ s1,
                            double *__restrict__ ccnt, double *__restrict__ cs1,
                            const double *__restrict__ colw, double *__restrict__ s2w) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nruns;
       e += (int64_t)gridDim.x * blockDim.x) {
    const unsigned long long key = uk[e];
    const int64_t r = row0 + (int64_t)(key >> 32);
    const int J = (int)(key & 0xffffffffull);
    const double v = (double)(float)sph_value(g, r, cnt[e]);
    if (s2) atomicAdd(s2 + r, v * v);
    if (s1) atomicAdd(s1 + r, fabs(v));
    if (s2w) atomicAdd(s2w + r, v * v * colw[J]);
    if (ccnt) atomicAdd(ccnt + J, 1.0);
    if (cs1) atomicAdd(cs1 + J, fabs(v));
  }
}

int bit_width(uint64_t v) {
  int b = 0;
  while (v) {
    ++b;
    v >>= 1;
  }
  return b;
}

// Samples per chunk: the keys, their sorted copy and the runs take about
// 28 bytes per sample, so 2^27 samples hold a chunk under 4 GB.
constexpr int64_t kChunkSamples = int64_t(1) << 27;

// Runs the key/sort/encode pipeline over whole angles and hands every
// chunk's distinct (row, J) keys and counts to fn(uk, cnt, nruns, row0).
template <class Fn>
void for_each_sphere_chunk(Problem &P, Fn &&fn) {
  cudaStream_t s = P.stream;
  const RayGeom g = P.geom();
  const int64_t S = P.koff_total;
  if (P.m == 0 || S == 0) return;
  AIRT_REQUIRE(S < INT32_MAX, "too many samples per angle");
  const int64_t per = std::max<int64_t>(1, std::min<int64_t>(P.nA, kChunkSamples / S));
  const int64_t cap = per * S;
  DevBuf<unsigned long long> keys, sorted, uk;
  DevBuf<int> cnt, nruns;
  keys.ensure(cap);
  sorted.ensure(cap);
  uk.ensure(cap);
  cnt.ensure(cap);
  nruns.ensure(1);
  DevBuf<unsigned char> tmp;
  for (int64_t a0 = 0; a0 < P.nA; a0 += per) {
    const int64_t na = std::min<int64_t>(per, P.nA - a0);
    const int rows = (int)(na * P.p);
    const int items = (int)(na * S);
    const int64_t row0 = a0 * P.p;
    k_sph_keys<<<std::min(rows, 148 * 16), 256, 0, s>>>(g, row0, rows, S, keys.p);
    AIRT_LAUNCH_CHECK();
    const int end_bit = 32 + bit_width((uint64_t)rows);
    size_t b1 = 0, b2 = 0;
    AIRT_CHECK_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, b1, keys.p, sorted.p, items, 0, end_bit, s));
    AIRT_CHECK_CUDA(cub::DeviceRunLengthEncode::Encode(nullptr, b2, sorted.p, uk.p, cnt.p, nruns.p,
                                                       items, s));
    tmp.ensure(std::max(b1, b2));
    AIRT_CHECK_CUDA(cub::DeviceRadixSort::SortKeys(tmp.p, b1, keys.p, sorted.p, items, 0, end_bit, s));
    AIRT_CHECK_CUDA(cub::DeviceRunLengthEncode::Encode(tmp.p, b2, sorted.p, uk.p, cnt.p, nruns.p,
                                                       items, s));
    int hn = 0;
    AIRT_CHECK_CUDA(cudaMemcpyAsync(&hn, nruns.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    AIRT_CHECK_CUDA(cudaStreamSynchronize(s));
    unsigned long long last = 0;
    if (hn > 0) {
      AIRT_CHECK_CUDA(cudaMemcpyAsync(&last, uk.p + hn - 1, sizeof(last), cudaMemcpyDeviceToHost, s));
      AIRT_CHECK_CUDA(cudaStreamSynchronize(s));
    }
    const int64_t valid = (hn > 0 && (last >> 32) == (unsigned long long)rows) ? hn - 1 : hn;
    fn(uk.p, cnt.p, valid, row0);
  }
}

}  // namespace

void generate_sphere_matrix(Problem &P) {
  cudaStream_t s = P.stream;
  const RayGeom g = P.geom();
  DevBuf<unsigned long long> counts;
  counts.ensure(P.m);
  AIRT_CHECK_CUDA(cudaMemsetAsync(counts.p, 0, P.m * sizeof(unsigned long long), s));
  // runs of every chunk, kept until the CSR is allocated
  std::vector<DevBuf<unsigned long long>> ukeep;
  std::vector<DevBuf<int>> ckeep;
  std::vector<std::pair<int64_t, int64_t>> span;  // (runs, row0)
  for_each_sphere_chunk(P, [&](const unsigned long long *uk, const int *cnt, int64_t n,
                               int64_t row0) {
    ukeep.emplace_back();
    ckeep.emplace_back();
    ukeep.back().ensure(std::max<int64_t>(n, 1));
    ckeep.back().ensure(std::max<int64_t>(n, 1));
    if (n) {
      AIRT_CHECK_CUDA(cudaMemcpyAsync(ukeep.back().p, uk, n * sizeof(*uk), cudaMemcpyDeviceToDevice, s));
      AIRT_CHECK_CUDA(cudaMemcpyAsync(ckeep.back().p, cnt, n * sizeof(*cnt), cudaMemcpyDeviceToDevice, s));
      k_sph_count<<<grid_for(n, 256, 4), 256, 0, s>>>(uk, n, row0, counts.p);
      AIRT_LAUNCH_CHECK();
    }
    span.emplace_back(n, row0);
  });
  P.rp.ensure(P.m + 1 + kPtrPad);
  AIRT_CHECK_CUDA(cudaMemsetAsync(P.rp.p + P.m + 1, 0, kPtrPad * sizeof(int64_t), s));
  exclusive_scan_i64(reinterpret_cast<const int64_t *>(counts.p), P.rp.p, P.m, s);
  AIRT_CHECK_CUDA(cudaMemcpyAsync(&P.nnz, P.rp.p + P.m, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  AIRT_CHECK_CUDA(cudaStreamSynchronize(s));
  P.ci.ensure(P.nnz + kPad);
  P.rv.ensure(P.nnz + kPad);
  AIRT_CHECK_CUDA(cudaMemsetAsync(P.ci.p + P.nnz, 0, kPad * sizeof(int), s));
  AIRT_CHECK_CUDA(cudaMemsetAsync(P.rv.p + P.nnz, 0, kPad * sizeof(float), s));
  int64_t base = 0;
  for (size_t c = 0; c < span.size(); ++c) {
    const int64_t n = span[c].first;
    if (n) {
      k_sph_fill<<<grid_for(n, 256, 4), 256, 0, s>>>(g, ukeep[c].p, ckeep[c].p, n, span[c].second,
                                                     base, P.ci.p, P.rv.p);
      AIRT_LAUNCH_CHECK();
    }
    base += n;
  }
  AIRT_REQUIRE(base == P.nnz, "sphere matrix: run count mismatch");
  build_csc_from_csr(P);
  finalize_matrix(P);
  AIRT_CHECK_CUDA(cudaStreamSynchronize(s));
}

void sphere_stats(Problem &P, double *s2, double *s1, double *colcnt, double *cols1,
                  const double *colw, double *s2w) {
  cudaStream_t s = P.stream;
  const RayGeom g = P.geom();
  if (s2) AIRT_CHECK_CUDA(cudaMemsetAsync(s2, 0, P.m * sizeof(double), s));
  if (s1) AIRT_CHECK_CUDA(cudaMemsetAsync(s1, 0, P.m * sizeof(double), s));
  if (s2w) AIRT_CHECK_CUDA(cudaMemsetAsync(s2w, 0, P.m * sizeof(double), s));
  if (colcnt) AIRT_CHECK_CUDA(cudaMemsetAsync(colcnt, 0, P.n * sizeof(double), s));
  if (cols1) AIRT_CHECK_CUDA(cudaMemsetAsync(cols1, 0, P.n * sizeof(double), s));
  for_each_sphere_chunk(P, [&](const unsigned long long *uk, const int *cnt, int64_t n,
                               int64_t row0) {
    if (!n) return;
    k_sph_stats<<<grid_for(n, 256, 4), 256, 0, s>>>(g, uk, cnt, n, row0, s2, s1, colcnt, cols1,
                                                    colw, s2w);
    AIRT_LAUNCH_CHECK();
  });
}

}  // namespace airt
