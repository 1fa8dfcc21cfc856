// Sparse-format plumbing of libairt: MATLAB CSC ingest, CSR <-> CSC
// transposition, export back to MATLAB CSC, the method weights of
// auxil/get_mfun_dfun.m and the plain operator products of
// auxil/afun_matrix.m:44-53.
//
// Layout in HBM: CSR over rays (int64 row starts, int32 columns, FP32 values)
// for A*x, and CSC over pixels (int64 column starts, int32 rows, FP32 values)
// for A'*y, so both products are gathers with no atomics.  The one-off
// transposition uses a stable key sort (CUB radix sort) so the entries of
// every column stay in ascending row order, as in MATLAB's CSC.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "common.cuh"
#include "spmv.cuh"
#include "stream.cuh"

namespace airt {

void exclusive_scan_i64(const int64_t *counts, int64_t *offs, int64_t n, cudaStream_t s) {
  AIRT_CHECK_CUDA(cudaMemsetAsync(offs, 0, sizeof(int64_t), s));
  if (n == 0) return;
  size_t tmp = 0;
  AIRT_CHECK_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tmp, counts, offs + 1, (int)n, s));
  DevBuf<unsigned char> t;
  t.ensure(tmp);
  AIRT_CHECK_CUDA(cub::DeviceScan::InclusiveSum(t.p, tmp, counts, offs + 1, (int)n, s));
  AIRT_CHECK_CUDA(cudaStreamSynchronize(s));
}

namespace {

__global__ void k_expand_major(int64_t nmaj, const int64_t *__restrict__ ptr, int *__restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nmaj;
       i += (int64_t)gridDim.x * blockDim.x)
    for (int64_t q = ptr[i]; q < ptr[i + 1]; ++q) out[q] = (int)i;
}

__global__ void k_pack(int64_t nnz, const int *__restrict__ major, const float *__restrict__ val,
                       unsigned long long *__restrict__ packed) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nnz;
       q += (int64_t)gridDim.x * blockDim.x)
    packed[q] = ((unsigned long long)(unsigned)major[q] << 32) | __float_as_uint(val[q]);
}

__global__ void k_unpack(int64_t nnz, const unsigned long long *__restrict__ packed,
                         int *__restrict__ idx, float *__restrict__ val) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nnz;
       q += (int64_t)gridDim.x * blockDim.x) {
    unsigned long long v = packed[q];
    idx[q] = (int)(v >> 32);
    val[q] = __uint_as_float((unsigned)(v & 0xffffffffu));
  }
}

__global__ void k_count(int64_t nnz, const int *__restrict__ key, unsigned long long *__restrict__ cnt) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nnz;
       q += (int64_t)gridDim.x * blockDim.x)
    atomicAdd(&cnt[key[q]], 1ull);
}

__global__ void k_csc64_to_f32(int64_t nnz, const uint64_t *__restrict__ ir, const double *__restrict__ pr,
                               int *__restrict__ ri, float *__restrict__ cv, int64_t m, int *bad) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nnz;
       q += (int64_t)gridDim.x * blockDim.x) {
    uint64_t r = ir[q];
    if (r >= (uint64_t)m) { atomicExch(bad, 1); r = 0; }
    ri[q] = (int)r;
    cv[q] = (float)pr[q];
  }
}

// MATLAB's canonical sparse form: row indices strictly increasing within
// each column (no duplicates).  One thread per column; sets *bad = 2.
__global__ void k_check_col_sorted(int64_t n, const uint64_t *__restrict__ jc,
                                   const uint64_t *__restrict__ ir, int *bad) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n;
       j += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t q1 = jc[j + 1];
    for (uint64_t q = jc[j] + 1; q < q1; ++q)
      if (ir[q] <= ir[q - 1]) {
        atomicExch(bad, 2);
        break;
      }
  }
}

__global__ void k_u64_to_i64(int64_t n, const uint64_t *__restrict__ a, int64_t *__restrict__ b) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n;
       q += (int64_t)gridDim.x * blockDim.x)
    b[q] = (int64_t)a[q];
}

// Stable transposition: entries given in major order (ptr_in / minor_in /
// val_in over nmaj segments) are regrouped by their minor index; within each
// new segment the old major index ascends.
void transpose(int64_t nmaj, int64_t nmin, int64_t nnz, const int64_t *ptr_in, const int *minor_in,
               const float *val_in, DevBuf<int64_t> &ptr_out, DevBuf<int> &minor_out,
               DevBuf<float> &val_out, cudaStream_t s) {
  ptr_out.ensure(nmin + 1 + kPtrPad);
  AIRT_CHECK_CUDA(cudaMemsetAsync(ptr_out.p + nmin + 1, 0, kPtrPad * sizeof(int64_t), s));
  minor_out.ensure(nnz + kPad);
  val_out.ensure(nnz + kPad);
  AIRT_CHECK_CUDA(cudaMemsetAsync(minor_out.p + nnz, 0, kPad * sizeof(int), s));
  AIRT_CHECK_CUDA(cudaMemsetAsync(val_out.p + nnz, 0, kPad * sizeof(float), s));
  if (nnz == 0) {
    AIRT_CHECK_CUDA(cudaMemsetAsync(ptr_out.p, 0, (nmin + 1) * sizeof(int64_t), s));
    return;
  }
  AIRT_REQUIRE(nnz < (int64_t)INT32_MAX * 2, "nnz too large for the transposition");
  DevBuf<int> major;
  DevBuf<unsigned> keys_out;
  DevBuf<unsigned long long> packed, packed_out, cnt;
  major.ensure(nnz);
  keys_out.ensure(nnz);
  packed.ensure(nnz);
  packed_out.ensure(nnz);
  cnt.ensure(nmin);
  unsigned g = grid_for(nnz, 256);
  k_expand_major<<<grid_for(nmaj, 256), 256, 0, s>>>(nmaj, ptr_in, major.p);
  AIRT_LAUNCH_CHECK();
  k_pack<<<g, 256, 0, s>>>(nnz, major.p, val_in, packed.p);
  AIRT_LAUNCH_CHECK();
  int bits = 1;
  while (bits < 31 && (1ll << bits) < nmin) ++bits;
  size_t tmp = 0;
  AIRT_CHECK_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, (const unsigned *)minor_in, keys_out.p, packed.p,
                                                  packed_out.p, (int)nnz, 0, bits, s));
  DevBuf<unsigned char> t;
  t.ensure(tmp);
  AIRT_CHECK_CUDA(cub::DeviceRadixSort::SortPairs(t.p, tmp, (const unsigned *)minor_in, keys_out.p, packed.p,
                                                  packed_out.p, (int)nnz, 0, bits, s));
  k_unpack<<<g, 256, 0, s>>>(nnz, packed_out.p, minor_out.p, val_out.p);
  AIRT_LAUNCH_CHECK();
  AIRT_CHECK_CUDA(cudaMemsetAsync(cnt.p, 0, nmin * sizeof(unsigned long long), s));
  k_count<<<g, 256, 0, s>>>(nnz, minor_in, cnt.p);
  AIRT_LAUNCH_CHECK();
  exclusive_scan_i64((const int64_t *)cnt.p, ptr_out.p, nmin, s);
}

}  // namespace

// Greedy tiles of whole segments: a tile closes before the segment that
// would push it past kTileNnz nonzeros or kTileSeg segments.
bool build_tiles(Problem &P, const int64_t *d_ptr, int64_t nseg, DevBuf<int> &tiles, int &ntiles) {
  ntiles = 0;
  if (nseg <= 0 || nseg >= INT32_MAX) return false;
  std::vector<int64_t> h(nseg + 1);
  AIRT_CHECK_CUDA(cudaMemcpyAsync(h.data(), d_ptr, (nseg + 1) * sizeof(int64_t),
                                  cudaMemcpyDeviceToHost, P.stream));
  AIRT_CHECK_CUDA(cudaStreamSynchronize(P.stream));
  std::vector<int> ts;
  ts.push_back(0);
  int64_t tile_e0 = h[0];
  int tile_nseg = 0;
  for (int64_t i = 0; i < nseg; ++i) {
    const int64_t len = h[i + 1] - h[i];
    if (len > kTileNnz) return false;
    if (tile_nseg == kTileSeg || h[i + 1] - tile_e0 > kTileNnz) {
      ts.push_back((int)i);
      tile_e0 = h[i];
      tile_nseg = 0;
    }
    ++tile_nseg;
  }
  ts.push_back((int)nseg);
  if (ts.size() >= (size_t)INT32_MAX) return false;
  ntiles = (int)ts.size() - 1;
  tiles.upload(ts.data(), ts.size(), P.stream);
  AIRT_CHECK_CUDA(cudaStreamSynchronize(P.stream));
  return true;
}

void finalize_matrix(Problem &P) {
  P.stream_ok = build_tiles(P, P.rp.p, P.m, P.rtiles, P.nrtiles) &&
                build_tiles(P, P.cp.p, P.n, P.ctiles, P.nctiles);
}

void build_csc_from_csr(Problem &P) {
  transpose(P.m, P.n, P.nnz, P.rp.p, P.ci.p, P.rv.p, P.cp, P.ri, P.cv, P.stream);
}

void build_csr_from_host_csc(Problem &P, const uint64_t *jc, const uint64_t *ir, const double *pr) {
  cudaStream_t s = P.stream;
  DevBuf<uint64_t> djc, dir;
  DevBuf<double> dpr;
  djc.upload(jc, P.n + 1, s);
  dir.upload(ir, P.nnz, s);
  dpr.upload(pr, P.nnz, s);
  P.cp.ensure(P.n + 1 + kPtrPad);
  AIRT_CHECK_CUDA(cudaMemsetAsync(P.cp.p + P.n + 1, 0, kPtrPad * sizeof(int64_t), s));
  P.ri.ensure(P.nnz + kPad);
  P.cv.ensure(P.nnz + kPad);
  AIRT_CHECK_CUDA(cudaMemsetAsync(P.ri.p + P.nnz, 0, kPad * sizeof(int), s));
  AIRT_CHECK_CUDA(cudaMemsetAsync(P.cv.p + P.nnz, 0, kPad * sizeof(float), s));
  DevBuf<int> bad;
  bad.ensure(1);
  AIRT_CHECK_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int), s));
  k_u64_to_i64<<<grid_for(P.n + 1, 256), 256, 0, s>>>(P.n + 1, djc.p, P.cp.p);
  AIRT_LAUNCH_CHECK();
  if (P.nnz) {
    k_csc64_to_f32<<<grid_for(P.nnz, 256), 256, 0, s>>>(P.nnz, dir.p, dpr.p, P.ri.p, P.cv.p, P.m,
                                                         bad.p);
    AIRT_LAUNCH_CHECK();
    k_check_col_sorted<<<grid_for(P.n, 256), 256, 0, s>>>(P.n, djc.p, dir.p, bad.p);
    AIRT_LAUNCH_CHECK();
  }
  int hbad = 0;
  AIRT_CHECK_CUDA(cudaMemcpyAsync(&hbad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  AIRT_CHECK_CUDA(cudaStreamSynchronize(s));
  AIRT_REQUIRE(hbad != 1, "row index out of range in the CSC input");
  AIRT_REQUIRE(hbad != 2,
               "row indices of a CSC column are not strictly increasing (the matrix must be in "
               "MATLAB's canonical sparse form: sorted, no duplicate entries)");
  transpose(P.n, P.m, P.nnz, P.cp.p, P.ri.p, P.cv.p, P.rp, P.ci, P.rv, s);
}

namespace {
__global__ void k_export(int64_t nnz, const int *__restrict__ ri, const float *__restrict__ cv,
                         uint64_t *__restrict__ ir, double *__restrict__ pr) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nnz;
       q += (int64_t)gridDim.x * blockDim.x) {
    ir[q] = (uint64_t)ri[q];
    pr[q] = (double)cv[q];
  }
}
}  // namespace

void export_csc(Problem &P, uint64_t *jc, uint64_t *ir, double *pr) {
  AIRT_REQUIRE(!P.matrix_free, "a matrix-free operator has no stored matrix to export");
  cudaStream_t s = P.stream;
  DevBuf<uint64_t> dir;
  DevBuf<double> dpr;
  dir.ensure(P.nnz);
  dpr.ensure(P.nnz);
  if (P.nnz) {
    k_export<<<grid_for(P.nnz, 256), 256, 0, s>>>(P.nnz, P.ri.p, P.cv.p, dir.p, dpr.p);
    AIRT_LAUNCH_CHECK();
  }
  std::vector<int64_t> hcp(P.n + 1);
  AIRT_CHECK_CUDA(cudaMemcpyAsync(hcp.data(), P.cp.p, (P.n + 1) * sizeof(int64_t),
                                  cudaMemcpyDeviceToHost, s));
  if (P.nnz) {
    AIRT_CHECK_CUDA(cudaMemcpyAsync(ir, dir.p, P.nnz * sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
    AIRT_CHECK_CUDA(cudaMemcpyAsync(pr, dpr.p, P.nnz * sizeof(double), cudaMemcpyDeviceToHost, s));
  }
  AIRT_CHECK_CUDA(cudaStreamSynchronize(s));
  for (int64_t j = 0; j <= P.n; ++j) jc[j] = (uint64_t)hcp[j];
}

// ------------------------------------------------------------------ weights
namespace {

// Per-row sums of squares and of absolute values (get_mfun_dfun.m:62-67,
// 203-207), FP64 accumulation of the FP32 entries.
template <int LANES>
__global__ void k_row_stats(int64_t m, const int64_t *__restrict__ rp, const int *__restrict__ ci,
                            const float *__restrict__ rv, const double *__restrict__ colw,
                            double *__restrict__ s2, double *__restrict__ s1,
                            double *__restrict__ s2w) {
  const int lane = threadIdx.x % LANES;
  const int64_t gid = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / LANES;
  const int64_t ng = (int64_t)gridDim.x * blockDim.x / LANES;
  const int64_t iters = (m + ng - 1) / ng;
  for (int64_t it = 0; it < iters; ++it) {
    const int64_t i = gid + it * ng;
    double a2 = 0, a1 = 0, aw = 0;
    if (i < m) {
      for (int64_t q = rp[i] + lane; q < rp[i + 1]; q += LANES) {
        double v = (double)rv[q];
        a2 += v * v;
        a1 += fabs(v);
        if (colw) aw += v * v * colw[ci[q]];
      }
    }
    a2 = group_sum<LANES>(a2);
    a1 = group_sum<LANES>(a1);
    if (colw) aw = group_sum<LANES>(aw);
    if (lane == 0 && i < m) {
      if (s2) s2[i] = a2;
      if (s1) s1[i] = a1;
      if (s2w) s2w[i] = aw;
    }
  }
}

// Per-column nonzero counts and absolute sums (get_mfun_dfun.m:93-97,
// 226-228).
template <int LANES>
__global__ void k_col_stats(int64_t n, const int64_t *__restrict__ cp, const float *__restrict__ cv,
                            double *__restrict__ cnt, double *__restrict__ s1) {
  const int lane = threadIdx.x % LANES;
  const int64_t gid = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / LANES;
  const int64_t ng = (int64_t)gridDim.x * blockDim.x / LANES;
  const int64_t iters = (n + ng - 1) / ng;
  for (int64_t it = 0; it < iters; ++it) {
    const int64_t j = gid + it * ng;
    double c = 0, a1 = 0;
    if (j < n) {
      for (int64_t q = cp[j] + lane; q < cp[j + 1]; q += LANES) {
        double v = (double)cv[q];
        c += (v != 0.0) ? 1.0 : 0.0;
        a1 += fabs(v);
      }
    }
    c = group_sum<LANES>(c);
    a1 = group_sum<LANES>(a1);
    if (lane == 0 && j < n) {
      if (cnt) cnt[j] = c;
      if (s1) s1[j] = a1;
    }
  }
}

// w[i] = scale * (1 / v[i]) with 1/0 = Inf replaced by 0 (get_mfun_dfun.m:83-85).
__global__ void k_recip(int64_t n, const double *__restrict__ v, double scale, double *__restrict__ w) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    double r = 1.0 / v[i];
    double x = (scale == 1.0) ? r : scale * r;
    w[i] = (x == __longlong_as_double(0x7ff0000000000000ll)) ? 0.0 : x;
  }
}

__global__ void k_fill(int64_t n, double v, double *__restrict__ w) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    w[i] = v;
}

}  // namespace

void row_col_stats_mf(Problem &P, double *s2, double *s1, double *colcnt, double *cols1,
                      const double *colw, double *s2w);

// Squared row norms of the stored matrix (FP64 sums of the FP32 entries).
void row_sums_sq(Problem &P, double *out) {
  k_row_stats<32><<<grid_for(P.m * 32, 256), 256, 0, P.stream>>>(P.m, P.rp.p, P.ci.p, P.rv.p,
                                                                  nullptr, out, nullptr, nullptr);
  AIRT_LAUNCH_CHECK();
}

// dM (m) and dD (n) receive the diagonals; landweber gives ones.
void compute_weights(Problem &P, int method, double *dM, double *dD) {
  cudaStream_t s = P.stream;
  const int64_t m = P.m, n = P.n;
  DevBuf<double> &t1 = P.w1, &t2 = P.w2;
  t1.ensure(m > n ? m : n);
  t2.ensure(n);
  auto rows = [&](double *s2, double *s1, const double *colw, double *s2w) {
    if (P.matrix_free) {
      row_col_stats_mf(P, s2, s1, nullptr, nullptr, colw, s2w);
      return;
    }
    k_row_stats<32><<<grid_for(m * 32, 256), 256, 0, s>>>(m, P.rp.p, P.ci.p, P.rv.p, colw, s2, s1, s2w);
    AIRT_LAUNCH_CHECK();
  };
  auto cols = [&](double *cnt, double *s1) {
    if (P.matrix_free) {
      row_col_stats_mf(P, nullptr, nullptr, cnt, s1, nullptr, nullptr);
      return;
    }
    k_col_stats<32><<<grid_for(n * 32, 256), 256, 0, s>>>(n, P.cp.p, P.cv.p, cnt, s1);
    AIRT_LAUNCH_CHECK();
  };
  switch (method) {
    case AIRT_LANDWEBER:
      k_fill<<<grid_for(m, 256), 256, 0, s>>>(m, 1.0, dM);
      k_fill<<<grid_for(n, 256), 256, 0, s>>>(n, 1.0, dD);
      break;
    case AIRT_CIMMINO:  // M = 1/m * (1./||a_i||^2), D = I
      rows(t1.p, nullptr, nullptr, nullptr);
      k_recip<<<grid_for(m, 256), 256, 0, s>>>(m, t1.p, 1.0 / (double)m, dM);
      k_fill<<<grid_for(n, 256), 256, 0, s>>>(n, 1.0, dD);
      break;
    case AIRT_CAV:  // M = 1./(sum_j a_ij^2 s_j), s_j = nnz(column j), D = I
      cols(t2.p, nullptr);
      rows(nullptr, nullptr, t2.p, t1.p);
      k_recip<<<grid_for(m, 256), 256, 0, s>>>(m, t1.p, 1.0, dM);
      k_fill<<<grid_for(n, 256), 256, 0, s>>>(n, 1.0, dD);
      break;
    case AIRT_DROP:  // M = 1./||a_i||^2, D = 1./nnz(column j)
      rows(t1.p, nullptr, nullptr, nullptr);
      k_recip<<<grid_for(m, 256), 256, 0, s>>>(m, t1.p, 1.0, dM);
      cols(t2.p, nullptr);
      k_recip<<<grid_for(n, 256), 256, 0, s>>>(n, t2.p, 1.0, dD);
      break;
    case AIRT_SART:  // M = 1./sum_j |a_ij|, D = 1./sum_i |a_ij|
      rows(nullptr, t1.p, nullptr, nullptr);
      k_recip<<<grid_for(m, 256), 256, 0, s>>>(m, t1.p, 1.0, dM);
      cols(nullptr, t2.p);
      k_recip<<<grid_for(n, 256), 256, 0, s>>>(n, t2.p, 1.0, dD);
      break;
    default:
      AIRT_REQUIRE(false, "SIRT method not defined.");
  }
  AIRT_LAUNCH_CHECK();
}

// ------------------------------------------------------------------ apply
void apply_operator(Problem &P, const double *d_in, double *d_out, int transp) {
  cudaStream_t s = P.stream;
  if (P.matrix_free) {
    apply_matrix_free(P, d_in, d_out, transp);
    return;
  }
  if (!transp)
    spmv_plain(P.m, P.rp.p, P.ci.p, P.rv.p, d_in, d_out, s);
  else
    spmv_plain(P.n, P.cp.p, P.ri.p, P.cv.p, d_in, d_out, s);
}

}  // namespace airt
