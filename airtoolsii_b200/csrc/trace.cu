// GPU system-matrix generation and matrix-free projectors for the
// paralleltomo / fanlineartomo / fancurvedtomo / seismictomo geometries (and
// the matrix-free products of sphericaltomo, whose matrix is in sphere.cu).
//
//  * generate_matrix: two passes over the rays (count, then fill) with an
//    exclusive scan in between give the CSR over rays; the CSC follows by a
//    stable transposition.  Row entries keep the ray order of the trace.
//    Replaces testprobs/paralleltomo.m:112-301, fanlineartomo.m:141-358 and
//    seismictomo.m:96-287 (isMatrix = 1).
//  * apply_matrix_free: forward projection (one thread per ray, FP64 sum in
//    ray order) and back projection (one thread per ray, scatter in 64-bit
//    fixed point, so the result does not depend on the order in which rays
//    arrive) that re-trace every ray, as the isMatrix = 0 handles of
//    paralleltomo.m:280-288 do.  Entry values are rounded to FP32 exactly as
//    the stored matrix holds them, so stored and matrix-free operators agree
//    up to summation order.
#include <climits>
#include <cstring>

#include "common.cuh"
#include "spmv.cuh"
#include "stream.cuh"
#include "trace.cuh"

namespace airt {

namespace {

__global__ void k_trace_count(RayGeom g, int64_t nrays, bool excl, int64_t *__restrict__ counts,
                              int *__restrict__ bad) {
  const int64_t nn = (int64_t)g.N * g.N;
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < nrays;
       r += (int64_t)gridDim.x * blockDim.x) {
    const Ray q = ray_of(g, r);
    int64_t c = 0;
    trace_entries(g.N, q, excl, [&](int col, double) {
      if (col < 0 || col >= nn) atomicExch(bad, 1);
      else ++c;
    });
    counts[r] = c;
  }
}

__global__ void k_trace_fill(RayGeom g, int64_t nrays, bool excl, const int64_t *__restrict__ rp,
                             int *__restrict__ ci, float *__restrict__ rv) {
  const int64_t nn = (int64_t)g.N * g.N;
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < nrays;
       r += (int64_t)gridDim.x * blockDim.x) {
    const Ray q = ray_of(g, r);
    int64_t pos = rp[r];
    const int64_t end = rp[r + 1];
    trace_entries(g.N, q, excl, [&](int col, double v) {
      if (col >= 0 && col < nn && pos < end) {
        ci[pos] = col;
        rv[pos] = (float)v;
        ++pos;
      }
    });
  }
}

__global__ void k_mf_forward(RayGeom g, int64_t nrays, bool excl, const double *__restrict__ x,
                             double *__restrict__ y) {
  const int64_t nn = (int64_t)g.N * g.N;
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < nrays;
       r += (int64_t)gridDim.x * blockDim.x) {
    double acc = 0.0;
    row_entries(g, r, excl, [&](int col, double v) {
      if (col >= 0 && col < nn) acc = fma((double)(float)v, x[col], acc);
    });
    y[r] = acc;
  }
}

// ---- back projection in fixed point
// FP64 atomics add the rays' terms in whatever order the rays arrive, so the
// last bits of a back projection would change from run to run.  Instead
// every term (float)v * u is rounded once to an integer multiple of 2^-s and
// added as a 64-bit integer, which is associative.  s is chosen per call so
// that no sum can leave +-2^62: with kbound = T * max|v| (T the power of two
// at or above the most terms any pixel receives, max|v| a bound on the
// entries) and 2^e > kbound * max|u|, each term is below 2^62 / T in
// magnitude when scaled by 2^(62-e).  The quantum is then 2^-52 of the
// largest possible term for T = 2^10 -- FP64 accuracy -- and the result is
// bitwise the same on every run.
// 2^e > kbound * umax; INT_MIN when the product is 0 (the sums are 0),
// INT_MAX when it is not finite (the sums are NaN).
__device__ __forceinline__ int fx_exponent(double kbound, double umax) {
  const double prod = kbound * umax;
  if (!(prod < INFINITY)) return INT_MAX;
  return prod > 0.0 ? ilogb(prod) + 1 : INT_MIN;
}

__global__ void k_absmax(int64_t n, const double *__restrict__ u, const float *__restrict__ u32,
                         unsigned long long *__restrict__ bits, const int *stop_flag) {
  if (stop_flag && *(volatile const int *)stop_flag) return;
  double m = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    m = fmax(m, fabs(u ? u[i] : (double)u32[i]));
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0 && m > 0.0)  // nonnegative doubles order as their bits
    atomicMax(bits, (unsigned long long)__double_as_longlong(m));
}

template <typename TU>
__global__ void k_mf_adjoint_fx(RayGeom g, int64_t nrays, bool excl, const TU *__restrict__ u,
                                long long *__restrict__ acc, double kbound,
                                const unsigned long long *__restrict__ umax_bits,
                                const int *stop_flag) {
  if (stop_flag && *(volatile const int *)stop_flag) return;
  const int e = fx_exponent(kbound, __longlong_as_double((long long)*umax_bits));
  if (e == INT_MIN || e == INT_MAX) return;  // u == 0 (result 0) or not finite (NaN)
  const double sc = ldexp(1.0, 62 - e);
  const int64_t nn = (int64_t)g.N * g.N;
  // two adjacent threads per ray, each scattering one half of its entries
  // (row_entries_part): the entries are the same, and integer sums do not
  // depend on their order
  const int part = threadIdx.x & 1;
  for (int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 1; r < nrays;
       r += ((int64_t)gridDim.x * blockDim.x) >> 1) {
    const double ur = (double)u[r];
    if (ur == 0.0) continue;
    row_entries_part(g, r, excl, part, [&](int col, double v) {
      if (col >= 0 && col < nn) {
        const long long t = __double2ll_rn(__dmul_rn((double)(float)v, ur) * sc);
        atomicAdd(reinterpret_cast<unsigned long long *>(acc + col), (unsigned long long)t);
      }
    });
  }
}

// Fixed-point sums back to FP64, in place (acc and out are the same array).
__global__ void k_fx_to_f64(int64_t n, double *__restrict__ out, double kbound,
                            const unsigned long long *__restrict__ umax_bits, const int *stop_flag) {
  if (stop_flag && *(volatile const int *)stop_flag) return;
  const int e = fx_exponent(kbound, umax_bits ? __longlong_as_double((long long)*umax_bits) : 1.0);
  const double inv = e == INT_MIN ? 0.0 : e == INT_MAX ? __longlong_as_double(0x7ff8000000000000LL)
                                                       : ldexp(1.0, e - 62);
  long long *acc = reinterpret_cast<long long *>(out);
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n;
       j += (int64_t)gridDim.x * blockDim.x)
    out[j] = (double)acc[j] * inv;
}

// Terms each pixel receives and the largest entry, over every ray (the
// bounds of the fixed-point scale).
__global__ void k_mf_emit_stats(RayGeom g, int64_t nrays, bool excl, int *__restrict__ cnt,
                                unsigned long long *__restrict__ vmax_bits) {
  const int64_t nn = (int64_t)g.N * g.N;
  double vm = 0.0;
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < nrays;
       r += (int64_t)gridDim.x * blockDim.x)
    row_entries(g, r, excl, [&](int col, double v) {
      if (col >= 0 && col < nn) {
        atomicAdd(cnt + col, 1);
        vm = fmax(vm, fabs((double)(float)v));
      }
    });
  if (vm > 0.0) atomicMax(vmax_bits, (unsigned long long)__double_as_longlong(vm));
}

__global__ void k_max_int(int64_t n, const int *__restrict__ a, int *__restrict__ out) {
  int m = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    m = max(m, a[i]);
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

// Per-ray sums (squares, absolute values, squares weighted by colw) and
// per-pixel counts and absolute sums, in one pass over the rays.
// cs1 (column sums of |v|) is accumulated in fixed point (see above) with
// max|u| = 1 and converted by k_fx_to_f64.
__global__ void k_mf_stats(RayGeom g, int64_t nrays, bool excl, double *__restrict__ s2,
                           double *__restrict__ s1, double *__restrict__ ccnt,
                           double *__restrict__ cs1, const double *__restrict__ colw,
                           double *__restrict__ s2w, double kbound) {
  const int64_t nn = (int64_t)g.N * g.N;
  const double sc = ldexp(1.0, 62 - fx_exponent(kbound, 1.0));
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < nrays;
       r += (int64_t)gridDim.x * blockDim.x) {
    const Ray q = ray_of(g, r);
    double a2 = 0, a1 = 0, aw = 0;
    trace_entries(g.N, q, excl, [&](int col, double v64) {
      if (col < 0 || col >= nn) return;
      const double v = (double)(float)v64;
      a2 += v * v;
      a1 += fabs(v);
      if (colw) aw += v * v * colw[col];
      if (ccnt) atomicAdd(ccnt + col, 1.0);
      if (cs1)
        atomicAdd(reinterpret_cast<unsigned long long *>(cs1) + col,
                  (unsigned long long)__double2ll_rn(fabs(v) * sc));
    });
    if (s2) s2[r] = a2;
    if (s1) s1[r] = a1;
    if (s2w) s2w[r] = aw;
  }
}

inline bool excl_of(const Problem &P) { return P.geo_kind == GEO_PARALLEL; }

}  // namespace

void generate_matrix(Problem &P) {
  if (P.geo_kind == GEO_SPHERE) {
    generate_sphere_matrix(P);
    return;
  }
  cudaStream_t s = P.stream;
  const RayGeom g = P.geom();
  const int64_t nrays = P.m;
  DevBuf<int64_t> counts;
  DevBuf<int> bad;
  counts.ensure(nrays);
  bad.ensure(1);
  AIRT_CHECK_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int), s));
  const unsigned grid = grid_for(nrays, 128, 16);
  k_trace_count<<<grid, 128, 0, s>>>(g, nrays, excl_of(P), counts.p, bad.p);
  AIRT_LAUNCH_CHECK();
  P.rp.ensure(nrays + 1 + kPtrPad);
  AIRT_CHECK_CUDA(cudaMemsetAsync(P.rp.p + nrays + 1, 0, kPtrPad * sizeof(int64_t), s));
  exclusive_scan_i64(counts.p, P.rp.p, nrays, s);
  int hbad = 0;
  AIRT_CHECK_CUDA(cudaMemcpyAsync(&P.nnz, P.rp.p + nrays, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  AIRT_CHECK_CUDA(cudaMemcpyAsync(&hbad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  AIRT_CHECK_CUDA(cudaStreamSynchronize(s));
  AIRT_REQUIRE(!hbad, "ray trace produced a pixel index outside the image");
  P.ci.ensure(P.nnz + kPad);
  P.rv.ensure(P.nnz + kPad);
  AIRT_CHECK_CUDA(cudaMemsetAsync(P.ci.p + P.nnz, 0, kPad * sizeof(int), s));
  AIRT_CHECK_CUDA(cudaMemsetAsync(P.rv.p + P.nnz, 0, kPad * sizeof(float), s));
  k_trace_fill<<<grid, 128, 0, s>>>(g, nrays, excl_of(P), P.rp.p, P.ci.p, P.rv.p);
  AIRT_LAUNCH_CHECK();
  build_csc_from_csr(P);
  finalize_matrix(P);
  AIRT_CHECK_CUDA(cudaStreamSynchronize(s));
}

void mf_prepare(Problem &P) {
  cudaStream_t s = P.stream;
  DevBuf<int> cnt, cmax;
  DevBuf<unsigned long long> vbits;
  cnt.ensure(P.n > 0 ? P.n : 1);
  cmax.ensure(1);
  vbits.ensure(1);
  AIRT_CHECK_CUDA(cudaMemsetAsync(cnt.p, 0, (P.n > 0 ? P.n : 1) * sizeof(int), s));
  AIRT_CHECK_CUDA(cudaMemsetAsync(cmax.p, 0, sizeof(int), s));
  AIRT_CHECK_CUDA(cudaMemsetAsync(vbits.p, 0, sizeof(unsigned long long), s));
  if (P.m > 0)
    k_mf_emit_stats<<<grid_for(P.m, 128, 16), 128, 0, s>>>(P.geom(), P.m, excl_of(P), cnt.p,
                                                            vbits.p);
  if (P.n > 0) k_max_int<<<grid_for(P.n, 256), 256, 0, s>>>(P.n, cnt.p, cmax.p);
  AIRT_LAUNCH_CHECK();
  int hmax = 0;
  unsigned long long hv = 0;
  AIRT_CHECK_CUDA(cudaMemcpyAsync(&hmax, cmax.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  AIRT_CHECK_CUDA(cudaMemcpyAsync(&hv, vbits.p, sizeof(hv), cudaMemcpyDeviceToHost, s));
  AIRT_CHECK_CUDA(cudaStreamSynchronize(s));
  double T = 1.0;
  while (T < (double)hmax) T *= 2.0;
  double vmax = 0.0;
  std::memcpy(&vmax, &hv, sizeof(vmax));
  P.mf_kbound = T * (vmax > 0.0 ? vmax : 1.0);
  P.mf_umax.ensure(1);
}

void apply_matrix_free(Problem &P, const double *d_in, double *d_out, int transp) {
  cudaStream_t s = P.stream;
  const RayGeom g = P.geom();
  const unsigned grid = grid_for(P.m, 128, 16);
  if (!transp) {
    k_mf_forward<<<grid, 128, 0, s>>>(g, P.m, excl_of(P), d_in, d_out);
  } else {
    AIRT_CHECK_CUDA(cudaMemsetAsync(d_out, 0, P.n * sizeof(double), s));
    AIRT_CHECK_CUDA(cudaMemsetAsync(P.mf_umax.p, 0, sizeof(unsigned long long), s));
    k_absmax<<<grid_for(P.m, 256), 256, 0, s>>>(P.m, d_in, nullptr, P.mf_umax.p, nullptr);
    k_mf_adjoint_fx<double><<<grid_for(2 * P.m, 128, 16), 128, 0, s>>>(g, P.m, excl_of(P), d_in,
                                                 reinterpret_cast<long long *>(d_out),
                                                 P.mf_kbound, P.mf_umax.p, nullptr);
    k_fx_to_f64<<<grid_for(P.n, 256), 256, 0, s>>>(P.n, d_out, P.mf_kbound, P.mf_umax.p, nullptr);
  }
  AIRT_LAUNCH_CHECK();
}

void row_col_stats_mf(Problem &P, double *s2, double *s1, double *colcnt, double *cols1,
                      const double *colw, double *s2w) {
  if (P.geo_kind == GEO_SPHERE) {  // a circle's hits need merging into (pixel, count) first
    sphere_stats(P, s2, s1, colcnt, cols1, colw, s2w);
    return;
  }
  cudaStream_t s = P.stream;
  if (colcnt) AIRT_CHECK_CUDA(cudaMemsetAsync(colcnt, 0, P.n * sizeof(double), s));
  if (cols1) AIRT_CHECK_CUDA(cudaMemsetAsync(cols1, 0, P.n * sizeof(double), s));
  k_mf_stats<<<grid_for(P.m, 128, 16), 128, 0, s>>>(P.geom(), P.m, excl_of(P), s2, s1, colcnt,
                                                      cols1, colw, s2w, P.mf_kbound);
  if (cols1)
    k_fx_to_f64<<<grid_for(P.n, 256), 256, 0, s>>>(P.n, cols1, P.mf_kbound, nullptr, nullptr);
  AIRT_LAUNCH_CHECK();
}

// ---- check of the split trace: per ray, the entries of trace_entries and
// the union of trace_entries_part(0) and (1) compared by count and an
// order-independent hash of (pixel, FP64 value bits).
namespace {
__device__ __forceinline__ unsigned long long entry_hash(int col, double v) {
  unsigned long long z = (unsigned long long)__double_as_longlong(v) ^ ((unsigned long long)(unsigned)col << 1);
  z ^= z >> 33;
  z *= 0xff51afd7ed558ccdull;
  z ^= z >> 33;
  z *= 0xc4ceb9fe1a85ec53ull;
  z ^= z >> 33;
  return z;
}

__global__ void k_test_split(RayGeom g, int64_t nrays, bool excl, unsigned long long *__restrict__ bad,
                             unsigned long long *__restrict__ nsplit) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < nrays;
       r += (int64_t)gridDim.x * blockDim.x) {
    const Ray q = ray_of(g, r);
    unsigned long long h0 = 0, h1 = 0;
    long long c0 = 0, c1 = 0, c2 = 0;
    trace_entries(g.N, q, excl, [&](int col, double v) { h0 += entry_hash(col, v); ++c0; });
    trace_entries_part(g.N, q, excl, 0, [&](int col, double v) { h1 += entry_hash(col, v); ++c1; });
    trace_entries_part(g.N, q, excl, 1, [&](int col, double v) { h1 += entry_hash(col, v); ++c2; });
    if (h0 != h1 || c0 != c1 + c2) atomicAdd(bad, 1ull);
    if (c2 > 0) atomicAdd(nsplit, 1ull);
  }
}
}  // namespace

int64_t test_split_trace(Problem &P, int64_t *nsplit) {
  AIRT_REQUIRE(P.geo_kind != GEO_NONE && P.geo_kind != GEO_SPHERE, "the problem has no straight-ray geometry");
  cudaStream_t s = P.stream;
  DevBuf<unsigned long long> c;
  c.ensure(2);
  AIRT_CHECK_CUDA(cudaMemsetAsync(c.p, 0, 2 * sizeof(unsigned long long), s));
  k_test_split<<<grid_for(P.m, 128, 16), 128, 0, s>>>(P.geom(), P.m, excl_of(P), c.p, c.p + 1);
  AIRT_LAUNCH_CHECK();
  unsigned long long hc[2] = {0, 0};
  AIRT_CHECK_CUDA(cudaMemcpyAsync(hc, c.p, sizeof(hc), cudaMemcpyDeviceToHost, s));
  AIRT_CHECK_CUDA(cudaStreamSynchronize(s));
  if (nsplit) *nsplit = (int64_t)hc[1];
  return (int64_t)hc[0];
}

// Matrix-free pieces of the SIRT iteration (used by sirt.cu).
void mf_backproject_f32(Problem &P, const float *u, double *g64, const int *stop_flag) {
  cudaStream_t s = P.stream;
  AIRT_CHECK_CUDA(cudaMemsetAsync(g64, 0, P.n * sizeof(double), s));
  AIRT_CHECK_CUDA(cudaMemsetAsync(P.mf_umax.p, 0, sizeof(unsigned long long), s));
  k_absmax<<<grid_for(P.m, 256), 256, 0, s>>>(P.m, nullptr, u, P.mf_umax.p, stop_flag);
  k_mf_adjoint_fx<float><<<grid_for(2 * P.m, 64, 32), 64, 0, s>>>(
      P.geom(), P.m, excl_of(P), u, reinterpret_cast<long long *>(g64), P.mf_kbound, P.mf_umax.p,
      stop_flag);
  k_fx_to_f64<<<grid_for(P.n, 256), 256, 0, s>>>(P.n, g64, P.mf_kbound, P.mf_umax.p, stop_flag);
  AIRT_LAUNCH_CHECK();
}

}  // namespace airt
