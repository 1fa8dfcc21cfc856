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
//    ray order) and back projection (one thread per ray, FP64 atomic scatter)
//    that re-trace every ray, as the isMatrix = 0 handles of
//    paralleltomo.m:280-288 do.  Entry values are rounded to FP32 exactly as
//    the stored matrix holds them, so stored and matrix-free operators agree
//    up to summation order.
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

__global__ void k_mf_adjoint(RayGeom g, int64_t nrays, bool excl, const double *__restrict__ u,
                             double *__restrict__ y) {
  const int64_t nn = (int64_t)g.N * g.N;
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < nrays;
       r += (int64_t)gridDim.x * blockDim.x) {
    const double ur = u[r];
    if (ur == 0.0) continue;
    row_entries(g, r, excl, [&](int col, double v) {
      if (col >= 0 && col < nn) atomicAdd(y + col, (double)(float)v * ur);
    });
  }
}

// Per-ray sums (squares, absolute values, squares weighted by colw) and
// per-pixel counts and absolute sums, in one pass over the rays.
__global__ void k_mf_stats(RayGeom g, int64_t nrays, bool excl, double *__restrict__ s2,
                           double *__restrict__ s1, double *__restrict__ ccnt,
                           double *__restrict__ cs1, const double *__restrict__ colw,
                           double *__restrict__ s2w) {
  const int64_t nn = (int64_t)g.N * g.N;
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
      if (cs1) atomicAdd(cs1 + col, fabs(v));
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

void apply_matrix_free(Problem &P, const double *d_in, double *d_out, int transp) {
  cudaStream_t s = P.stream;
  const RayGeom g = P.geom();
  const unsigned grid = grid_for(P.m, 128, 16);
  if (!transp) {
    k_mf_forward<<<grid, 128, 0, s>>>(g, P.m, excl_of(P), d_in, d_out);
  } else {
    AIRT_CHECK_CUDA(cudaMemsetAsync(d_out, 0, P.n * sizeof(double), s));
    k_mf_adjoint<<<grid, 128, 0, s>>>(g, P.m, excl_of(P), d_in, d_out);
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
                                                      cols1, colw, s2w);
  AIRT_LAUNCH_CHECK();
}

// Matrix-free pieces of the SIRT iteration (used by sirt.cu).
namespace {
__global__ void k_mf_adjoint_f32(RayGeom g, int64_t nrays, bool excl, const float *__restrict__ u,
                                 double *__restrict__ y, const int *stop_flag) {
  if (stop_flag && *(volatile const int *)stop_flag) return;
  const int64_t nn = (int64_t)g.N * g.N;
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < nrays;
       r += (int64_t)gridDim.x * blockDim.x) {
    const double ur = (double)u[r];
    if (ur == 0.0) continue;
    row_entries(g, r, excl, [&](int col, double v) {
      if (col >= 0 && col < nn) atomicAdd(y + col, (double)(float)v * ur);
    });
  }
}
}  // namespace

void mf_backproject_f32(Problem &P, const float *u, double *g64, const int *stop_flag) {
  cudaStream_t s = P.stream;
  AIRT_CHECK_CUDA(cudaMemsetAsync(g64, 0, P.n * sizeof(double), s));
  k_mf_adjoint_f32<<<grid_for(P.m, 128, 16), 128, 0, s>>>(P.geom(), P.m, excl_of(P), u, g64,
                                                          stop_flag);
  AIRT_LAUNCH_CHECK();
}

}  // namespace airt
