// Internal types of libairt: device buffers, the problem handle, error
// plumbing and small device helpers shared by the kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/airt.h"

namespace airt {

// ---------------------------------------------------------------- errors
struct Status {
  int code;
};

void set_error(const char *fmt, ...);

#define AIRT_CHECK_CUDA(call)                                                              \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess) {                                                               \
      ::airt::set_error("%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, \
                        __LINE__);                                                         \
      throw ::airt::Status{e_ == cudaErrorMemoryAllocation ? AIRT_ERR_OOM : AIRT_ERR_CUDA}; \
    }                                                                                      \
  } while (0)

#define AIRT_REQUIRE(cond, ...)      \
  do {                               \
    if (!(cond)) {                   \
      ::airt::set_error(__VA_ARGS__); \
      throw ::airt::Status{AIRT_ERR_ARG}; \
    }                                \
  } while (0)

#define AIRT_LAUNCH_CHECK() AIRT_CHECK_CUDA(cudaGetLastError())

// ---------------------------------------------------------------- buffers
// Test hook (airt_test_fail_alloc): < 0 off; otherwise the number of device
// allocations through DevBuf that still succeed before one fails as if the
// device were out of memory.
extern int g_alloc_fail_countdown;

template <typename T>
struct DevBuf {
  T *p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  DevBuf(DevBuf &&o) noexcept : p(o.p), n(o.n) {
    o.p = nullptr;
    o.n = 0;
  }
  DevBuf &operator=(DevBuf &&o) noexcept {
    if (this != &o) {
      release();
      p = o.p;
      n = o.n;
      o.p = nullptr;
      o.n = 0;
    }
    return *this;
  }
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  // Grow-only allocation; contents are not preserved.
  void ensure(size_t count) {
    if (count <= n && p) return;
    release();
    size_t bytes = (count ? count : 1) * sizeof(T);
    if (g_alloc_fail_countdown >= 0 && g_alloc_fail_countdown-- == 0) {
      set_error("cudaMalloc of %zu bytes failed: injected allocation failure (test hook)", bytes);
      throw Status{AIRT_ERR_OOM};
    }
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
      p = nullptr;
      set_error("cudaMalloc of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
      throw Status{AIRT_ERR_OOM};
    }
    n = count;
  }
  void upload(const T *host, size_t count, cudaStream_t s) {
    ensure(count);
    if (count)
      AIRT_CHECK_CUDA(cudaMemcpyAsync(p, host, count * sizeof(T), cudaMemcpyHostToDevice, s));
  }
};

// ---------------------------------------------------------------- geometry
enum GeoKind { GEO_NONE = 0, GEO_PARALLEL = 1, GEO_FAN = 2, GEO_SEISMIC = 3, GEO_SPHERE = 4 };

// Per-ray parameters of the geometries, prepared on the device: ray
// r = i*p + j (i = angle or source, j = detector or receiver) starts at
// (x0t, y0t) with direction (a, b).  For GEO_SPHERE, row r = i*p + n is
// circle n of radius radius[n] about (cos_t[i], sin_t[i]), sampled at the
// angles whose cosines and sines are cos_k/sin_k[koff[n] .. koff[n+1]).
struct RayGeom {
  int kind;
  int N, nA, p;
  double R;
  const double *cos_t, *sin_t;  // nA
  const double *offsets;         // p (parallel)
  const double *cos_w, *sin_w;  // p (fan)
  const double *src_x, *src_y;  // nA sources (seismic)
  const double *rcv_x, *rcv_y;  // p receivers (seismic)
  const double *radius, *cscale;  // p circles: radius, entry value per hit (sphere)
  const int64_t *koff;            // p + 1 sample offsets (sphere)
  const double *cos_k, *sin_k;    // koff[p] samples (sphere)
  double dx;                      // pixel size sqrt(2)/N (sphere)
  int center;                     // ceil(N/2) (sphere)
};

// ---------------------------------------------------------------- SIRT state
// Device-resident iteration state.  The control kernel is its only writer
// between kernels; all other kernels only read it (and add to acc[]).
struct SirtState {
  int iter;       // iteration whose residual the next control step judges
  int stop;       // 1 once a stopping rule fired
  int stoprule;   // info.stoprule
  int finaliter;  // info.finaliter
  double acc[6];  // [0] sum r^2  [1] sum r.*M.*r  [2] sum rprev^2  [3] sum rprev.*r
                  // [4] sum D.*g.^2 (line search)
  double lam_cur; // relaxpar applied in the iteration being computed
  double lam_last;
  double rmr_prev;  // r'*M*r of the previous residual (line search numerator)
};

// State of the multi-right-hand-side SIRT (multirhs.cu).
struct MultiState {
  int iter;    // global iteration whose residuals the control step judges next
  int active;  // instances not stopped
  double lam;  // relaxpar of the iteration being computed
};

struct SirtParams {
  int64_t kmax;
  int stoprule;
  double taudelta;
  int relax_kind;
  double relaxpar;
  const double *relax_table;  // device, kmax entries
  double *resn_hist;          // device, kmax+1
  double *lam_hist;           // device, kmax+1
  // NCP: per-column distances of the current residual, history of ncc
  const double *ncc_col;      // device, ncp_cols
  double *dk;                 // device, ncp_smooth (starts at +inf)
  int ncp_cols, ncp_smooth;
};

// Dependency schedule of a Kaczmarz row order (art.cu): the steps sorted by
// level, their positions in the order, and each step's predecessors.
struct ArtSchedule {
  int nlev = 0;
  int64_t nsteps = 0;
  uint64_t key = 0;  // hash of the row order it was built for (0: none)
  DevBuf<int> steps, pos, pred_ptr, preds;
};

// ---------------------------------------------------------------- problem
struct Problem {
  int64_t m = 0, n = 0, nnz = 0;
  bool matrix_free = false;
  int geo_kind = GEO_NONE;
  int N = 0, nA = 0, p = 0;
  double R = 0;
  DevBuf<double> cos_t, sin_t, offsets, cos_w, sin_w;
  DevBuf<double> src_x, src_y, rcv_x, rcv_y;  // seismic: nA sources, p receivers
  DevBuf<double> radius, cscale, cos_k, sin_k;  // sphere: p circles and their samples
  DevBuf<int64_t> koff;
  int64_t koff_total = 0;  // samples per angle
  double dx = 0;
  int center = 0;

  // stored matrix: CSR over rays (rows) and CSC over pixels (columns)
  DevBuf<int64_t> rp, cp;
  DevBuf<int> ci, ri;
  DevBuf<float> rv, cv;

  // SIRT SpMV kernel family: 0 vectorised gathers (spmv.cuh), 1 bulk-async
  // streamed tiles (stream.cuh); chosen from AIRT_SPMV=stream at creation
  int spmv_kind = 0;
  // tile tables of the streamed kernels (stream.cuh)
  bool stream_ok = false;
  DevBuf<int> rtiles, ctiles;
  int nrtiles = 0, nctiles = 0;
  DevBuf<int> err;  // device error flag (bounded waits)

  // reusable scratch of the weight and rho computations
  DevBuf<double> w1, w2;
  // matrix-free back projection in fixed point (trace.cu): bound on
  // (terms per pixel) x max |entry|, and the per-call max |u| (as bits)
  double mf_kbound = 0.0;
  DevBuf<unsigned long long> mf_umax;

  cudaStream_t stream = nullptr;

  // solver work vectors
  DevBuf<double> x64, r64, rprev, g64, b64, M, D, lbv, ubv, vin, vout, table, resn, lamh, Xd;
  // custom SIRT weights given as full matrices (get_mfun_dfun.m:252-307, flag 2):
  // column-major m x m / n x n, and the column sums of D (line search)
  DevBuf<double> Mfull, Dfull, Dcol, dscratch;
  // Kaczmarz schedule of the last fixed row order (kept between calls: the
  // matrix never changes, so the same order gives the same schedule)
  ArtSchedule art_sched;
  // multi-right-hand-side SIRT (multirhs.cu): interleaved [row or pixel][instance]
  DevBuf<double> mr_b, mr_x64, mr_part, mr_resn, mr_taud, mr_lam;
  DevBuf<float> mr_x32, mr_r32;
  DevBuf<int> mr_stop, mr_iters, mr_rule;
  DevBuf<MultiState> mr_state;
  // NCP stopping rule: DFT twiddles (cos, sin pairs), power spectra, column distances, history
  DevBuf<double> ncp_tw, ncp_pk, ncp_col, ncp_dk;
  // fbp: filter kernel, per-column scales, filtered sinogram (kept between calls)
  DevBuf<double> fbp_h, fbp_scale, fbp_tmp;
  int ncp_len = 0;  // column length the twiddles were made for
  DevBuf<float> x32, mr32;
  DevBuf<SirtState> state;
  DevBuf<SirtParams> params;
  DevBuf<int> save_slot;
  SirtState *h_state = nullptr;  // pinned mirror

  // instrumentation
  bool profiling = false;
  std::vector<cudaEvent_t> ev_pool;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> ev_pending;
  int64_t prof_launches[2] = {0, 0};
  double prof_ms[2] = {0, 0};

  RayGeom geom() const {
    RayGeom g;
    g.kind = geo_kind;
    g.N = N;
    g.nA = nA;
    g.p = p;
    g.R = R;
    g.cos_t = cos_t.p;
    g.sin_t = sin_t.p;
    g.offsets = offsets.p;
    g.cos_w = cos_w.p;
    g.sin_w = sin_w.p;
    g.src_x = src_x.p;
    g.src_y = src_y.p;
    g.rcv_x = rcv_x.p;
    g.rcv_y = rcv_y.p;
    g.radius = radius.p;
    g.cscale = cscale.p;
    g.koff = koff.p;
    g.cos_k = cos_k.p;
    g.sin_k = sin_k.p;
    g.dx = dx;
    g.center = center;
    return g;
  }
};

// ---------------------------------------------------------------- helpers
inline int num_sms() {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 148;
  }
  return sms;
}

inline unsigned grid_for(int64_t work, int per_block, int blocks_per_sm = 8) {
  int64_t need = (work + per_block - 1) / per_block;
  int64_t cap = (int64_t)num_sms() * blocks_per_sm;
  if (need < 1) need = 1;
  return (unsigned)(need < cap ? need : cap);
}

// Profiling brackets around one kernel launch (no-ops unless enabled).
void prof_begin(Problem &P, int which, cudaEvent_t *ev0);
void prof_end(Problem &P, int which, cudaEvent_t ev0);
void prof_collect(Problem &P);

// Kernel drivers implemented in the .cu files.
void build_csc_from_csr(Problem &P);
// sphericaltomo (sphere.cu): the system matrix, and the exact row/column
// statistics of its matrix-free operator
void generate_sphere_matrix(Problem &P);
void sphere_stats(Problem &P, double *s2, double *s1, double *colcnt, double *cols1,
                  const double *colw, double *s2w);
void build_csr_from_host_csc(Problem &P, const uint64_t *jc, const uint64_t *ir, const double *pr);
void finalize_matrix(Problem &P);
void generate_matrix(Problem &P);
// Bounds of the fixed-point back projection of a matrix-free problem (one
// pass over the rays at creation; trace.cu).
void mf_prepare(Problem &P);
// Rays whose two-part trace differs from the whole trace (test hook); *nsplit: rays split.
int64_t test_split_trace(Problem &P, int64_t *nsplit);
void apply_operator(Problem &P, const double *d_in, double *d_out, int transp);
void compute_weights(Problem &P, int method, double *dM, double *dD);
void run_sirt_multi(Problem &P, const airt_sirt_opts &o, int K, const double *d_B,
                    const double *d_X0, const double *taud_host, const double *lam_host,
                    const int64_t *Ksave, int64_t nsave, double *d_Xs, double *d_X,
                    int64_t *finaliter, int *stoprule, double *gpu_ms);
void run_sirt(Problem &P, const airt_sirt_opts &o, const double *d_b, const double *d_x0,
              const int64_t *K, int64_t nK, double *d_X, double *resn_host, airt_info *info);
// Stopping-rule state of the sweep loops of ART and CART (DP, NCP and NONE
// branches of check_stoprules.m:54-151): judge(k, ||r_k||, ncc_k) once per
// sweep, with the NCP history dk of check_inputs.m:209 (+inf initially).
struct SweepStop {
  int rule;
  double taudelta;
  int64_t kmax;
  std::vector<double> dk;
  bool stop = false;
  int stoprule = 0;
  int64_t finaliter = 0;
  SweepStop(int rule_, double taudelta_, int64_t kmax_, int ncp_smooth)
      : rule(rule_), taudelta(taudelta_), kmax(kmax_),
        dk(rule_ == AIRT_STOP_NCP ? ncp_smooth : 0, INFINITY) {}
  void judge(int64_t k, double nrk, double ncc) {
    if (rule == AIRT_STOP_DP) {
      if (nrk <= taudelta || k >= kmax) {
        stop = true;
        stoprule = (k != kmax) ? 2 : 0;
      }
    } else if (rule == AIRT_STOP_NCP) {  // check_stoprules.m:124-149
      double mx = -INFINITY, mxn = ncc;
      for (double v : dk) mx = std::fmax(mx, v);
      for (size_t i = 1; i < dk.size(); ++i) mxn = std::fmax(mxn, dk[i]);
      if (mx < mxn || k >= kmax) {
        stop = true;
        stoprule = (k != kmax) ? 1 : 0;
      } else {
        dk.erase(dk.begin());
        dk.push_back(ncc);
      }
    } else if (k >= kmax) {
      stop = true;
    }
    if (stop) finaliter = k;
  }
};

void run_cart(Problem &P, const airt_cart_opts &o, const double *d_b, const double *d_x0,
              const int64_t *K, int64_t nK, double *d_X, double *resn_host, airt_info *info);
void run_art(Problem &P, const airt_art_opts &o, const double *d_b, const double *d_x0,
             const int64_t *K, int64_t nK, double *d_X, double *resn_host, airt_info *info);
double estimate_rho(Problem &P, const double *dM, const double *dD, double tol, int maxit);
// Custom weights: dM / dD are device diagonals, or full column-major matrices
// when mfull / dfull; nullptr is the identity.
double estimate_rho_custom(Problem &P, const double *dM, bool mfull, const double *dD, bool dfull,
                           double tol, int maxit);
void export_csc(Problem &P, uint64_t *jc, uint64_t *ir, double *pr);
void row_sums_sq(Problem &P, double *out);

// Batched independent problems (batch.cu).
struct Batch;
Batch *batch_build(int ninst, const int *N, const int *nA, const int *p, const double *cos_t,
                   const double *sin_t, const double *offsets);
void batch_destroy(Batch *B);
Problem &batch_problem(Batch &B);
int batch_ninst(const Batch &B);
const int64_t *batch_row_off(const Batch &B);
const int64_t *batch_col_off(const Batch &B);
void batch_rho(Batch &B, int method, double tol, int maxit, double *rho_host);
void batch_sirt(Batch &B, int method, const double *lam_host, const double *d_b, int rule,
                const double *taud_host, int ncp_smooth, int64_t kmax, int lbk, double lb, int ubk,
                double ub, const double *d_x0, double *d_x, int64_t *finaliter, int *stoprule,
                double *gpu_ms);
void batch_kaczmarz(Batch &B, const double *d_b, int64_t sweeps, double lam, int lbk, double lb,
                    int ubk, double ub, double *d_x, double *gpu_ms);
void batch_backproject(Batch &B, int method, const double *d_b, double *d_x, double *gpu_ms);
// fbp.cu: out = col_scale (or scale) * the circular convolution of every
// nr-sample column of in with the order-entry kernel h, cropped to nr
void fbp_filter(const double *d_in, double *d_out, int nr, int64_t ncols, const double *d_h,
                int order, const double *d_col_scale, double scale, cudaStream_t s);

// Exclusive scan of counts[0..n) into offs[0..n] (offs[n] = total), device.
void exclusive_scan_i64(const int64_t *counts, int64_t *offs, int64_t n, cudaStream_t s);

}  // namespace airt

// ------------------------------------------------------------ device helpers
__device__ __forceinline__ double warp_sum(double v, unsigned mask = 0xffffffffu) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o);
  return v;
}

template <int LANES>
__device__ __forceinline__ double group_sum(double v) {
#pragma unroll
  for (int o = LANES / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o, LANES);
  return v;
}

// Block-wide sum of one double per thread; result valid in thread 0.
template <int THREADS>
__device__ __forceinline__ double block_sum(double v) {
  __shared__ double sh[THREADS / 32];
  v = warp_sum(v);
  int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = v;
  __syncthreads();
  double t = 0.0;
  if (w == 0) {
    t = (l < THREADS / 32) ? sh[l] : 0.0;
    t = warp_sum(t);
  }
  __syncthreads();
  return t;
}
