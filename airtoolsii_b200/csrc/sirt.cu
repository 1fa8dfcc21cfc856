// SIRT iteration on the GPU:  x <- P_C(x + lambda_k * D .* A'*(M .* (b - A*x)))
// (sirt/sirt.m:198-261) with the stopping rules of
// auxil/check_stoprules.m:54-94,153-161 evaluated on the device.
//
// Per iteration k the stream runs
//   bwd : g = A'*(M.*r) over the CSC (gather of the FP32 copy of M.*r),
//         fused with x += lambda*D.*g, the box projection (sirt.m:232-237),
//         the FP32 copy of x for the next gather and the save of x into X
//         when k is in K;
//   fwd : r = b - A*x over the CSR (gather of the FP32 copy of x), fused
//         with M.*r (FP32 copy for the next gather) and the FP64 sums
//         ||r||^2, r'*M*r and, for ME, the previous-residual products;
//   ctrl: one thread applies the stopping rule to the sums, records
//         ||r_k|| and the relaxpar used, and selects the next relaxpar.
// Kernels read the device stop flag first and return at once after a stop,
// so the host can enqueue iterations in chunks and poll the flag lazily.
//
// Precision: matrix values and the two gathered vectors are FP32; products
// are accumulated in FP64; x, r, b, M, D and all reductions are FP64.
#include <cmath>

#include "common.cuh"
#include "spmv.cuh"
#include "stream.cuh"
#include "ncp.cuh"
#include "trace.cuh"

namespace airt {

void mf_backproject_f32(Problem &P, const float *u, double *g64, const int *stop_flag);

namespace {

constexpr int kThreads = 256;

struct FwdOut {
  const double *b;
  const double *M;
  float *mr32;
  double *rprev;  // ME only
  SirtState *st;
};

struct Acc4 {
  double r2 = 0, rmr = 0, p2 = 0, pr = 0;
};

template <bool ME>
__device__ __forceinline__ void resid_row_pre(int64_t i, double s, const FwdOut &o, Acc4 &a, double bi,
                                              double Mi) {
  const double r = bi - s;
  const double mr = Mi * r;
  o.mr32[i] = (float)mr;
  a.r2 += r * r;
  a.rmr += r * mr;
  if (ME) {
    const double p = o.rprev[i];
    a.p2 += p * p;
    a.pr += p * (p + r);
    o.rprev[i] = r;
  }
}

template <bool ME>
__device__ __forceinline__ void resid_row(int64_t i, double s, const FwdOut &o, Acc4 &a) {
  const double r = o.b[i] - s;
  const double mr = o.M[i] * r;
  o.mr32[i] = (float)mr;
  a.r2 += r * r;
  a.rmr += r * mr;
  if (ME) {
    const double p = o.rprev[i];
    a.p2 += p * p;
    a.pr += p * (p + r);
    o.rprev[i] = r;
  }
}

template <bool ME>
__device__ __forceinline__ void flush(SirtState *st, Acc4 &a) {
  double r2 = block_sum<kThreads>(a.r2);
  double rmr = block_sum<kThreads>(a.rmr);
  double p2 = 0, pr = 0;
  if (ME) {
    p2 = block_sum<kThreads>(a.p2);
    pr = block_sum<kThreads>(a.pr);
  }
  if (threadIdx.x == 0) {
    atomicAdd(&st->acc[0], r2);
    atomicAdd(&st->acc[1], rmr);
    if (ME) {
      atomicAdd(&st->acc[2], p2);
      atomicAdd(&st->acc[3], pr);
    }
  }
}

__device__ __forceinline__ bool stopped(const SirtState *st) {
  return *(volatile const int *)&st->stop != 0;
}

template <int LANES, bool ME>
__global__ void __launch_bounds__(kThreads, 4)
    k_sirt_fwd(int64_t m, const int64_t *__restrict__ rp, const int *__restrict__ ci,
               const float *__restrict__ rv, const float *__restrict__ x32, FwdOut o) {
  if (stopped(o.st)) return;
  Acc4 a;
  struct BM {
    double b, m;
  };
  for_each_segment_vpre<LANES>(
      m, rp, ci, rv, x32, [&](int64_t i) { return BM{o.b[i], o.M[i]}; },
      [&](int64_t i, double s, bool lead, BM pv) {
        if (lead) resid_row_pre<ME>(i, s, o, a, pv.b, pv.m);
      });
  flush<ME>(o.st, a);
}

// Streamed variants (stream.cuh): same epilogues, tiles of the CSR / CSC
// brought into shared memory by bulk-async copies.
template <bool ME>
__global__ void __launch_bounds__(kStreamThreads, kStreamCtasPerSm)
    k_sirt_fwd_stream(StreamArgs sa, FwdOut o) {
  if (stopped(o.st)) return;
  Acc4 a;
  stream_segments(sa, [&](int64_t i, double s, bool lead) {
    if (lead) resid_row<ME>(i, s, o, a);
  });
  flush<ME>(o.st, a);
}

// 12 resident 64-thread blocks per SM (80 registers, 40-90 bytes of spills):
// the tracer is issue and latency bound, and 24 warps per SM ran C2 3 %
// faster than the 20 that 96 registers allow.
template <bool ME>
__global__ void __launch_bounds__(64, 12)
    k_sirt_fwd_mf(RayGeom g, int64_t nrays, bool excl, const float *__restrict__ x32, FwdOut o) {
  if (stopped(o.st)) return;
  Acc4 a;
  const int64_t nn = (int64_t)g.N * g.N;
  // two adjacent threads per ray, each tracing one half (row_entries_part);
  // the pair adds its halves by a shuffle, every lane runs every trip
  const int part = threadIdx.x & 1;
  const int64_t np = ((int64_t)gridDim.x * blockDim.x) >> 1;
  const int64_t trips = (nrays + np - 1) / np;
  for (int64_t t = 0, r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 1; t < trips; ++t, r += np) {
    double acc = 0.0;
    if (r < nrays)
      row_entries_part(g, r, excl, part, [&](int col, double v) {
        if (col >= 0 && col < nn) acc = fma((double)(float)v, (double)x32[col], acc);
      });
    acc += __shfl_xor_sync(0xffffffffu, acc, 1);
    if (r < nrays && part == 0) resid_row<ME>(r, acc, o, a);
  }
  // warp sums (no block barrier: a warp whose rays are short leaves at once)
  double r2 = warp_sum(a.r2), rmr = warp_sum(a.rmr), p2 = 0, pr = 0;
  if (ME) {
    p2 = warp_sum(a.p2);
    pr = warp_sum(a.pr);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&o.st->acc[0], r2);
    atomicAdd(&o.st->acc[1], rmr);
    if (ME) {
      atomicAdd(&o.st->acc[2], p2);
      atomicAdd(&o.st->acc[3], pr);
    }
  }
}

struct UpdArgs {
  const double *D;
  double *x64;
  float *x32;
  int lbk, ubk;
  double lb, ub;
  const double *lbv, *ubv;
  double *X;
  int64_t n;
  const int *save_slot;
  SirtState *st;
  double *g64;
};

__device__ __forceinline__ void update_x(int64_t j, double g, double lam, const UpdArgs &u, int slot) {
  double x = u.x64[j] + lam * (u.D[j] * g);
  if (u.lbk == AIRT_BOUND_SCALAR) x = fmax(x, u.lb);
  else if (u.lbk == AIRT_BOUND_VECTOR) x = fmax(x, u.lbv[j]);
  if (u.ubk == AIRT_BOUND_SCALAR) x = fmin(x, u.ub);
  else if (u.ubk == AIRT_BOUND_VECTOR) x = fmin(x, u.ubv[j]);
  u.x64[j] = x;
  u.x32[j] = (float)x;
  if (slot >= 0) u.X[(int64_t)slot * u.n + j] = x;
}

// update_x with x64[j] and D[j] already loaded.
__device__ __forceinline__ void update_x_pre(int64_t j, double g, double lam, const UpdArgs &u, int slot,
                                             double x0, double dj) {
  double x = x0 + lam * (dj * g);
  if (u.lbk == AIRT_BOUND_SCALAR) x = fmax(x, u.lb);
  else if (u.lbk == AIRT_BOUND_VECTOR) x = fmax(x, u.lbv[j]);
  if (u.ubk == AIRT_BOUND_SCALAR) x = fmin(x, u.ub);
  else if (u.ubk == AIRT_BOUND_VECTOR) x = fmin(x, u.ubv[j]);
  u.x64[j] = x;
  u.x32[j] = (float)x;
  if (slot >= 0) u.X[(int64_t)slot * u.n + j] = x;
}

// MODE 0: fused update with st->lam_cur.  MODE 1: line-search pass that
// stores g and accumulates sum(D.*g.^2) (sirt.m:219-222).
template <int LANES, int MODE>
__global__ void __launch_bounds__(kThreads, 4)
    k_sirt_bwd(int64_t n, const int64_t *__restrict__ cp, const int *__restrict__ ri,
               const float *__restrict__ cv, const float *__restrict__ mr32, UpdArgs u) {
  if (stopped(u.st)) return;
  const int it = u.st->iter;
  const int slot = u.save_slot[it];
  const double lam = u.st->lam_cur;
  double a4 = 0;
  struct XD {
    double x, d;
  };
  for_each_segment_vpre<LANES>(
      n, cp, ri, cv, mr32, [&](int64_t j) { return XD{MODE == 0 ? u.x64[j] : 0.0, u.D[j]}; },
      [&](int64_t j, double g, bool lead, XD pv) {
        if (!lead) return;
        if (MODE == 0) {
          update_x_pre(j, g, lam, u, slot, pv.x, pv.d);
        } else {
          u.g64[j] = g;
          a4 += pv.d * (g * g);
        }
      });
  if (MODE == 1) {
    a4 = block_sum<kThreads>(a4);
    if (threadIdx.x == 0) atomicAdd(&u.st->acc[4], a4);
  }
}

template <int MODE>
__global__ void __launch_bounds__(kStreamThreads, kStreamCtasPerSm)
    k_sirt_bwd_stream(StreamArgs sa, UpdArgs u) {
  if (stopped(u.st)) return;
  const int it = u.st->iter;
  const int slot = u.save_slot[it];
  const double lam = u.st->lam_cur;
  double a4 = 0;
  stream_segments(sa, [&](int64_t j, double g, bool lead) {
    if (!lead) return;
    if (MODE == 0) {
      update_x(j, g, lam, u, slot);
    } else {
      u.g64[j] = g;
      a4 += u.D[j] * (g * g);
    }
  });
  if (MODE == 1) {
    a4 = block_sum<kStreamThreads>(a4);
    if (threadIdx.x == 0) atomicAdd(&u.st->acc[4], a4);
  }
}

// Elementwise update from a stored g (line search and matrix-free paths).
template <bool LINE>
__global__ void __launch_bounds__(kThreads) k_sirt_update(UpdArgs u) {
  if (stopped(u.st)) return;
  const int it = u.st->iter;
  const int slot = u.save_slot[it];
  double lam;
  if (LINE) {
    lam = u.st->rmr_prev / u.st->acc[4];
  } else {
    lam = u.st->lam_cur;
  }
  if (LINE && blockIdx.x == 0 && threadIdx.x == 0) u.st->lam_cur = lam;
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < u.n;
       j += (int64_t)gridDim.x * blockDim.x)
    update_x(j, u.g64[j], lam, u, slot);
}

// sum(D .* g.^2) for the line search on the matrix-free path.
__global__ void __launch_bounds__(kThreads) k_dg2(int64_t n, const double *__restrict__ D,
                                                   const double *__restrict__ g, SirtState *st) {
  if (stopped(st)) return;
  double a = 0;
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n;
       j += (int64_t)gridDim.x * blockDim.x)
    a += D[j] * (g[j] * g[j]);
  a = block_sum<kThreads>(a);
  if (threadIdx.x == 0) atomicAdd(&st->acc[4], a);
}

// ---- custom weights given as full matrices (get_mfun_dfun.m:252-307,
// Mflag/Dflag = 2): M*r and D*g are dense FP64 products over the caller's
// column-major matrix.  A block of 256 threads owns 32 consecutive rows;
// thread (row lane l, phase c) sums columns j = c, c+8, ... of its row (the
// 32 lanes of a warp read 256 contiguous bytes of one column and share the
// broadcast v[j]), and the 8 phase sums are added in a fixed order, so the
// product repeats bit for bit.
constexpr int kGemvRows = 32, kGemvPhases = 8;

__device__ __forceinline__ double dense_row(int64_t k, const double *__restrict__ W,
                                            const double *__restrict__ v, int64_t row,
                                            double (*part)[kGemvRows]) {
  const int l = threadIdx.x % kGemvRows, c = threadIdx.x / kGemvRows;
  double a0 = 0.0, a1 = 0.0;
  if (row < k) {
    const double *__restrict__ w = W + row;
    int64_t j = c;
    for (; j + kGemvPhases < k; j += 2 * kGemvPhases) {
      a0 = fma(w[j * k], v[j], a0);
      a1 = fma(w[(j + kGemvPhases) * k], v[j + kGemvPhases], a1);
    }
    if (j < k) a0 = fma(w[j * k], v[j], a0);
  }
  part[c][l] = a0 + a1;
  __syncthreads();
  double y = 0.0;
  if (c == 0)
    for (int q = 0; q < kGemvPhases; ++q) y += part[q][l];
  return y;  // valid on the phase-0 threads (threadIdx.x < 32)
}

// y = W*v (rho estimation).
__global__ void __launch_bounds__(256) k_dense_apply(int64_t k, const double *__restrict__ W,
                                                     const double *__restrict__ v,
                                                     double *__restrict__ y) {
  __shared__ double part[kGemvPhases][kGemvRows];
  const int64_t row = blockIdx.x * (int64_t)kGemvRows + threadIdx.x % kGemvRows;
  const double r = dense_row(k, W, v, row, part);
  if (threadIdx.x < kGemvRows && row < k) y[row] = r;
}

// M*r with M full (r = the residual kept by the forward pass): the FP32 copy
// for the transpose gather, and r'*M*r into acc[1] (sirt.m:221).
__global__ void __launch_bounds__(256) k_dense_M(int64_t m, const double *__restrict__ Mf,
                                                 const double *__restrict__ r,
                                                 float *__restrict__ mr32, SirtState *st) {
  if (stopped(st)) return;
  __shared__ double part[kGemvPhases][kGemvRows];
  const int64_t row = blockIdx.x * (int64_t)kGemvRows + threadIdx.x % kGemvRows;
  const double y = dense_row(m, Mf, r, row, part);
  if (threadIdx.x < kGemvRows) {
    double a = 0.0;
    if (row < m) {
      mr32[row] = (float)y;
      a = r[row] * y;
    }
    a = group_sum<32>(a);
    if (threadIdx.x == 0) atomicAdd(&st->acc[1], a);
  }
}

// x += lam * (D*g) with D full (sirt.m:229), then the box projection, the
// FP32 copy and the save of x; LINE takes the line-search relaxpar.
template <bool LINE>
__global__ void __launch_bounds__(256) k_dense_D_update(const double *__restrict__ Df,
                                                        const double *__restrict__ g, UpdArgs u) {
  if (stopped(u.st)) return;
  __shared__ double part[kGemvPhases][kGemvRows];
  const int it = u.st->iter;
  const int slot = u.save_slot[it];
  const double lam = LINE ? u.st->rmr_prev / u.st->acc[4] : u.st->lam_cur;
  const int64_t row = blockIdx.x * (int64_t)kGemvRows + threadIdx.x % kGemvRows;
  const double y = dense_row(u.n, Df, g, row, part);
  if (LINE && blockIdx.x == 0 && threadIdx.x == 0) u.st->lam_cur = lam;
  if (threadIdx.x < kGemvRows && row < u.n) update_x_pre(row, y, lam, u, slot, u.x64[row], 1.0);
}

// Column sums of a full column-major D: sum(D*(g.^2)) = sum_j colsum_j g_j^2
// (the line-search denominator of sirt.m:220).
__global__ void k_colsum(int64_t k, const double *__restrict__ W, double *__restrict__ out) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < k;
       j += (int64_t)gridDim.x * blockDim.x) {
    double a = 0.0;
    for (int64_t i = 0; i < k; ++i) a += W[i + j * k];
    out[j] = a;
  }
}

inline unsigned dense_grid(int64_t k) { return (unsigned)((k + kGemvRows - 1) / kGemvRows); }

// Stopping rule of check_stoprules.m on the sums of the residual just
// computed, then the relaxpar of the next iteration (sirt.m:216-226).
__global__ void k_sirt_ctrl(SirtState *st, const SirtParams *p) {
  if (threadIdx.x || blockIdx.x) return;
  if (st->stop) return;
  const int k = st->iter;
  const double nrk = sqrt(st->acc[0]);
  p->resn_hist[k] = nrk;
  p->lam_hist[k] = st->lam_cur;
  bool stop = false;
  int rule = 0;
  const int64_t kmax = p->kmax;
  switch (p->stoprule) {
    case AIRT_STOP_DP:  // check_stoprules.m:56-72
      if (nrk <= p->taudelta || k >= kmax) {
        stop = true;
        rule = (k != kmax) ? 2 : 0;
      }
      break;
    case AIRT_STOP_ME: {  // check_stoprules.m:74-94
      const double np = sqrt(st->acc[2]);
      const double dme = st->acc[3] / 2.0;
      if (k > 0 && dme / np <= p->taudelta) {
        stop = true;
        rule = 3;
      } else if (k >= kmax) {
        stop = true;
        rule = 0;
      }
      break;
    }
    case AIRT_STOP_NCP: {  // check_stoprules.m:97-150
      double sum = 0.0;
      for (int j = 0; j < p->ncp_cols; ++j) sum += p->ncc_col[j];
      const double ncc = sum / p->ncp_cols;
      const int ns = p->ncp_smooth;
      double mx = -INFINITY, mxn = ncc;  // max(dk), max([dk(2:end); ncc]); NaN ignored
      for (int i = 0; i < ns; ++i) mx = fmax(mx, p->dk[i]);
      for (int i = 1; i < ns; ++i) mxn = fmax(mxn, p->dk[i]);
      if (mx < mxn || k >= kmax) {
        stop = true;
        rule = (k != kmax) ? 1 : 0;
      } else {
        for (int i = 0; i + 1 < ns; ++i) p->dk[i] = p->dk[i + 1];
        p->dk[ns - 1] = ncc;
      }
      break;
    }
    default:  // NONE, check_stoprules.m:153-161
      if (k >= kmax) stop = true;
  }
  st->rmr_prev = st->acc[1];
  for (int q = 0; q < 6; ++q) st->acc[q] = 0.0;
  if (stop) {
    st->stop = 1;
    st->stoprule = rule;
    st->finaliter = k;
    st->lam_last = st->lam_cur;
  } else {
    const int kn = k + 1;
    if (p->relax_kind == AIRT_RELAX_CONST) st->lam_cur = p->relaxpar;
    else if (p->relax_kind == AIRT_RELAX_TABLE) st->lam_cur = p->relax_table[kn - 1];
    st->iter = kn;
  }
}

__global__ void k_to_f32(int64_t n, const double *__restrict__ a, float *__restrict__ b) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}

__global__ void k_copy(int64_t n, const double *__restrict__ a, double *__restrict__ b) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    b[i] = a[i];
}

// ---------------------------------------------------------------- launchers
StreamArgs stream_args(Problem &P, bool rows, const float *gvec) {
  StreamArgs a;
  a.nseg = rows ? P.m : P.n;
  a.ptr = rows ? P.rp.p : P.cp.p;
  a.idx = rows ? P.ci.p : P.ri.p;
  a.val = rows ? P.rv.p : P.cv.p;
  a.gvec = gvec;
  a.tile_seg = rows ? P.rtiles.p : P.ctiles.p;
  a.ntiles = rows ? P.nrtiles : P.nctiles;
  a.err = P.err.p;
  return a;
}

template <class K>
unsigned stream_grid(K kernel, int ntiles) {
  static bool attr = false;
  (void)attr;
  AIRT_CHECK_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)stream_smem_bytes()));
  int g = kStreamCtasPerSm * num_sms();
  return (unsigned)(ntiles < g ? ntiles : g);
}

#define AIRT_STREAM_LAUNCH(KERNEL, NT, ...)                                              \
  do {                                                                                  \
    auto kfn = KERNEL;                                                                  \
    const unsigned g_ = stream_grid(kfn, NT);                                           \
    kfn<<<g_, kStreamThreads, stream_smem_bytes(), s>>>(__VA_ARGS__);                   \
  } while (0)

template <bool ME>
void launch_fwd_t(Problem &P, const FwdOut &o) {
  cudaStream_t s = P.stream;
  if (P.spmv_kind == 1 && P.stream_ok && !P.matrix_free) {
    const StreamArgs sa = stream_args(P, true, P.x32.p);
    AIRT_STREAM_LAUNCH((k_sirt_fwd_stream<ME>), sa.ntiles, sa, o);
    return;
  }
  if (P.matrix_free) {
    k_sirt_fwd_mf<ME><<<grid_for(2 * P.m, 64, 32), 64, 0, s>>>(P.geom(), P.m,
                                                              P.geo_kind == GEO_PARALLEL,
                                                              P.x32.p, o);
    return;
  }
  const int L = vec_lanes_for(P.nnz, P.m);
  const unsigned g = grid_for(P.m * L, kThreads, 4);
  switch (L) {
    case 8: k_sirt_fwd<8, ME><<<g, kThreads, 0, s>>>(P.m, P.rp.p, P.ci.p, P.rv.p, P.x32.p, o); break;
    case 4: k_sirt_fwd<4, ME><<<g, kThreads, 0, s>>>(P.m, P.rp.p, P.ci.p, P.rv.p, P.x32.p, o); break;
    default: k_sirt_fwd<2, ME><<<g, kThreads, 0, s>>>(P.m, P.rp.p, P.ci.p, P.rv.p, P.x32.p, o); break;
  }
}

void launch_fwd(Problem &P, const FwdOut &o, bool me) {
  cudaEvent_t e0 = nullptr;
  prof_begin(P, 0, &e0);
  if (me) launch_fwd_t<true>(P, o);
  else launch_fwd_t<false>(P, o);
  AIRT_LAUNCH_CHECK();
  prof_end(P, 0, e0);
}

template <int MODE>
void launch_bwd_t(Problem &P, const UpdArgs &u) {
  cudaStream_t s = P.stream;
  if (P.spmv_kind == 1 && P.stream_ok) {
    const StreamArgs sa = stream_args(P, false, P.mr32.p);
    AIRT_STREAM_LAUNCH((k_sirt_bwd_stream<MODE>), sa.ntiles, sa, u);
    return;
  }
  const int L = vec_lanes_for(P.nnz, P.n);
  const unsigned g = grid_for(P.n * L, kThreads, 4);
  switch (L) {
    case 8: k_sirt_bwd<8, MODE><<<g, kThreads, 0, s>>>(P.n, P.cp.p, P.ri.p, P.cv.p, P.mr32.p, u); break;
    case 4: k_sirt_bwd<4, MODE><<<g, kThreads, 0, s>>>(P.n, P.cp.p, P.ri.p, P.cv.p, P.mr32.p, u); break;
    default: k_sirt_bwd<2, MODE><<<g, kThreads, 0, s>>>(P.n, P.cp.p, P.ri.p, P.cv.p, P.mr32.p, u); break;
  }
}

void launch_bwd(Problem &P, const UpdArgs &u, int relax_kind, const double *Dfull) {
  cudaStream_t s = P.stream;
  cudaEvent_t e0 = nullptr;
  prof_begin(P, 1, &e0);
  const unsigned ge = grid_for(P.n, kThreads);
  const bool line = relax_kind == AIRT_RELAX_LINE;
  if (Dfull) {
    // g = A'*(M.*r) kept in g64 with sum(colsum(D).*g.^2), then the dense update
    UpdArgs ul = u;
    ul.D = P.Dcol.p;
    if (P.matrix_free) {
      mf_backproject_f32(P, P.mr32.p, P.g64.p, &P.state.p->stop);
      if (line) k_dg2<<<ge, kThreads, 0, s>>>(P.n, P.Dcol.p, P.g64.p, P.state.p);
    } else {
      launch_bwd_t<1>(P, ul);
    }
    if (line) k_dense_D_update<true><<<dense_grid(P.n), 256, 0, s>>>(Dfull, P.g64.p, u);
    else k_dense_D_update<false><<<dense_grid(P.n), 256, 0, s>>>(Dfull, P.g64.p, u);
  } else if (P.matrix_free) {
    mf_backproject_f32(P, P.mr32.p, P.g64.p, &P.state.p->stop);
    if (relax_kind == AIRT_RELAX_LINE) {
      k_dg2<<<ge, kThreads, 0, s>>>(P.n, P.D.p, P.g64.p, P.state.p);
      k_sirt_update<true><<<ge, kThreads, 0, s>>>(u);
    } else {
      k_sirt_update<false><<<ge, kThreads, 0, s>>>(u);
    }
  } else if (relax_kind == AIRT_RELAX_LINE) {
    launch_bwd_t<1>(P, u);
    k_sirt_update<true><<<ge, kThreads, 0, s>>>(u);
  } else {
    launch_bwd_t<0>(P, u);
  }
  AIRT_LAUNCH_CHECK();
  prof_end(P, 1, e0);
}

}  // namespace

void run_sirt(Problem &P, const airt_sirt_opts &o, const double *d_b, const double *d_x0,
              const int64_t *K, int64_t nK, double *d_X, double *resn_host, airt_info *info) {
  cudaStream_t s = P.stream;
  const int64_t m = P.m, n = P.n;
  AIRT_REQUIRE(nK >= 1 && K, "Max no. of iterations must ALWAYS be specified.");
  for (int64_t l = 1; l < nK; ++l)
    AIRT_REQUIRE(K[l] > K[l - 1], "Elements of K must be strictly increasing.");
  AIRT_REQUIRE(o.kmax == K[nK - 1], "kmax must equal K(end)");
  AIRT_REQUIRE(o.kmax >= 0 && o.kmax < (int64_t)INT32_MAX, "kmax out of range");
  AIRT_REQUIRE(K[0] >= 0, "iteration numbers must be nonnegative");
  AIRT_REQUIRE(o.stoprule == AIRT_STOP_NONE || o.stoprule == AIRT_STOP_DP ||
                   o.stoprule == AIRT_STOP_ME || o.stoprule == AIRT_STOP_NCP,
               "The chosen stopping rule is not valid.");
  const bool ncp = o.stoprule == AIRT_STOP_NCP;
  if (ncp) {
    AIRT_REQUIRE(o.ncp_rows >= 2 && o.ncp_cols >= 1 && (int64_t)o.ncp_rows * o.ncp_cols == m,
                 "NCP: res_dims must multiply to the number of rows of A");
    AIRT_REQUIRE(o.ncp_smooth >= 1 && o.ncp_smooth <= 4096, "NCP: ncp_smooth must be in 1..4096");
  }
  AIRT_REQUIRE(o.relax_kind >= AIRT_RELAX_CONST && o.relax_kind <= AIRT_RELAX_TABLE,
               "invalid relaxation strategy");
  AIRT_REQUIRE(o.relax_kind != AIRT_RELAX_TABLE || o.relax_table || o.kmax == 0,
               "relax_table required");
  const int64_t kmax = o.kmax;
  // NCP and a full custom M need the residual itself: the ME variant of the
  // forward kernel keeps it
  const bool me = o.stoprule == AIRT_STOP_ME || ncp || (o.method == AIRT_CUSTOM && o.M && o.M_full);

  cudaEvent_t t0, t1;
  AIRT_CHECK_CUDA(cudaEventCreate(&t0));
  AIRT_CHECK_CUDA(cudaEventCreate(&t1));
  AIRT_CHECK_CUDA(cudaEventRecord(t0, s));

  P.err.ensure(1);
  AIRT_CHECK_CUDA(cudaMemsetAsync(P.err.p, 0, sizeof(int), s));

  // weights (get_mfun_dfun.m)
  P.M.ensure(m);
  P.D.ensure(n);
  const bool mfull = o.method == AIRT_CUSTOM && o.M && o.M_full;
  const bool dfull = o.method == AIRT_CUSTOM && o.D && o.D_full;
  if (o.method == AIRT_CUSTOM) {
    AIRT_REQUIRE(!mfull || (double)m * (double)m <= 4e9,
                 "a full custom M of %lld x %lld does not fit the device", (long long)m,
                 (long long)m);
    AIRT_REQUIRE(!dfull || (double)n * (double)n <= 4e9,
                 "a full custom D of %lld x %lld does not fit the device", (long long)n,
                 (long long)n);
    std::vector<double> fill;
    if (mfull) {
      // the forward pass keeps r and adds nothing to r'*M*r (M diagonal 0);
      // k_dense_M forms M*r and r'*M*r
      P.Mfull.upload(o.M, (size_t)m * m, s);
      fill.assign(m, 0.0);
      P.M.upload(fill.data(), m, s);
    } else if (o.M) {
      P.M.upload(o.M, m, s);
    } else {
      fill.assign(m, 1.0);
      P.M.upload(fill.data(), m, s);
    }
    if (dfull) {
      P.Dfull.upload(o.D, (size_t)n * n, s);
      P.Dcol.ensure(n);
      k_colsum<<<grid_for(n, kThreads), kThreads, 0, s>>>(n, P.Dfull.p, P.Dcol.p);
      AIRT_LAUNCH_CHECK();
      fill.assign(n, 1.0);
      P.D.upload(fill.data(), n, s);
    } else if (o.D) {
      P.D.upload(o.D, n, s);
    } else {
      fill.assign(n, 1.0);
      P.D.upload(fill.data(), n, s);
    }
    AIRT_CHECK_CUDA(cudaStreamSynchronize(s));
  } else {
    compute_weights(P, o.method, P.M.p, P.D.p);
  }

  // vectors
  P.x64.ensure(n);
  P.x32.ensure(n);
  P.mr32.ensure(m);
  if (me) P.rprev.ensure(m);
  if (o.relax_kind == AIRT_RELAX_LINE || P.matrix_free || dfull) P.g64.ensure(n);
  if (d_x0)
    k_copy<<<grid_for(n, kThreads), kThreads, 0, s>>>(n, d_x0, P.x64.p);
  else
    AIRT_CHECK_CUDA(cudaMemsetAsync(P.x64.p, 0, n * sizeof(double), s));
  k_to_f32<<<grid_for(n, kThreads), kThreads, 0, s>>>(n, P.x64.p, P.x32.p);
  AIRT_LAUNCH_CHECK();
  if (me) AIRT_CHECK_CUDA(cudaMemsetAsync(P.rprev.p, 0, m * sizeof(double), s));
  if (o.lb_kind == AIRT_BOUND_VECTOR) {
    AIRT_REQUIRE(o.lbv, "lbound vector missing");
    P.lbv.upload(o.lbv, n, s);
  }
  if (o.ub_kind == AIRT_BOUND_VECTOR) {
    AIRT_REQUIRE(o.ubv, "ubound vector missing");
    P.ubv.upload(o.ubv, n, s);
  }
  if (o.relax_kind == AIRT_RELAX_TABLE && kmax > 0) P.table.upload(o.relax_table, kmax, s);
  std::vector<int> slots(kmax + 1, -1);
  for (int64_t l = 0; l < nK; ++l)
    if (K[l] >= 1 && K[l] <= kmax) slots[K[l]] = (int)l;
  P.save_slot.upload(slots.data(), kmax + 1, s);
  P.resn.ensure(kmax + 1);
  P.lamh.ensure(kmax + 1);

  SirtState st0{};
  st0.lam_cur = (o.relax_kind == AIRT_RELAX_CONST) ? o.relaxpar : NAN;
  P.state.upload(&st0, 1, s);
  SirtParams prm{};
  prm.kmax = kmax;
  prm.stoprule = o.stoprule;
  prm.taudelta = o.taudelta;
  prm.relax_kind = o.relax_kind;
  prm.relaxpar = o.relaxpar;
  prm.relax_table = P.table.p;
  prm.resn_hist = P.resn.p;
  prm.lam_hist = P.lamh.p;
  int ncp_q = 0;
  if (ncp) {
    const int L = o.ncp_rows;
    ncp_q = L / 2;
    if (P.ncp_len != L) {
      const std::vector<double> tw = ncp_twiddles(L);
      P.ncp_tw.upload(tw.data(), tw.size(), s);
      P.ncp_len = L;
    }
    P.ncp_pk.ensure((size_t)o.ncp_cols * ncp_q);
    P.ncp_col.ensure(o.ncp_cols);
    const std::vector<double> dk0(o.ncp_smooth, INFINITY);
    P.ncp_dk.upload(dk0.data(), dk0.size(), s);
    prm.ncc_col = P.ncp_col.p;
    prm.dk = P.ncp_dk.p;
    prm.ncp_cols = o.ncp_cols;
    prm.ncp_smooth = o.ncp_smooth;
  }
  P.params.upload(&prm, 1, s);


  FwdOut fo{d_b, P.M.p, P.mr32.p, me ? P.rprev.p : nullptr, P.state.p};
  UpdArgs ua{};
  ua.D = P.D.p;
  ua.x64 = P.x64.p;
  ua.x32 = P.x32.p;
  ua.lbk = o.lb_kind;
  ua.ubk = o.ub_kind;
  ua.lb = o.lb;
  ua.ub = o.ub;
  ua.lbv = P.lbv.p;
  ua.ubv = P.ubv.p;
  ua.X = d_X;
  ua.n = n;
  ua.save_slot = P.save_slot.p;
  ua.st = P.state.p;
  ua.g64 = P.g64.p;

  // forward pass, and with NCP the periodogram of the new residual
  const double *Dfull = dfull ? P.Dfull.p : nullptr;
  auto fwd = [&]() {
    launch_fwd(P, fo, me);
    if (mfull) {
      k_dense_M<<<dense_grid(m), 256, 0, s>>>(m, P.Mfull.p, P.rprev.p, P.mr32.p, P.state.p);
      AIRT_LAUNCH_CHECK();
    }
    if (ncp) {
      k_ncp_power<<<dim3(o.ncp_cols, (ncp_q + 255) / 256), 256, 0, s>>>(o.ncp_rows, ncp_q, P.rprev.p,
                                                                      P.ncp_tw.p, P.ncp_pk.p, &P.state.p->stop);
      k_ncp_col<<<o.ncp_cols, 256, 0, s>>>(ncp_q, P.ncp_pk.p, P.ncp_col.p, &P.state.p->stop);
      AIRT_LAUNCH_CHECK();
    }
  };
  // initial residual and stop check (sirt.m:153-162)
  fwd();
  k_sirt_ctrl<<<1, 32, 0, s>>>(P.state.p, P.params.p);
  AIRT_LAUNCH_CHECK();

  // main loop, enqueued in chunks; the flag of chunk c is read after chunk
  // c+1 has been queued so the device never idles on the poll
  if (!P.h_state) AIRT_CHECK_CUDA(cudaMallocHost(&P.h_state, 3 * sizeof(SirtState)));
  cudaEvent_t ev[3];
  for (int q = 0; q < 3; ++q)
    AIRT_CHECK_CUDA(cudaEventCreateWithFlags(&ev[q], cudaEventDisableTiming));
  // Without a data-dependent stopping rule every iteration runs: enqueue
  // them all.  Otherwise poll the flag of chunk c once chunk c+2 is queued,
  // so host-side stalls never drain the device queue.
  const bool poll = o.stoprule != AIRT_STOP_NONE;
  const int64_t chunk = 16;
  const int lag = 2;
  int64_t c = 0;
  // A full chunk is captured once as a CUDA graph and replayed: the kernel
  // arguments never change between iterations (all loop state lives in
  // device memory), so one graph serves the whole solve.  With per-launch
  // profiling on, kernels are launched one by one so each gets its events.
  cudaGraphExec_t chunk_graph = nullptr;
  if (!P.profiling && kmax >= chunk) {
    cudaGraph_t g = nullptr;
    AIRT_CHECK_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    for (int64_t j = 0; j < chunk; ++j) {
      launch_bwd(P, ua, o.relax_kind, Dfull);
      fwd();
      k_sirt_ctrl<<<1, 32, 0, s>>>(P.state.p, P.params.p);
    }
    const cudaError_t ec = cudaStreamEndCapture(s, &g);
    if (ec == cudaSuccess && g) {
      if (cudaGraphInstantiate(&chunk_graph, g, 0) != cudaSuccess) chunk_graph = nullptr;
      cudaGraphDestroy(g);
    }
    cudaGetLastError();
  }
  for (int64_t it = 1; it <= kmax; ++c) {
    const int64_t cnt = (kmax - it + 1 < chunk) ? (kmax - it + 1) : chunk;
    if (cnt == chunk && chunk_graph) {
      AIRT_CHECK_CUDA(cudaGraphLaunch(chunk_graph, s));
    } else {
      for (int64_t j = 0; j < cnt; ++j) {
        launch_bwd(P, ua, o.relax_kind, Dfull);
        fwd();
        k_sirt_ctrl<<<1, 32, 0, s>>>(P.state.p, P.params.p);
      }
    }
    AIRT_LAUNCH_CHECK();
    it += cnt;
    if (!poll) continue;
    AIRT_CHECK_CUDA(cudaMemcpyAsync(P.h_state + (c % 3), P.state.p, sizeof(SirtState),
                                    cudaMemcpyDeviceToHost, s));
    AIRT_CHECK_CUDA(cudaEventRecord(ev[c % 3], s));
    if (c >= lag) {
      AIRT_CHECK_CUDA(cudaEventSynchronize(ev[(c - lag) % 3]));
      if (P.h_state[(c - lag) % 3].stop) break;
    }
  }
  AIRT_CHECK_CUDA(cudaMemcpyAsync(P.h_state, P.state.p, sizeof(SirtState), cudaMemcpyDeviceToHost, s));
  AIRT_CHECK_CUDA(cudaStreamSynchronize(s));
  if (chunk_graph) cudaGraphExecDestroy(chunk_graph);
  for (int q = 0; q < 3; ++q) cudaEventDestroy(ev[q]);
  const SirtState st = P.h_state[0];
  int herr = 0;
  AIRT_CHECK_CUDA(cudaMemcpy(&herr, P.err.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (herr) {
    set_error("a bounded device wait gave up (bulk copy did not complete)");
    throw Status{AIRT_ERR_TIMEOUT};
  }
  AIRT_REQUIRE(st.stop, "internal: SIRT loop ended without a stop");

  // X keeps the iterates in K below finaliter plus the final one (sirt.m:270)
  int64_t nsaved = 0;
  if (st.finaliter > 0) {
    int64_t below = 0;
    for (int64_t l = 0; l < nK; ++l)
      if (K[l] < st.finaliter) ++below;
    nsaved = below + 1;
    AIRT_CHECK_CUDA(cudaMemcpyAsync(d_X + below * n, P.x64.p, n * sizeof(double),
                                    cudaMemcpyDeviceToDevice, s));
  }
  AIRT_CHECK_CUDA(cudaEventRecord(t1, s));
  if (resn_host)
    AIRT_CHECK_CUDA(cudaMemcpyAsync(resn_host, P.resn.p, (st.finaliter + 1) * sizeof(double),
                                    cudaMemcpyDeviceToHost, s));
  double lam_final = o.relaxpar;
  if (st.finaliter > 0)
    AIRT_CHECK_CUDA(cudaMemcpyAsync(&lam_final, P.lamh.p + st.finaliter, sizeof(double),
                                    cudaMemcpyDeviceToHost, s));
  AIRT_CHECK_CUDA(cudaStreamSynchronize(s));
  float ms = 0;
  cudaEventElapsedTime(&ms, t0, t1);
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  prof_collect(P);
  if (info) {
    info->stoprule = st.stoprule;
    info->finaliter = st.finaliter;
    info->relaxpar = lam_final;
    info->nsaved = nsaved;
    info->gpu_ms = ms;
  }
}

// ---------------------------------------------------------------- rho
namespace {

__global__ void k_sqrt_vec(int64_t n, const double *__restrict__ a, double *__restrict__ b) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    b[i] = sqrt(a[i] > 0 ? a[i] : 0.0);
}
__global__ void k_mul(int64_t n, const double *__restrict__ a, const double *__restrict__ b,
                      double *__restrict__ c) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    c[i] = a[i] * b[i];
}
__global__ void k_dot2(int64_t n, const double *__restrict__ u, const double *__restrict__ w,
                       double *__restrict__ out) {
  double a = 0, b = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    a += u[i] * w[i];
    b += w[i] * w[i];
  }
  a = block_sum<kThreads>(a);
  b = block_sum<kThreads>(b);
  if (threadIdx.x == 0) {
    atomicAdd(out, a);
    atomicAdd(out + 1, b);
  }
}
// w -= a * x
__global__ void k_axmy(int64_t n, double a, const double *__restrict__ x, double *__restrict__ w) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    w[i] -= a * x[i];
}
__global__ void k_scale_by(int64_t n, double c, const double *__restrict__ w,
                           double *__restrict__ u) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    u[i] = w[i] * c;
}

// Largest eigenvalue of the symmetric tridiagonal matrix with diagonal
// alpha[0..k) and off-diagonal beta[1..k): bisection on the Sturm count
// (the number of eigenvalues below x is the number of negative pivots of
// T - x*I) inside the Gershgorin interval.
double tridiag_max_eig(const std::vector<double> &alpha, const std::vector<double> &beta) {
  const size_t k = alpha.size();
  double lo = INFINITY, hi = -INFINITY;
  for (size_t i = 0; i < k; ++i) {
    const double r = (i > 0 ? std::fabs(beta[i]) : 0.0) + (i + 1 < k ? std::fabs(beta[i + 1]) : 0.0);
    lo = std::fmin(lo, alpha[i] - r);
    hi = std::fmax(hi, alpha[i] + r);
  }
  auto below = [&](double x) {
    size_t cnt = 0;
    double d = 1.0;
    for (size_t i = 0; i < k; ++i) {
      d = alpha[i] - x - (i > 0 ? beta[i] * beta[i] / d : 0.0);
      if (d == 0.0) d = -1e-300;
      if (d < 0) ++cnt;
    }
    return cnt;
  };
  for (int it = 0; it < 200 && hi - lo > 1e-15 * std::fmax(std::fabs(hi), std::fabs(lo)); ++it) {
    const double mid = 0.5 * (lo + hi);
    if (below(mid) >= k) hi = mid;  // every eigenvalue lies below mid
    else lo = mid;
  }
  return hi;
}

}  // namespace

// Largest eigenvalue of D*A'*M*A, through the similar symmetric operator
// S = D^(1/2)*A'*M*A*D^(1/2) (M, D nonnegative), by the Lanczos iteration
// from the normalised ones vector: the largest Ritz value of the
// tridiagonal matrix, stopped once it changes by at most tol (relative)
// after at least five steps, or on an invariant subspace.  Replaces
// eigs(...,'lm',tol=1e-4) of calc_relaxpar.m:91-103; unlike a power
// iteration it does not stall below rho when the top eigenvalues cluster.
double estimate_rho(Problem &P, const double *dM, const double *dD, double tol, int maxit) {
  cudaStream_t s = P.stream;
  const int64_t m = P.m, n = P.n;
  if (n == 0) return 0.0;
  DevBuf<double> sd, v, vprev, t, y, w, red;
  sd.ensure(n);
  v.ensure(n);
  vprev.ensure(n);
  t.ensure(n);
  y.ensure(std::max<int64_t>(m, 1));
  w.ensure(n);
  red.ensure(2);
  const unsigned gn = grid_for(n, kThreads), gm = grid_for(std::max<int64_t>(m, 1), kThreads);
  k_sqrt_vec<<<gn, kThreads, 0, s>>>(n, dD, sd.p);
  std::vector<double> h(n, 1.0 / std::sqrt((double)n));
  v.upload(h.data(), n, s);
  std::vector<double> alpha, beta{0.0};
  double theta = 0.0, prev = 0.0;
  auto dot = [&](const double *a, const double *b) {  // a.b
    AIRT_CHECK_CUDA(cudaMemsetAsync(red.p, 0, 2 * sizeof(double), s));
    k_dot2<<<gn, kThreads, 0, s>>>(n, a, b, red.p);
    AIRT_LAUNCH_CHECK();
    double hr[2];
    AIRT_CHECK_CUDA(cudaMemcpyAsync(hr, red.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    AIRT_CHECK_CUDA(cudaStreamSynchronize(s));
    return hr[0];
  };
  for (int it = 0; it < std::max(maxit, 1); ++it) {
    // w = S v - beta_j v_(j-1)
    k_mul<<<gn, kThreads, 0, s>>>(n, sd.p, v.p, t.p);
    if (m) {
      apply_operator(P, t.p, y.p, 0);
      k_mul<<<gm, kThreads, 0, s>>>(m, dM, y.p, y.p);
      apply_operator(P, y.p, t.p, 1);
    } else {
      AIRT_CHECK_CUDA(cudaMemsetAsync(t.p, 0, n * sizeof(double), s));
    }
    k_mul<<<gn, kThreads, 0, s>>>(n, sd.p, t.p, w.p);
    if (it > 0) k_axmy<<<gn, kThreads, 0, s>>>(n, beta.back(), vprev.p, w.p);
    AIRT_LAUNCH_CHECK();
    const double a = dot(v.p, w.p);
    alpha.push_back(a);
    k_axmy<<<gn, kThreads, 0, s>>>(n, a, v.p, w.p);
    AIRT_LAUNCH_CHECK();
    const double b = std::sqrt(std::fmax(dot(w.p, w.p), 0.0));
    theta = tridiag_max_eig(alpha, beta);
    if (!(b > 1e-14 * std::fmax(std::fabs(theta), 1e-300))) break;  // invariant subspace
    if (it >= 4 && std::fabs(theta - prev) <= tol * std::fabs(theta)) break;
    prev = theta;
    beta.push_back(b);
    std::swap(vprev.p, v.p);
    std::swap(vprev.n, v.n);
    k_scale_by<<<gn, kThreads, 0, s>>>(n, 1.0 / b, w.p, v.p);
    AIRT_LAUNCH_CHECK();
  }
  return theta;
}

// Dominant eigenvalue of T = D*A'*M*A for custom weights that may be full
// matrices (T is then not similar to a symmetric operator built from
// diagonal square roots, so the Lanczos form above does not apply): the
// power iteration v <- T v / ||T v|| from the normalised ones vector with the
// Rayleigh quotient v'*T*v as the estimate, stopped once it changes by at
// most tol (relative) after at least five steps, or after maxit steps.
// Replaces eigs(atma,n,1,'lm') of calc_relaxpar.m:91-103 for these weights.
double estimate_rho_custom(Problem &P, const double *dM, bool mfull, const double *dD, bool dfull,
                           double tol, int maxit) {
  cudaStream_t s = P.stream;
  const int64_t m = P.m, n = P.n;
  if (n == 0) return 0.0;
  DevBuf<double> v, t, y, y2, w, red;
  v.ensure(n);
  t.ensure(n);
  y.ensure(std::max<int64_t>(m, 1));
  y2.ensure(std::max<int64_t>(m, 1));
  w.ensure(n);
  red.ensure(2);
  const unsigned gn = grid_for(n, kThreads), gm = grid_for(std::max<int64_t>(m, 1), kThreads);
  std::vector<double> h(n, 1.0 / std::sqrt((double)n));
  v.upload(h.data(), n, s);
  double theta = 0.0, prev = 0.0;
  for (int it = 0; it < std::max(maxit, 1); ++it) {
    if (m) {
      apply_operator(P, v.p, y.p, 0);
      const double *my = y.p;
      if (dM && mfull) {
        k_dense_apply<<<dense_grid(m), 256, 0, s>>>(m, dM, y.p, y2.p);
        my = y2.p;
      } else if (dM) {
        k_mul<<<gm, kThreads, 0, s>>>(m, dM, y.p, y.p);
      }
      apply_operator(P, my, t.p, 1);
    } else {
      AIRT_CHECK_CUDA(cudaMemsetAsync(t.p, 0, n * sizeof(double), s));
    }
    const double *tw = t.p;
    if (dD && dfull) {
      k_dense_apply<<<dense_grid(n), 256, 0, s>>>(n, dD, t.p, w.p);
      tw = w.p;
    } else if (dD) {
      k_mul<<<gn, kThreads, 0, s>>>(n, dD, t.p, w.p);
      tw = w.p;
    }
    AIRT_LAUNCH_CHECK();
    AIRT_CHECK_CUDA(cudaMemsetAsync(red.p, 0, 2 * sizeof(double), s));
    k_dot2<<<gn, kThreads, 0, s>>>(n, v.p, tw, red.p);  // v'Tv, ||Tv||^2
    AIRT_LAUNCH_CHECK();
    double hr[2];
    AIRT_CHECK_CUDA(cudaMemcpyAsync(hr, red.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    AIRT_CHECK_CUDA(cudaStreamSynchronize(s));
    theta = hr[0];
    const double nrm = std::sqrt(std::fmax(hr[1], 0.0));
    if (!(nrm > 0.0)) break;
    if (it >= 4 && std::fabs(theta - prev) <= tol * std::fabs(theta)) break;
    prev = theta;
    k_scale_by<<<gn, kThreads, 0, s>>>(n, 1.0 / nrm, tw, v.p);
    AIRT_LAUNCH_CHECK();
  }
  return theta;
}

}  // namespace airt
