// Kaczmarz (ART) sweeps on the GPU in the reference's row order
// (art/art.m:227-309).
//
// A sweep is strictly sequential: row step t reads the x that step t-1 wrote.
// Two steps whose rows share no pixel commute exactly, so the order is
// turned into a level schedule: level(t) = 1 + max level of the earlier steps
// that touch one of its pixels.  Steps of one level touch disjoint pixels and
// run concurrently (one warp per step, fixed lane order and shuffle tree, so
// every step computes exactly what it would compute alone); a block barrier
// separates levels.  Each pixel therefore sees the same update sequence, and
// each dot product reads the same values, as in the sequential sweep.
//
// The sweep runs as one cooperative launch over all SMs with one warp per
// step: the steps, sorted by level, are dealt round-robin to every warp of
// the grid, and a step waits only for its predecessors -- the last earlier
// step that touched each of its pixels -- through per-step completion
// stamps in global memory (release store after the step's x writes, acquire
// loads before its gathers).  The chain of levels is the critical path; no
// grid-wide barrier separates levels.  Each wait is bounded: on expiry the
// kernel raises an error flag, every warp leaves, and the host reports
// AIRT_ERR_TIMEOUT.
//
// The whole-vector box projection after every row (art.m:279-284) is
// equivalent to clamping x0 once right after the first row step and the
// row's support after every later step: once x is feasible only the updated
// entries can leave the box.  The first step reads x0 unclamped.
#include <algorithm>
#include <cmath>
#include <numeric>

#include "common.cuh"
#include "ncp.cuh"
#include "spmv.cuh"

namespace airt {

namespace {

struct KaczArgs {
  const int64_t *rp;
  const int *ci;
  const float *rv;
  const double *b;
  const double *nrm;
  double lam;
  const double *lam_tab;  // per step of this sweep, or null
  double *x;
  int lbk, ubk;
  double lb, ub;
  const double *lbv, *ubv;
};

__device__ __forceinline__ double clampv(double v, int64_t j, const KaczArgs &a) {
  if (a.lbk == AIRT_BOUND_SCALAR) v = fmax(v, a.lb);
  else if (a.lbk == AIRT_BOUND_VECTOR) v = fmax(v, a.lbv[j]);
  if (a.ubk == AIRT_BOUND_SCALAR) v = fmin(v, a.ub);
  else if (a.ubk == AIRT_BOUND_VECTOR) v = fmin(v, a.ubv[j]);
  return v;
}

// Test hook: a cycle budget for the bounded waits of the sweep kernel and
// an injected stall (the first step waits for a stamp that no step writes),
// so that a test can make a wait run out.  Defaults: ~2 s, no stall.
long long g_kacz_wait_budget = 4000000000ll;
int g_kacz_inject_stall = 0;

constexpr int kDagCache = 16;  // entries per lane kept in registers (rows <= 512)
// Warps per CTA of the sweep kernel (one CTA per SM) and the pause between
// two polls of an unfinished predecessor (0: none).
#ifndef AIRT_KACZ_WARPS
#define AIRT_KACZ_WARPS 8
#endif
#ifndef AIRT_KACZ_BACKOFF_NS
#define AIRT_KACZ_BACKOFF_NS 0
#endif
constexpr int kDagThreads = 32 * AIRT_KACZ_WARPS;

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u32(unsigned *p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// One Kaczmarz sweep in the level-sorted step order: warp w of the grid
// (consecutive warps on different SMs) runs steps w, w+W, w+2W, ... ; step q
// waits until done[pred] >= stamp for each of its predecessors
// preds[pred_ptr[q] .. pred_ptr[q+1]) (indices into the same order), then
// computes exactly what the sequential sweep computes for its row and
// publishes done[q] = stamp.  The row's indices, values, b and the norm are
// loaded before the wait; x is read through L2 (other SMs wrote it).
__global__ void __launch_bounds__(kDagThreads, 1)
    k_kacz_dag(int nsteps, const int *__restrict__ steps, const int *__restrict__ step_pos,
               const int *__restrict__ pred_ptr, const int *__restrict__ preds, unsigned stamp,
               unsigned *__restrict__ done, int *__restrict__ err, long long budget, int stall,
               KaczArgs a) {
  const int lane = threadIdx.x & 31;
  const int W = gridDim.x * (blockDim.x >> 5);
  const int w = (threadIdx.x >> 5) * gridDim.x + blockIdx.x;
  const bool clamp = a.lbk != AIRT_BOUND_NONE || a.ubk != AIRT_BOUND_NONE;
  for (int q = w; q < nsteps; q += W) {
    const int row = __ldg(steps + q);
    const int64_t s0 = __ldg(a.rp + row), s1 = __ldg(a.rp + row + 1);
    const int64_t e0 = s0 + lane;
    int cj[kDagCache];
    float cv[kDagCache];
#pragma unroll
    for (int u = 0; u < kDagCache; ++u) {
      const int64_t e = e0 + 32 * u;
      cj[u] = e < s1 ? __ldg(a.ci + e) : -1;
      cv[u] = e < s1 ? __ldg(a.rv + e) : 0.f;
    }
    const double bi = __ldg(a.b + row), ni = __ldg(a.nrm + row);
    const double lam = a.lam_tab ? __ldg(a.lam_tab + __ldg(step_pos + q)) : a.lam;
    // wait for the predecessors (each lane polls its share of them)
    const int p0 = __ldg(pred_ptr + q), p1 = __ldg(pred_ptr + q + 1);
    bool ok = true;
    const long long t0 = clock64();
    for (int pi = p0 + lane; ok && pi < p1 + (stall && q == 0 ? 1 : 0); pi += 32) {
      const unsigned *f = pi < p1 ? done + __ldg(preds + pi) : done + q;  // stall: own stamp
      const unsigned want = pi < p1 ? stamp : stamp + 1u;
      while (ld_acquire_u32(f) < want) {
        if (AIRT_KACZ_BACKOFF_NS > 0) __nanosleep(AIRT_KACZ_BACKOFF_NS);
        if (*(volatile int *)err) {
          ok = false;
          break;
        }
        if (clock64() - t0 > budget) {
          atomicExch(err, 1);
          ok = false;
          break;
        }
      }
    }
    if (!__all_sync(0xffffffffu, ok)) return;
    // gathers (through L2) and the dot product in the order of the plain
    // strided loop
    double cx[kDagCache];
#pragma unroll
    for (int u = 0; u < kDagCache; ++u) cx[u] = cj[u] >= 0 ? __ldcg(a.x + cj[u]) : 0.0;
    double acc = 0.0;
#pragma unroll
    for (int u = 0; u < kDagCache; ++u)
      if (cj[u] >= 0) acc = fma((double)cv[u], cx[u], acc);
    for (int64_t e = e0 + 32 * kDagCache; e < s1; e += 32)
      acc = fma((double)__ldg(a.rv + e), __ldcg(a.x + __ldg(a.ci + e)), acc);
    acc = warp_sum(acc);
    const double c = __ddiv_rn(__dmul_rn(lam, __dsub_rn(bi, acc)), ni);
#pragma unroll
    for (int u = 0; u < kDagCache; ++u)
      if (cj[u] >= 0) {
        double v = __dadd_rn(cx[u], __dmul_rn(c, (double)cv[u]));
        if (clamp) v = clampv(v, cj[u], a);
        __stcg(a.x + cj[u], v);
      }
    for (int64_t e = e0 + 32 * kDagCache; e < s1; e += 32) {
      const int j = __ldg(a.ci + e);
      double v = __dadd_rn(__ldcg(a.x + j), __dmul_rn(c, (double)__ldg(a.rv + e)));
      if (clamp) v = clampv(v, j, a);
      __stcg(a.x + j, v);
    }
    __threadfence();
    __syncwarp();
    if (lane == 0) st_release_u32(done + q, stamp);
  }
}

// Clamp x0 everywhere except on the support of the first row, whose step
// must read x0 unclamped (one block).
__global__ void __launch_bounds__(1024)
    k_preclamp(int64_t n, int first_row, double *__restrict__ keep, KaczArgs a) {
  const int64_t s0 = a.rp[first_row], s1 = a.rp[first_row + 1];
  for (int64_t e = s0 + threadIdx.x; e < s1; e += blockDim.x) keep[e - s0] = a.x[a.ci[e]];
  __syncthreads();
  for (int64_t j = threadIdx.x; j < n; j += blockDim.x) a.x[j] = clampv(a.x[j], j, a);
  __syncthreads();
  for (int64_t e = s0 + threadIdx.x; e < s1; e += blockDim.x) a.x[a.ci[e]] = keep[e - s0];
}

// ||b - A*x||^2 into *out; with rout the residual itself is kept (NCP).
template <int LANES>
__global__ void __launch_bounds__(256)
    k_resid_norm(int64_t m, const int64_t *__restrict__ rp, const int *__restrict__ ci,
                 const float *__restrict__ rv, const double *__restrict__ x,
                 const double *__restrict__ b, double *__restrict__ out, double *__restrict__ rout) {
  double a = 0;
  for_each_segment<LANES>(m, rp, ci, rv, x, [&](int64_t i, double s, bool lead) {
    if (lead) {
      const double r = b[i] - s;
      a += r * r;
      if (rout) rout[i] = r;
    }
  });
  a = block_sum<256>(a);
  if (threadIdx.x == 0) atomicAdd(out, a);
}

__global__ void k_rownorm2(int64_t m, const int64_t *__restrict__ rp, const float *__restrict__ rv,
                           double *__restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t i = w; i < m; i += nw) {
    double a = 0;
    for (int64_t q = rp[i] + lane; q < rp[i + 1]; q += 32) {
      const double v = (double)rv[q];
      a += v * v;
    }
    a = warp_sum(a);
    if (lane == 0) out[i] = a;
  }
}

__global__ void k_copy_d(int64_t n, const double *__restrict__ a, double *__restrict__ b) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    b[i] = a[i];
}

using Schedule = ArtSchedule;

// FNV-1a hash of a row order (the key of the cached schedule; never 0).
uint64_t order_key(const int64_t *order, int64_t nsteps) {
  uint64_t h = 1469598103934665603ull ^ (uint64_t)nsteps;
  for (int64_t t = 0; t < nsteps; ++t) {
    h ^= (uint64_t)order[t];
    h *= 1099511628211ull;
  }
  return h ? h : 1;
}

// Level schedule of a row order (see the file comment): steps sorted by
// level (stable), each with the distinct last earlier writers of its pixels
// as predecessors, given as indices into the sorted order.
void build_schedule(const std::vector<int64_t> &hrp, const std::vector<int> &hci,
                    const int64_t *order, int64_t nsteps, int64_t n, Schedule &S,
                    cudaStream_t s) {
  std::vector<int> level(nsteps), last(n, -1), seen(nsteps, -1);
  std::vector<int64_t> tptr(nsteps + 1, 0);
  std::vector<int> tpred;
  int maxlev = -1;
  for (int64_t t = 0; t < nsteps; ++t) {
    const int64_t row = order[t];
    int L = 0;
    for (int64_t e = hrp[row]; e < hrp[row + 1]; ++e) {
      const int w = last[hci[e]];
      if (w >= 0 && seen[w] != (int)t) {
        seen[w] = (int)t;
        tpred.push_back(w);
        L = std::max(L, level[w] + 1);
      }
    }
    tptr[t + 1] = (int64_t)tpred.size();
    level[t] = L;
    for (int64_t e = hrp[row]; e < hrp[row + 1]; ++e) last[hci[e]] = (int)t;
    maxlev = std::max(maxlev, L);
  }
  S.nlev = maxlev + 1;
  S.nsteps = nsteps;
  std::vector<int> ptr(S.nlev + 1, 0), steps(nsteps), pos(nsteps), qof(nsteps);
  for (int64_t t = 0; t < nsteps; ++t) ++ptr[level[t] + 1];
  for (int L = 0; L < S.nlev; ++L) ptr[L + 1] += ptr[L];
  for (int64_t t = 0; t < nsteps; ++t) {
    const int q = ptr[level[t]]++;
    steps[q] = (int)order[t];
    pos[q] = (int)t;
    qof[t] = q;
  }
  std::vector<int> pptr(nsteps + 1, 0), preds(tpred.size());
  for (int64_t q = 0; q < nsteps; ++q) {
    const int t = pos[q];
    pptr[q + 1] = pptr[q] + (int)(tptr[t + 1] - tptr[t]);
  }
  for (int64_t q = 0; q < nsteps; ++q) {
    const int t = pos[q];
    int o = pptr[q];
    for (int64_t k = tptr[t]; k < tptr[t + 1]; ++k) preds[o++] = qof[tpred[k]];
  }
  S.steps.upload(steps.data(), nsteps, s);
  S.pos.upload(pos.data(), nsteps, s);
  S.pred_ptr.upload(pptr.data(), nsteps + 1, s);
  if (preds.empty()) S.preds.ensure(1);
  else S.preds.upload(preds.data(), preds.size(), s);
}

}  // namespace

void run_art(Problem &P, const airt_art_opts &o, const double *d_b, const double *d_x0,
             const int64_t *K, int64_t nK, double *d_X, double *resn_host, airt_info *info) {
  cudaStream_t s = P.stream;
  const int64_t m = P.m, n = P.n;
  AIRT_REQUIRE(!P.matrix_free, "ART needs the stored matrix (row access)");
  AIRT_REQUIRE(nK >= 1 && K, "Max no. of iterations must ALWAYS be specified.");
  for (int64_t l = 1; l < nK; ++l)
    AIRT_REQUIRE(K[l] > K[l - 1], "Elements of K must be strictly increasing.");
  AIRT_REQUIRE(o.kmax == K[nK - 1] && o.kmax >= 0, "kmax must equal K(end)");
  AIRT_REQUIRE(o.stoprule == AIRT_STOP_NONE || o.stoprule == AIRT_STOP_DP || o.stoprule == AIRT_STOP_NCP,
               "ART supports the NONE, DP and NCP stopping rules");
  const bool ncp = o.stoprule == AIRT_STOP_NCP;
  if (ncp) {
    AIRT_REQUIRE(o.ncp_rows >= 2 && o.ncp_cols >= 1 && (int64_t)o.ncp_rows * o.ncp_cols == m,
                 "NCP: res_dims must multiply to the number of rows of A");
    AIRT_REQUIRE(o.ncp_smooth >= 1, "NCP: ncp_smooth must be positive");
  }
  AIRT_REQUIRE(o.damp >= 0, "Damping must be positive");
  AIRT_REQUIRE(m < (int64_t)INT32_MAX, "too many rows for ART");
  const int64_t kmax = o.kmax;

  cudaEvent_t t0, t1;
  AIRT_CHECK_CUDA(cudaEventCreate(&t0));
  AIRT_CHECK_CUDA(cudaEventCreate(&t1));
  AIRT_CHECK_CUDA(cudaEventRecord(t0, s));

  // squared row norms (art.m:161-181) and damping (art.m:206)
  DevBuf<double> nrm;
  nrm.ensure(m);
  k_rownorm2<<<grid_for(m * 32, 256), 256, 0, s>>>(m, P.rp.p, P.rv.p, nrm.p);
  AIRT_LAUNCH_CHECK();
  std::vector<double> hn(m);
  AIRT_CHECK_CUDA(cudaMemcpyAsync(hn.data(), nrm.p, m * sizeof(double), cudaMemcpyDeviceToHost, s));
  AIRT_CHECK_CUDA(cudaStreamSynchronize(s));

  // row order (art.m:183-203)
  std::vector<int64_t> I;
  for (int64_t i = 0; i < m; ++i)
    if (hn[i] > 0) I.push_back(i);
  std::vector<int64_t> order;
  int64_t stride = 0;
  if (o.order_kind == 0) {
    order = I;
  } else if (o.order_kind == 1) {
    order = I;
    order.insert(order.end(), I.rbegin(), I.rend());
  } else {
    AIRT_REQUIRE(o.rows && o.nrows >= 0, "row list missing");
    stride = o.rows_stride;
    const int64_t lists = stride > 0 ? kmax : 1;
    for (int64_t k = 0; k < lists; ++k) {
      for (int64_t t = 0; t < o.nrows; ++t) {
        const int64_t r = o.rows[k * stride + t];
        AIRT_REQUIRE(r >= 0 && r < m, "row index out of range");
        if (hn[r] > 0) order.push_back(r);
      }
    }
  }
  if (o.damp > 0) {
    double mx = 0;
    for (double v : hn) mx = std::max(mx, v);
    for (double &v : hn) v = v + o.damp * mx;
    nrm.upload(hn.data(), m, s);
  }
  const int64_t per_sweep =
      (o.order_kind == 2 && stride > 0) ? (int64_t)order.size() / std::max<int64_t>(kmax, 1)
                                        : (int64_t)order.size();
  AIRT_REQUIRE(o.order_kind != 2 || stride == 0 || (int64_t)order.size() == per_sweep * kmax,
               "each sweep of the row stream must keep the same number of nonzero rows");

  // the schedule of a fixed order is kept in the problem and rebuilt only for
  // a new order; per-sweep orders (a row stream) get one per sweep
  const bool per_sweep_sched = (o.order_kind == 2 && stride > 0);
  Schedule local;
  Schedule &S = per_sweep_sched ? local : P.art_sched;
  const uint64_t key = per_sweep_sched ? 0 : order_key(order.data(), per_sweep);
  const bool need_pattern = per_sweep_sched || S.key != key || S.nsteps != per_sweep;
  // host copy of the sparsity pattern, only when a schedule is built
  std::vector<int64_t> hrp;
  std::vector<int> hci;
  if (need_pattern) {
    hrp.resize(m + 1);
    hci.resize(P.nnz);
    AIRT_CHECK_CUDA(cudaMemcpyAsync(hrp.data(), P.rp.p, (m + 1) * sizeof(int64_t),
                                    cudaMemcpyDeviceToHost, s));
    if (P.nnz)
      AIRT_CHECK_CUDA(cudaMemcpyAsync(hci.data(), P.ci.p, P.nnz * sizeof(int), cudaMemcpyDeviceToHost, s));
    AIRT_CHECK_CUDA(cudaStreamSynchronize(s));
  }
  if (!per_sweep_sched && need_pattern) {
    S.key = 0;
    build_schedule(hrp, hci, order.data(), per_sweep, n, S, s);
    S.key = key;
  }

  // iterate
  P.x64.ensure(n);
  if (d_x0)
    k_copy_d<<<grid_for(n, 256), 256, 0, s>>>(n, d_x0, P.x64.p);
  else
    AIRT_CHECK_CUDA(cudaMemsetAsync(P.x64.p, 0, n * sizeof(double), s));
  if (o.lb_kind == AIRT_BOUND_VECTOR) P.lbv.upload(o.lbv, n, s);
  if (o.ub_kind == AIRT_BOUND_VECTOR) P.ubv.upload(o.ubv, n, s);
  // sweep kernel: completion stamps of the steps, error flag, grid size
  DevBuf<unsigned> done;
  done.ensure(std::max<int64_t>(per_sweep, 1));
  AIRT_CHECK_CUDA(cudaMemsetAsync(done.p, 0, std::max<int64_t>(per_sweep, 1) * sizeof(unsigned), s));
  P.err.ensure(1);
  AIRT_CHECK_CUDA(cudaMemsetAsync(P.err.p, 0, sizeof(int), s));
  int occ = 0;
  AIRT_CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_kacz_dag, kDagThreads, 0));
  AIRT_REQUIRE(occ >= 1, "the Kaczmarz sweep kernel cannot be resident");
  const int dag_grid = num_sms();
  const long long budget = g_kacz_wait_budget;
  const int stall = g_kacz_inject_stall;
  int herr = 0;
  DevBuf<double> tab, red, keep;
  if (o.relax_table && kmax > 0) tab.upload(o.relax_table, kmax * per_sweep, s);
  red.ensure(1);
  keep.ensure(std::max<int64_t>(P.N ? 2 * P.N + 2 : 1, 1));

  KaczArgs a{};
  a.rp = P.rp.p;
  a.ci = P.ci.p;
  a.rv = P.rv.p;
  a.b = d_b;
  a.nrm = nrm.p;
  a.lam = o.relaxpar;
  a.x = P.x64.p;
  a.lbk = o.lb_kind;
  a.ubk = o.ub_kind;
  a.lb = o.lb;
  a.ub = o.ub;
  a.lbv = P.lbv.p;
  a.ubv = P.ubv.p;

  const int L = lanes_for(P.nnz, m);
  // NCP: the residual, the periodogram distances per column, and the
  // ncp_smooth history (check_inputs.m:209, +inf initially)
  DevBuf<double> r64, tw, pk, ccol;
  const int q = ncp ? o.ncp_rows / 2 : 0;
  std::vector<double> hcol(ncp ? o.ncp_cols : 0);
  if (ncp) {
    r64.ensure(m);
    const std::vector<double> t = ncp_twiddles(o.ncp_rows);
    tw.upload(t.data(), t.size(), s);
    pk.ensure((size_t)o.ncp_cols * q);
    ccol.ensure(o.ncp_cols);
  }
  double ncc = 0.0;
  auto resid = [&]() -> double {
    AIRT_CHECK_CUDA(cudaMemsetAsync(red.p, 0, sizeof(double), s));
    const unsigned g = grid_for(m * L, 256);
    switch (L) {
      case 32: k_resid_norm<32><<<g, 256, 0, s>>>(m, P.rp.p, P.ci.p, P.rv.p, P.x64.p, d_b, red.p, ncp ? r64.p : nullptr); break;
      case 16: k_resid_norm<16><<<g, 256, 0, s>>>(m, P.rp.p, P.ci.p, P.rv.p, P.x64.p, d_b, red.p, ncp ? r64.p : nullptr); break;
      case 8: k_resid_norm<8><<<g, 256, 0, s>>>(m, P.rp.p, P.ci.p, P.rv.p, P.x64.p, d_b, red.p, ncp ? r64.p : nullptr); break;
      default: k_resid_norm<4><<<g, 256, 0, s>>>(m, P.rp.p, P.ci.p, P.rv.p, P.x64.p, d_b, red.p, ncp ? r64.p : nullptr); break;
    }
    AIRT_LAUNCH_CHECK();
    if (ncp) {
      k_ncp_power<<<dim3(o.ncp_cols, (q + 255) / 256), 256, 0, s>>>(o.ncp_rows, q, r64.p, tw.p, pk.p, nullptr);
      k_ncp_col<<<o.ncp_cols, 256, 0, s>>>(q, pk.p, ccol.p, nullptr);
      AIRT_LAUNCH_CHECK();
      AIRT_CHECK_CUDA(cudaMemcpyAsync(hcol.data(), ccol.p, o.ncp_cols * sizeof(double), cudaMemcpyDeviceToHost, s));
    }
    double h = 0;
    AIRT_CHECK_CUDA(cudaMemcpyAsync(&h, red.p, sizeof(double), cudaMemcpyDeviceToHost, s));
    AIRT_CHECK_CUDA(cudaStreamSynchronize(s));
    if (ncp) {
      double sum = 0.0;
      for (double v : hcol) sum += v;
      ncc = sum / o.ncp_cols;
    }
    return std::sqrt(h);
  };

  std::vector<double> resn;
  resn.push_back(resid());
  SweepStop st(o.stoprule, o.taudelta, kmax, o.ncp_smooth);
  st.judge(0, resn[0], ncc);
  int64_t l = 0;
  const bool bounded = o.lb_kind != AIRT_BOUND_NONE || o.ub_kind != AIRT_BOUND_NONE;
  double lam_last = o.relaxpar;
  for (int64_t k = 1; !st.stop; ++k) {
    const int64_t *ord = order.data() + (per_sweep_sched ? (k - 1) * per_sweep : 0);
    if (per_sweep_sched) build_schedule(hrp, hci, ord, per_sweep, n, S, s);
    if (k == 1 && bounded && per_sweep > 0) {
      const int64_t r0 = ord[0];
      int64_t rr[2];
      AIRT_CHECK_CUDA(cudaMemcpyAsync(rr, P.rp.p + r0, 2 * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
      AIRT_CHECK_CUDA(cudaStreamSynchronize(s));
      const int64_t len = rr[1] - rr[0];
      keep.ensure(std::max<int64_t>(len, 1));
      k_preclamp<<<1, 1024, 0, s>>>(n, (int)r0, keep.p, a);
    }
    a.lam_tab = tab.p ? tab.p + (k - 1) * per_sweep : nullptr;
    if (S.nsteps > 0) {
      int nsteps = (int)S.nsteps;
      unsigned stamp = (unsigned)k;
      void *args[] = {&nsteps, &S.steps.p, &S.pos.p, &S.pred_ptr.p, &S.preds.p, &stamp,
                      &done.p, &P.err.p, (void *)&budget, (void *)&stall, &a};
      AIRT_CHECK_CUDA(cudaLaunchCooperativeKernel((const void *)k_kacz_dag, dim3(dag_grid),
                                                  dim3(kDagThreads), args, 0, s));
    }
    AIRT_LAUNCH_CHECK();
    AIRT_CHECK_CUDA(cudaMemcpyAsync(&herr, P.err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    if (o.relax_table && per_sweep > 0) lam_last = o.relax_table[(k - 1) * per_sweep + per_sweep - 1];
    const double nrk = resid();  // synchronises the stream (herr is current)
    if (herr) {
      cudaEventDestroy(t0);
      cudaEventDestroy(t1);
      set_error("a bounded device wait of the Kaczmarz sweep gave up (sweep %lld)", (long long)k);
      throw Status{AIRT_ERR_TIMEOUT};
    }
    resn.push_back(nrk);
    st.judge(k, nrk, ncc);
    if ((l < nK && k == K[l]) || st.stop) {
      AIRT_CHECK_CUDA(cudaMemcpyAsync(d_X + l * n, P.x64.p, n * sizeof(double),
                                      cudaMemcpyDeviceToDevice, s));
      ++l;
    }
  }
  AIRT_CHECK_CUDA(cudaEventRecord(t1, s));
  AIRT_CHECK_CUDA(cudaStreamSynchronize(s));
  float ms = 0;
  cudaEventElapsedTime(&ms, t0, t1);
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  if (resn_host) std::copy(resn.begin(), resn.end(), resn_host);
  if (info) {
    info->stoprule = st.stoprule;
    info->finaliter = st.finaliter;
    info->relaxpar = lam_last;
    info->nsaved = l;
    info->gpu_ms = ms;
  }
}

}  // namespace airt

extern "C" int airt_test_set_wait_budget(long long cycles) {
  if (cycles <= 0) return AIRT_ERR_ARG;
  airt::g_kacz_wait_budget = cycles;
  return AIRT_OK;
}

extern "C" int airt_test_inject_stall(int on) {
  airt::g_kacz_inject_stall = on ? 1 : 0;
  return AIRT_OK;
}
