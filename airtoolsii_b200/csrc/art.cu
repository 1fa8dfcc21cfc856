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

// Entries per lane whose gathered x is kept in registers across a row step:
// for rows of up to 32 * kKaczCache entries the update reuses the value of x
// the dot product read (the column indices and values it re-reads are in L1).
constexpr int kKaczCache = 8;

__global__ void __launch_bounds__(1024)
    k_kacz_levels(int nlev, const int *__restrict__ lev_ptr, const int *__restrict__ steps,
                  const int *__restrict__ step_pos, KaczArgs a) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const bool clamp = a.lbk != AIRT_BOUND_NONE || a.ubk != AIRT_BOUND_NONE;
  for (int L = 0; L < nlev; ++L) {
    const int q1 = lev_ptr[L + 1];
    for (int q = lev_ptr[L] + warp; q < q1; q += nw) {
      const int row = steps[q];
      const int64_t s0 = a.rp[row], s1 = a.rp[row + 1];
      const int64_t e0 = s0 + lane;
      // the gathers of the cached part are all issued before the first FMA;
      // the FMAs run in the order of the plain strided loop
      double cx[kKaczCache];
#pragma unroll
      for (int u = 0; u < kKaczCache; ++u)
        cx[u] = e0 + 32 * u < s1 ? a.x[a.ci[e0 + 32 * u]] : 0.0;
      double acc = 0.0;
#pragma unroll
      for (int u = 0; u < kKaczCache; ++u)
        if (e0 + 32 * u < s1) acc = fma((double)a.rv[e0 + 32 * u], cx[u], acc);
      for (int64_t e = e0 + 32 * kKaczCache; e < s1; e += 32)
        acc = fma((double)a.rv[e], a.x[a.ci[e]], acc);
      acc = warp_sum(acc);
      const double lam = a.lam_tab ? a.lam_tab[step_pos[q]] : a.lam;
      const double c = __ddiv_rn(__dmul_rn(lam, __dsub_rn(a.b[row], acc)), a.nrm[row]);
      // no other step of this level touches these pixels, so the gathered x
      // is still the current value
#pragma unroll
      for (int u = 0; u < kKaczCache; ++u)
        if (e0 + 32 * u < s1) {
          const int j = a.ci[e0 + 32 * u];
          double v = __dadd_rn(cx[u], __dmul_rn(c, (double)a.rv[e0 + 32 * u]));
          if (clamp) v = clampv(v, j, a);
          a.x[j] = v;
        }
      for (int64_t e = e0 + 32 * kKaczCache; e < s1; e += 32) {
        const int j = a.ci[e];
        double v = __dadd_rn(a.x[j], __dmul_rn(c, (double)a.rv[e]));
        if (clamp) v = clampv(v, j, a);
        a.x[j] = v;
      }
    }
    __syncthreads();
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

struct Schedule {
  int nlev = 0;
  DevBuf<int> lev_ptr, steps, pos;
};

// Level schedule of a row order (see the file comment).
void build_schedule(const std::vector<int64_t> &hrp, const std::vector<int> &hci,
                    const int64_t *order, int64_t nsteps, int64_t n, Schedule &S,
                    cudaStream_t s) {
  std::vector<int> level(nsteps), last(n, -1);
  int maxlev = -1;
  for (int64_t t = 0; t < nsteps; ++t) {
    const int64_t row = order[t];
    int L = 0;
    for (int64_t e = hrp[row]; e < hrp[row + 1]; ++e) L = std::max(L, last[hci[e]] + 1);
    level[t] = L;
    for (int64_t e = hrp[row]; e < hrp[row + 1]; ++e) last[hci[e]] = L;
    maxlev = std::max(maxlev, L);
  }
  S.nlev = maxlev + 1;
  std::vector<int> ptr(S.nlev + 1, 0), steps(nsteps), pos(nsteps);
  for (int64_t t = 0; t < nsteps; ++t) ++ptr[level[t] + 1];
  for (int L = 0; L < S.nlev; ++L) ptr[L + 1] += ptr[L];
  std::vector<int> fill(ptr.begin(), ptr.end() - 1);
  for (int64_t t = 0; t < nsteps; ++t) {
    const int q = fill[level[t]]++;
    steps[q] = (int)order[t];
    pos[q] = (int)t;
  }
  S.lev_ptr.upload(ptr.data(), ptr.size(), s);
  S.steps.upload(steps.data(), nsteps, s);
  S.pos.upload(pos.data(), nsteps, s);
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

  // host copy of the sparsity pattern for the level schedule
  std::vector<int64_t> hrp(m + 1);
  std::vector<int> hci(P.nnz);
  AIRT_CHECK_CUDA(cudaMemcpyAsync(hrp.data(), P.rp.p, (m + 1) * sizeof(int64_t),
                                  cudaMemcpyDeviceToHost, s));
  if (P.nnz)
    AIRT_CHECK_CUDA(cudaMemcpyAsync(hci.data(), P.ci.p, P.nnz * sizeof(int), cudaMemcpyDeviceToHost, s));
  AIRT_CHECK_CUDA(cudaStreamSynchronize(s));
  Schedule S;
  const bool per_sweep_sched = (o.order_kind == 2 && stride > 0);
  if (!per_sweep_sched) build_schedule(hrp, hci, order.data(), per_sweep, n, S, s);

  // iterate
  P.x64.ensure(n);
  if (d_x0)
    k_copy_d<<<grid_for(n, 256), 256, 0, s>>>(n, d_x0, P.x64.p);
  else
    AIRT_CHECK_CUDA(cudaMemsetAsync(P.x64.p, 0, n * sizeof(double), s));
  if (o.lb_kind == AIRT_BOUND_VECTOR) P.lbv.upload(o.lbv, n, s);
  if (o.ub_kind == AIRT_BOUND_VECTOR) P.ubv.upload(o.ubv, n, s);
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
      const int64_t len = hrp[r0 + 1] - hrp[r0];
      keep.ensure(std::max<int64_t>(len, 1));
      k_preclamp<<<1, 1024, 0, s>>>(n, (int)r0, keep.p, a);
    }
    a.lam_tab = tab.p ? tab.p + (k - 1) * per_sweep : nullptr;
    if (S.nlev > 0) k_kacz_levels<<<1, 1024, 0, s>>>(S.nlev, S.lev_ptr.p, S.steps.p, S.pos.p, a);
    AIRT_LAUNCH_CHECK();
    if (o.relax_table && per_sweep > 0) lam_last = o.relax_table[(k - 1) * per_sweep + per_sweep - 1];
    const double nrk = resid();
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
