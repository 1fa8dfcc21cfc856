// CART column-action sweeps on the GPU (cart/cart.m:139-320).
//
// A sweep visits the columns j of its order one after the other.  An
// unflagged column takes the step od = relaxpar * (a_j'*r)/||a_j||^2,
// clipped so that x(j) + od stays in the box, adds it to x(j) and subtracts
// od*a_j from the residual r; it is flagged when, from sweep Kbegin on,
// |od| < THR * max(abs(x)) with x as it was before the step.  A flagged
// column is skipped until randi(Nunflag) no longer exceeds its count.
//
// Every step reads the residual the previous step wrote, so one CTA walks the
// order.  When the residual fits in shared memory, one warp does: the column's
// entries are spread over the lanes for the dot product (a fixed shuffle tree)
// and the residual update, with no block barrier, and the next column's index,
// flag, x(j), norm and first entries load during the current step (1.10 us per
// column against 1.46 us for the CTA kernel on N=256, 60 angles).  Otherwise
// one 256-thread CTA spreads each column over all its threads, which gathers a
// long column from global memory faster than a warp (N=256, 180 angles: 1.74
// against 2.06 us per column).  max(abs(x)) before each step is kept exact
// without an O(n) scan: the sweep holds the maximum of every 256-entry block of
// |x| in shared memory and the overall maximum in a register; a step changes
// one entry, and a block (or the total) is rescanned only when the entry that
// held its maximum shrank.
#include <algorithm>
#include <cmath>

#include "common.cuh"
#include "ncp.cuh"

namespace airt {

namespace {

constexpr int kCartThreads = 256;  // threads of the CTA sweep
constexpr int kCartBlock = 256;  // entries of x per block maximum
constexpr int kCartPre = 8;      // entries per lane loaded ahead with the next column

struct CartArgs {
  const int64_t *cp;
  const int *ri;
  const float *cv;
  const double *nrm;  // damped squared column norms
  const int *cols;    // sweep order (0-based)
  int64_t ncols;
  double lam;
  double *x, *r;
  unsigned char *flag;  // F of cart.m
  int *nflag;           // Nflag of cart.m
  int lbk, ubk;
  double lb, ub;
  const double *lbv, *ubv;
  double thr;
  int64_t kbegin, nunflag;
  unsigned long long seed;
  int64_t n, m;
  double *r2;  // ||r||^2 after the sweep
  int *err;    // 1: randi(Nunflag) with Nunflag < 1
};

__host__ __device__ inline unsigned long long splitmix64(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// randi(N) of the unflagging test of sweep k at column j: 1 + floor(u*N)
// with u = the top 53 bits of splitmix64(seed ^ splitmix64(k << 32 | j)).
__device__ inline int64_t cart_randi(unsigned long long seed, int64_t k, int j, int64_t N) {
  const unsigned long long key = ((unsigned long long)k << 32) | (unsigned)j;
  const unsigned long long z = splitmix64(seed ^ splitmix64(key));
  const double u = (double)(z >> 11) * 0x1.0p-53;
  return 1 + min((int64_t)floor(u * (double)N), N - 1);
}

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Sum / maximum over the CTA, returned to every thread (the same value in
// all of them: each warp folds the per-warp partials in the same order).
__device__ __forceinline__ double cta_allsum(double v, double *sh) {
  v = warp_sum(v);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = v;
  __syncthreads();
  double t = (l < kCartThreads / 32) ? sh[l] : 0.0;
  t = warp_sum(t);
  __syncthreads();
  return t;
}

__device__ __forceinline__ double cta_allmax(double v, double *sh) {
  v = warp_max(v);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = v;
  __syncthreads();
  double t = (l < kCartThreads / 32) ? sh[l] : 0.0;
  t = warp_max(t);
  __syncthreads();
  return t;
}

// One sweep by one 256-thread CTA with the residual in global memory (used
// when the residual does not fit in shared memory): every column's entries
// are spread over all threads, with block barriers between the steps.
__global__ void __launch_bounds__(kCartThreads) k_cart_sweep_cta(CartArgs a, int64_t k) {
  extern __shared__ double bmax[];  // max |x| of each kCartBlock-entry block
  __shared__ double sh[kCartThreads / 32];
  const int tid = threadIdx.x;
  const int64_t nb = (a.n + kCartBlock - 1) / kCartBlock;
  for (int64_t b = 0; b < nb; ++b) {
    const int64_t i = b * kCartBlock + tid;
    const double v = cta_allmax(i < a.n ? fabs(a.x[i]) : 0.0, sh);
    if (tid == 0) bmax[b] = v;
  }
  __syncthreads();
  double M = 0.0;
  {
    double v = 0.0;
    for (int64_t b = tid; b < nb; b += kCartThreads) v = fmax(v, bmax[b]);
    M = cta_allmax(v, sh);
  }
  const bool lbon = a.lbk != AIRT_BOUND_NONE, ubon = a.ubk != AIRT_BOUND_NONE;
  for (int64_t t = 0; t < a.ncols; ++t) {
    const int j = a.cols[t];
    if (a.flag[j]) {
      const double mm = M;  // max(abs(xk)) before the step, cart.m:227
      const int64_t s0 = a.cp[j], s1 = a.cp[j + 1];
      double part = 0.0;
      for (int64_t q = s0 + tid; q < s1; q += kCartThreads)
        part = fma((double)a.cv[q], a.r[a.ri[q]], part);
      const double dot = cta_allsum(part, sh);
      // cart.m:242-278
      double od = __dmul_rn(a.lam, __ddiv_rn(dot, a.nrm[j]));
      const double xkj = a.x[j];
      if (lbon) {
        const double lo = __dsub_rn(a.lbk == AIRT_BOUND_SCALAR ? a.lb : a.lbv[j], xkj);
        if (od < lo) od = lo;
      }
      if (ubon) {
        const double hi = __dsub_rn(a.ubk == AIRT_BOUND_SCALAR ? a.ub : a.ubv[j], xkj);
        if (od > hi) od = hi;
      }
      const double xn = __dadd_rn(xkj, od);
      for (int64_t q = s0 + tid; q < s1; q += kCartThreads) {
        const int i = a.ri[q];
        a.r[i] = __dsub_rn(a.r[i], __dmul_rn(od, (double)a.cv[q]));
      }
      if (tid == 0) {
        a.x[j] = xn;
        if (k >= a.kbegin && fabs(od) < a.thr * mm) {
          a.flag[j] = 0;
          a.nflag[j] = 1;
        }
      }
      // running maximum of |x|
      const int64_t b = j / kCartBlock;
      const double cur = bmax[b], ao = fabs(xkj), an = fabs(xn);
      __syncthreads();  // x(j), r and the flags are written; bmax[b] is read
      double nbv = cur;
      if (an >= cur) {
        nbv = an;
      } else if (ao == cur) {  // the entry that held the block's maximum shrank
        const int64_t i = b * kCartBlock + tid;
        nbv = cta_allmax(i < a.n ? fabs(a.x[i]) : 0.0, sh);
      }
      if (nbv >= M) {
        M = nbv;
      } else if (cur == M) {  // the block that held the overall maximum dropped
        if (tid == 0) bmax[b] = nbv;
        __syncthreads();
        double v = 0.0;
        for (int64_t bb = tid; bb < nb; bb += kCartThreads) v = fmax(v, bmax[bb]);
        M = cta_allmax(v, sh);
      }
      if (tid == 0) bmax[b] = nbv;
      __syncthreads();
    } else {
      if (tid == 0) {  // cart.m:281-285
        if (a.nunflag < 1) {
          *a.err = 1;
        } else if (a.nflag[j] < cart_randi(a.seed, k, j, a.nunflag)) {
          a.nflag[j] += 1;
        } else {
          a.flag[j] = 1;
        }
      }
      __syncthreads();
    }
  }
  double v = 0.0;
  for (int64_t i = tid; i < a.m; i += kCartThreads) v += a.r[i] * a.r[i];
  v = cta_allsum(v, sh);
  if (tid == 0) *a.r2 = v;
}

// The prefetched part of one step: the column, its start and end, flag,
// x(j), damped norm, and its first kCartPre*32 entries (lane l holds
// entries s0 + l + 32*u).
struct CartCol {
  int j;
  int64_t s0, s1;
  unsigned char f;
  double xj, nrm;
  int ri[kCartPre];
  float cv[kCartPre];
};

__device__ __forceinline__ void cart_load(const CartArgs &a, int64_t t, CartCol &c) {
  const int lane = threadIdx.x;
  c.j = a.cols[t];
  c.s0 = a.cp[c.j];
  c.s1 = a.cp[c.j + 1];
  c.f = a.flag[c.j];
  c.xj = a.x[c.j];
  c.nrm = a.nrm[c.j];
#pragma unroll
  for (int u = 0; u < kCartPre; ++u) {
    const int64_t q = c.s0 + lane + 32 * u;
    c.ri[u] = q < c.s1 ? a.ri[q] : 0;
    c.cv[u] = q < c.s1 ? a.cv[q] : 0.f;
  }
}

// One sweep, one warp (launched as a single 32-thread CTA), with the
// residual copied into shared memory for the sweep and back after it.  Sums
// and maxima use xor shuffles, which leave the same value in every lane.
__global__ void __launch_bounds__(32) k_cart_sweep_warp(CartArgs a, int64_t k) {
  extern __shared__ double smem[];
  const int lane = threadIdx.x;
  const int64_t nb = (a.n + kCartBlock - 1) / kCartBlock;
  double *bmax = smem;  // max |x| of each kCartBlock-entry block
  double *r = smem + ((nb + 1) & ~(int64_t)1);
  for (int64_t i = lane; i < a.m; i += 32) r[i] = a.r[i];
  for (int64_t b = 0; b < nb; ++b) {
    double v = 0.0;
    for (int u = lane; u < kCartBlock; u += 32) {
      const int64_t i = b * kCartBlock + u;
      if (i < a.n) v = fmax(v, fabs(a.x[i]));
    }
    v = warp_max(v);
    if (lane == 0) bmax[b] = v;
  }
  __syncwarp();
  double M = 0.0;
  {
    double v = 0.0;
    for (int64_t b = lane; b < nb; b += 32) v = fmax(v, bmax[b]);
    M = warp_max(v);
  }
  const bool lbon = a.lbk != AIRT_BOUND_NONE, ubon = a.ubk != AIRT_BOUND_NONE;
  CartCol cur, nxt;
  if (a.ncols > 0) cart_load(a, 0, cur);
  int prev = -1;
  for (int64_t t = 0; t < a.ncols; ++t) {
    if (t + 1 < a.ncols) cart_load(a, t + 1, nxt);  // in flight during this step
    const int j = cur.j;
    if (j == prev) {  // the prefetch predates the previous step on the same column
      cur.f = a.flag[j];
      cur.xj = a.x[j];
    }
    if (cur.f) {
      const double mm = M;  // max(abs(xk)) before the step, cart.m:227
      double part = 0.0;
#pragma unroll
      for (int u = 0; u < kCartPre; ++u)
        if (cur.s0 + lane + 32 * u < cur.s1) part = fma((double)cur.cv[u], r[cur.ri[u]], part);
      for (int64_t q = cur.s0 + lane + 32 * kCartPre; q < cur.s1; q += 32)
        part = fma((double)a.cv[q], r[a.ri[q]], part);
      const double dot = warp_sum(part);
      // cart.m:242-278
      double od = __dmul_rn(a.lam, __ddiv_rn(dot, cur.nrm));
      const double xkj = cur.xj;
      if (lbon) {
        const double lo = __dsub_rn(a.lbk == AIRT_BOUND_SCALAR ? a.lb : a.lbv[j], xkj);
        if (od < lo) od = lo;
      }
      if (ubon) {
        const double hi = __dsub_rn(a.ubk == AIRT_BOUND_SCALAR ? a.ub : a.ubv[j], xkj);
        if (od > hi) od = hi;
      }
      const double xn = __dadd_rn(xkj, od);
#pragma unroll
      for (int u = 0; u < kCartPre; ++u)
        if (cur.s0 + lane + 32 * u < cur.s1) {
          const int i = cur.ri[u];
          r[i] = __dsub_rn(r[i], __dmul_rn(od, (double)cur.cv[u]));
        }
      for (int64_t q = cur.s0 + lane + 32 * kCartPre; q < cur.s1; q += 32) {
        const int i = a.ri[q];
        r[i] = __dsub_rn(r[i], __dmul_rn(od, (double)a.cv[q]));
      }
      if (lane == 0) {
        a.x[j] = xn;
        if (k >= a.kbegin && fabs(od) < a.thr * mm) {
          a.flag[j] = 0;
          a.nflag[j] = 1;
        }
      }
      // running maximum of |x|
      const int64_t b = j / kCartBlock;
      const double cur_b = bmax[b], ao = fabs(xkj), an = fabs(xn);
      __syncwarp();  // x(j), r and the flags are written; bmax[b] is read
      double nbv = cur_b;
      if (an >= cur_b) {
        nbv = an;
      } else if (ao == cur_b) {  // the entry that held the block's maximum shrank
        double v = 0.0;
        for (int u = lane; u < kCartBlock; u += 32) {
          const int64_t i = b * kCartBlock + u;
          if (i < a.n) v = fmax(v, fabs(a.x[i]));
        }
        nbv = warp_max(v);
      }
      if (nbv >= M) {
        M = nbv;
      } else if (cur_b == M) {  // the block that held the overall maximum dropped
        if (lane == 0) bmax[b] = nbv;
        __syncwarp();
        double v = 0.0;
        for (int64_t bb = lane; bb < nb; bb += 32) v = fmax(v, bmax[bb]);
        M = warp_max(v);
      }
      __syncwarp();
      if (lane == 0) bmax[b] = nbv;
      __syncwarp();
    } else {
      if (lane == 0) {  // cart.m:281-285
        if (a.nunflag < 1) {
          *a.err = 1;
        } else if (a.nflag[j] < cart_randi(a.seed, k, j, a.nunflag)) {
          a.nflag[j] += 1;
        } else {
          a.flag[j] = 1;
        }
      }
      __syncwarp();
    }
    prev = j;
    cur = nxt;
  }
  double v = 0.0;
  for (int64_t i = lane; i < a.m; i += 32) {
    const double ri = r[i];
    v += ri * ri;
    a.r[i] = ri;
  }
  v = warp_sum(v);
  if (lane == 0) *a.r2 = v;
}

// Squared norms of the CSC columns (cart.m:155-171).
__global__ void k_colnorm2(int64_t n, const int64_t *__restrict__ cp, const float *__restrict__ cv,
                           double *__restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t j = w; j < n; j += nw) {
    double s = 0;
    for (int64_t q = cp[j] + lane; q < cp[j + 1]; q += 32) {
      const double v = (double)cv[q];
      s += v * v;
    }
    s = warp_sum(s);
    if (lane == 0) out[j] = s;
  }
}

__global__ void k_sub_from(int64_t m, const double *__restrict__ b, double *__restrict__ r) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m;
       i += (int64_t)gridDim.x * blockDim.x)
    r[i] = b[i] - r[i];
}

__global__ void k_sumsq(int64_t m, const double *__restrict__ r, double *__restrict__ out) {
  double v = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m;
       i += (int64_t)gridDim.x * blockDim.x)
    v += r[i] * r[i];
  v = block_sum<256>(v);
  if (threadIdx.x == 0) atomicAdd(out, v);
}

}  // namespace

void run_cart(Problem &P, const airt_cart_opts &o, const double *d_b, const double *d_x0,
              const int64_t *K, int64_t nK, double *d_X, double *resn_host, airt_info *info) {
  cudaStream_t s = P.stream;
  const int64_t m = P.m, n = P.n;
  AIRT_REQUIRE(!P.matrix_free, "CART needs the stored matrix (column access)");
  AIRT_REQUIRE(nK >= 1 && K, "Max no. of iterations must ALWAYS be specified.");
  for (int64_t l = 1; l < nK; ++l)
    AIRT_REQUIRE(K[l] > K[l - 1], "Elements of K must be strictly increasing.");
  AIRT_REQUIRE(o.kmax == K[nK - 1] && o.kmax >= 0, "kmax must equal K(end)");
  AIRT_REQUIRE(o.stoprule == AIRT_STOP_NONE || o.stoprule == AIRT_STOP_DP || o.stoprule == AIRT_STOP_NCP,
               "CART supports the NONE, DP and NCP stopping rules");
  const bool ncp = o.stoprule == AIRT_STOP_NCP;
  if (ncp) {
    AIRT_REQUIRE(o.ncp_rows >= 2 && o.ncp_cols >= 1 && (int64_t)o.ncp_rows * o.ncp_cols == m,
                 "NCP: res_dims must multiply to the number of rows of A");
    AIRT_REQUIRE(o.ncp_smooth >= 1, "NCP: ncp_smooth must be positive");
  }
  AIRT_REQUIRE(o.damp >= 0, "Damping must be positive");
  AIRT_REQUIRE(n < (int64_t)INT32_MAX, "too many columns for CART");
  const int64_t nb = (n + kCartBlock - 1) / kCartBlock;
  // shared memory: the block maxima, and the residual too when it fits
  const size_t smem_max = (size_t)(((nb + 1) & ~(int64_t)1) + std::max<int64_t>(m, 1)) * sizeof(double);
  const bool rsmem = smem_max <= 200 * 1024;
  const size_t smem = rsmem ? smem_max : (size_t)std::max<int64_t>(nb, 1) * sizeof(double);
  AIRT_REQUIRE(smem <= 200 * 1024, "CART: too many unknowns for the block maxima in shared memory");
  if (smem > 48 * 1024) {
    if (rsmem)
      AIRT_CHECK_CUDA(cudaFuncSetAttribute(k_cart_sweep_warp,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    else
      AIRT_CHECK_CUDA(cudaFuncSetAttribute(k_cart_sweep_cta,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  }
  const int64_t kmax = o.kmax;

  cudaEvent_t t0, t1;
  AIRT_CHECK_CUDA(cudaEventCreate(&t0));
  AIRT_CHECK_CUDA(cudaEventCreate(&t1));
  AIRT_CHECK_CUDA(cudaEventRecord(t0, s));

  // squared column norms and the column order (cart.m:155-193)
  DevBuf<double> nrm;
  nrm.ensure(std::max<int64_t>(n, 1));
  if (n) {
    k_colnorm2<<<grid_for(n * 32, 256), 256, 0, s>>>(n, P.cp.p, P.cv.p, nrm.p);
    AIRT_LAUNCH_CHECK();
  }
  std::vector<double> hn(n);
  if (n)
    AIRT_CHECK_CUDA(cudaMemcpyAsync(hn.data(), nrm.p, n * sizeof(double), cudaMemcpyDeviceToHost, s));
  AIRT_CHECK_CUDA(cudaStreamSynchronize(s));
  std::vector<int> order;
  if (o.order_kind == 0) {
    for (int64_t j = 0; j < n; ++j)
      if (hn[j] > 0) order.push_back((int)j);
  } else {
    AIRT_REQUIRE(o.order_kind == 2 && (o.cols || o.ncols == 0), "column list missing");
    for (int64_t t = 0; t < o.ncols; ++t) {
      const int64_t j = o.cols[t];
      AIRT_REQUIRE(j >= 0 && j < n, "column index out of range");
      if (hn[j] > 0) order.push_back((int)j);
    }
  }
  if (o.damp > 0) {
    double mx = 0;
    for (double v : hn) mx = std::max(mx, v);
    for (double &v : hn) v = v + o.damp * mx;
    nrm.upload(hn.data(), n, s);
  }
  DevBuf<int> cols, nflag, err;
  DevBuf<unsigned char> flag;
  cols.upload(order.data(), order.size(), s);
  nflag.ensure(std::max<int64_t>(n, 1));
  flag.ensure(std::max<int64_t>(n, 1));
  err.ensure(1);
  AIRT_CHECK_CUDA(cudaMemsetAsync(nflag.p, 0, std::max<int64_t>(n, 1) * sizeof(int), s));
  AIRT_CHECK_CUDA(cudaMemsetAsync(flag.p, 1, std::max<int64_t>(n, 1), s));
  AIRT_CHECK_CUDA(cudaMemsetAsync(err.p, 0, sizeof(int), s));

  // x0 and rk = b - A*x0 (cart.m:139)
  P.x64.ensure(std::max<int64_t>(n, 1));
  P.r64.ensure(std::max<int64_t>(m, 1));
  if (d_x0)
    AIRT_CHECK_CUDA(cudaMemcpyAsync(P.x64.p, d_x0, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  else
    AIRT_CHECK_CUDA(cudaMemsetAsync(P.x64.p, 0, std::max<int64_t>(n, 1) * sizeof(double), s));
  if (m) {
    apply_operator(P, P.x64.p, P.r64.p, 0);
    k_sub_from<<<grid_for(m, 256), 256, 0, s>>>(m, d_b, P.r64.p);
    AIRT_LAUNCH_CHECK();
  }
  if (o.lb_kind == AIRT_BOUND_VECTOR) P.lbv.upload(o.lbv, n, s);
  if (o.ub_kind == AIRT_BOUND_VECTOR) P.ubv.upload(o.ubv, n, s);
  DevBuf<double> red;
  red.ensure(1);

  // NCP periodogram of the residual (check_stoprules.m:96-151)
  DevBuf<double> tw, pk, ccol;
  const int q = ncp ? o.ncp_rows / 2 : 0;
  std::vector<double> hcol(ncp ? o.ncp_cols : 0);
  if (ncp) {
    const std::vector<double> tt = ncp_twiddles(o.ncp_rows);
    tw.upload(tt.data(), tt.size(), s);
    pk.ensure((size_t)o.ncp_cols * q);
    ccol.ensure(o.ncp_cols);
  }
  double ncc = 0.0;
  // ||r|| (and the NCP distance) of the residual the sweeps keep
  auto judge_inputs = [&](bool from_sweep) -> double {
    if (!from_sweep) {
      AIRT_CHECK_CUDA(cudaMemsetAsync(red.p, 0, sizeof(double), s));
      if (m) k_sumsq<<<grid_for(m, 256), 256, 0, s>>>(m, P.r64.p, red.p);
      AIRT_LAUNCH_CHECK();
    }
    if (ncp) {
      k_ncp_power<<<dim3(o.ncp_cols, (q + 255) / 256), 256, 0, s>>>(o.ncp_rows, q, P.r64.p, tw.p,
                                                                    pk.p, nullptr);
      k_ncp_col<<<o.ncp_cols, 256, 0, s>>>(q, pk.p, ccol.p, nullptr);
      AIRT_LAUNCH_CHECK();
      AIRT_CHECK_CUDA(cudaMemcpyAsync(hcol.data(), ccol.p, o.ncp_cols * sizeof(double),
                                      cudaMemcpyDeviceToHost, s));
    }
    double h = 0;
    int herr = 0;
    AIRT_CHECK_CUDA(cudaMemcpyAsync(&h, red.p, sizeof(double), cudaMemcpyDeviceToHost, s));
    AIRT_CHECK_CUDA(cudaMemcpyAsync(&herr, err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    AIRT_CHECK_CUDA(cudaStreamSynchronize(s));
    AIRT_REQUIRE(!herr, "randi: Nunflag must be a positive integer");
    if (ncp) {
      double sum = 0.0;
      for (double v : hcol) sum += v;
      ncc = sum / o.ncp_cols;
    }
    return std::sqrt(h);
  };

  CartArgs a{};
  a.cp = P.cp.p;
  a.ri = P.ri.p;
  a.cv = P.cv.p;
  a.nrm = nrm.p;
  a.cols = cols.p;
  a.ncols = (int64_t)order.size();
  a.lam = o.relaxpar;
  a.x = P.x64.p;
  a.r = P.r64.p;
  a.flag = flag.p;
  a.nflag = nflag.p;
  a.lbk = o.lb_kind;
  a.ubk = o.ub_kind;
  a.lb = o.lb;
  a.ub = o.ub;
  a.lbv = P.lbv.p;
  a.ubv = P.ubv.p;
  a.thr = o.thr;
  a.kbegin = o.kbegin;
  a.nunflag = o.nunflag;
  a.seed = o.seed;
  a.n = n;
  a.m = m;
  a.r2 = red.p;
  a.err = err.p;

  std::vector<double> resn;
  resn.push_back(judge_inputs(false));
  SweepStop st(o.stoprule, o.taudelta, kmax, o.ncp_smooth);
  st.judge(0, resn[0], ncc);
  int64_t l = 0;
  for (int64_t k = 1; !st.stop; ++k) {
    if (rsmem)
      k_cart_sweep_warp<<<1, 32, smem, s>>>(a, k);
    else
      k_cart_sweep_cta<<<1, kCartThreads, smem, s>>>(a, k);
    AIRT_LAUNCH_CHECK();
    const double nrk = judge_inputs(true);
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
    info->relaxpar = o.relaxpar;
    info->nsaved = l;
    info->gpu_ms = ms;
  }
}

}  // namespace airt
