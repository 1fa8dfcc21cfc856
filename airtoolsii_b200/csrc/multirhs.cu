// SIRT on K right-hand sides of one system matrix (no counterpart in the
// reference, which takes one b per sirt call, sirt/sirt.m:1).
//
// When many reconstructions share a geometry (the warm-start workload: one
// N = 256, 60-angle paralleltomo matrix, hundreds of sinograms), a block-
// diagonal batch would re-read the same matrix once per instance.  Here the
// K iterates live interleaved, [pixel][instance] (and residuals [ray]
// [instance]), so each nonzero of A is read once per iteration and meets a
// contiguous vector of K instance values: the two SpMVs become SpMMs whose
// gathers are 16-byte coalesced loads from L2.
//
// Per iteration the stream runs
//   bwd : g = A'*(M.*R) over the CSC, x += lambda*D.*g with the box
//         projection, for the instances still running;
//   fwd : R = B - A*X over the CSR, the FP32 copy of M.*R for the next
//         gather (0 for stopped instances), per-block partial ||r_k||^2;
//   ctrl: one block per instance sums the partials in a fixed order and
//         applies check_stoprules.m's DP rule (or kmax) to that instance.
// A lane owns 8 consecutive instances; a group of G lanes (G the smallest
// power of two with 8G >= K, Kp = 8G slots, at most 256 per pass) walks one
// row or column.  All sums
// run in a fixed order, so results repeat bit for bit.  Matrix values and
// the gathered vectors are FP32, accumulation and the iterates FP64, as in
// the single-problem loop.
#include <algorithm>
#include <vector>

#include "common.cuh"

namespace airt {
namespace {

constexpr int kMaxK = 256;      // instances per pass
constexpr int kMrThreads = 256;

struct MrArgs {
  int K, Kp;
  const double *bil;   // [m][Kp]
  const double *M, *D;
  double *x64;         // [n][Kp]
  float *x32;          // [n][Kp]
  float *mr32;         // [m][Kp]
  const int *stop;     // [Kp]
  double *partial;     // [grid][Kp]
  int lbk, ubk;
  double lb, ub;
  MultiState *st;
  const double *lamk;  // per-instance relaxpar [Kp], or null (st->lam for all)
};

__device__ __forceinline__ void load8(const float *p, float v[8]) {
  const float4 a = __ldg(reinterpret_cast<const float4 *>(p));
  const float4 b = __ldg(reinterpret_cast<const float4 *>(p) + 1);
  v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
  v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
}

// Walk segment i (row of the CSR or column of the CSC) with a group of G
// lanes: acc[s] = sum_q val[q] * vec[idx[q]][8*lane + s].
template <int G>
__device__ __forceinline__ void seg_dot(int64_t q0, int64_t q1, const int *__restrict__ idx,
                                        const float *__restrict__ val,
                                        const float *__restrict__ vec, int Kp, int lane,
                                        double acc[8]) {
#pragma unroll
  for (int s = 0; s < 8; ++s) acc[s] = 0.0;
  int64_t q = q0;
  // four nonzeros per round: their indices, values and gathers are all in
  // flight before the first FMA; the FMAs run in nonzero order
  for (; q + 4 <= q1; q += 4) {
    int c[4];
    float v[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      c[u] = __ldg(idx + q + u);
      v[u] = __ldg(val + q + u);
    }
    float g[4][8];
#pragma unroll
    for (int u = 0; u < 4; ++u) load8(vec + (int64_t)c[u] * Kp + 8 * lane, g[u]);
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int s = 0; s < 8; ++s) acc[s] = fma((double)v[u], (double)g[u][s], acc[s]);
  }
  for (; q < q1; ++q) {
    const int c = __ldg(idx + q);
    const double v = (double)__ldg(val + q);
    float g[8];
    load8(vec + (int64_t)c * Kp + 8 * lane, g);
#pragma unroll
    for (int s = 0; s < 8; ++s) acc[s] = fma(v, (double)g[s], acc[s]);
  }
}

// Per-block sums of part[8] over the lanes that own the same 8 instances,
// written to partial[blockIdx.x][8*lane + s] in a fixed order.
template <int G>
__device__ __forceinline__ void block_partials(double part[8], double *__restrict__ partial, int Kp) {
  __shared__ double sh[kMrThreads / 32][kMaxK];
  const int lane32 = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int s = 0; s < 8; ++s)
    for (int o = G; o < 32; o <<= 1) part[s] += __shfl_xor_sync(0xffffffffu, part[s], o);
  if (lane32 < G)
#pragma unroll
    for (int s = 0; s < 8; ++s) sh[warp][8 * lane32 + s] = part[s];
  __syncthreads();
  for (int k = threadIdx.x; k < Kp; k += blockDim.x) {
    double a = 0.0;
    for (int w = 0; w < kMrThreads / 32; ++w) a += sh[w][k];
    partial[(int64_t)blockIdx.x * Kp + k] = a;
  }
}

// R = B - A*X, M.*R (FP32, 0 for stopped instances), per-block ||r_k||^2.
template <int G>
__global__ void __launch_bounds__(kMrThreads, 2) k_mr_fwd(int64_t m, const int64_t *__restrict__ rp,
                                                       const int *__restrict__ ci,
                                                       const float *__restrict__ rv, MrArgs a) {
  if (a.st->active == 0) return;
  const int lane = threadIdx.x % G;
  const int64_t gid = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / G;
  const int64_t ng = (int64_t)gridDim.x * blockDim.x / G;
  const int Kp = a.Kp;
  bool live[8];
#pragma unroll
  for (int s = 0; s < 8; ++s) live[s] = (8 * lane + s) < a.K && !a.stop[8 * lane + s];
  double part[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int64_t i = gid; i < m; i += ng) {
    double acc[8];
    seg_dot<G>(__ldg(rp + i), __ldg(rp + i + 1), ci, rv, a.x32, Kp, lane, acc);
    const double Mi = __ldg(a.M + i);
    const double *bi = a.bil + i * Kp + 8 * lane;
    float mr[8];
#pragma unroll
    for (int s = 0; s < 8; ++s) {
      const double r = __ldg(bi + s) - acc[s];
      mr[s] = live[s] ? (float)(Mi * r) : 0.0f;
      part[s] += live[s] ? r * r : 0.0;
    }
    float4 *o = reinterpret_cast<float4 *>(a.mr32 + i * Kp + 8 * lane);
    o[0] = make_float4(mr[0], mr[1], mr[2], mr[3]);
    o[1] = make_float4(mr[4], mr[5], mr[6], mr[7]);
  }
  block_partials<G>(part, a.partial, Kp);
}

// g = A'*(M.*R); x += lam*D.*g, box projection, FP32 copy (running instances).
template <int G>
__global__ void __launch_bounds__(kMrThreads, 2) k_mr_bwd(int64_t n, const int64_t *__restrict__ cp,
                                                       const int *__restrict__ ri,
                                                       const float *__restrict__ cv, MrArgs a) {
  if (a.st->active == 0) return;
  const int lane = threadIdx.x % G;
  const int64_t gid = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / G;
  const int64_t ng = (int64_t)gridDim.x * blockDim.x / G;
  const int Kp = a.Kp;
  double lam[8];
  bool live[8];
#pragma unroll
  for (int s = 0; s < 8; ++s) {
    live[s] = (8 * lane + s) < a.K && !a.stop[8 * lane + s];
    lam[s] = a.lamk ? a.lamk[8 * lane + s] : a.st->lam;
  }
  for (int64_t j = gid; j < n; j += ng) {
    double g[8];
    seg_dot<G>(__ldg(cp + j), __ldg(cp + j + 1), ri, cv, a.mr32, Kp, lane, g);
    const double Dj = __ldg(a.D + j);
    double *xj = a.x64 + j * Kp + 8 * lane;
    float *xj32 = a.x32 + j * Kp + 8 * lane;
#pragma unroll
    for (int s = 0; s < 8; ++s) {
      if (!live[s]) continue;
      double x = xj[s] + lam[s] * (Dj * g[s]);
      if (a.lbk) x = fmax(x, a.lb);
      if (a.ubk) x = fmin(x, a.ub);
      xj[s] = x;
      xj32[s] = (float)x;
    }
  }
}

// One block per instance: ||r_k||^2 from the per-block partials (fixed
// order), then the DP rule of check_stoprules.m:56-72 or kmax.
__global__ void __launch_bounds__(256) k_mr_ctrl(int K, int Kp, int nparts, int initial,
                                                 int64_t kmax, const double *__restrict__ partial,
                                                 const double *__restrict__ taud, int *stop,
                                                 int *iters, int *rule, double *resn,
                                                 MultiState *st) {
  const int k = blockIdx.x;
  if (k >= K) return;
  if (stop[k]) return;
  double a = 0.0;
  for (int b = threadIdx.x; b < nparts; b += blockDim.x) a += partial[(int64_t)b * Kp + k];
  a = block_sum<256>(a);
  if (threadIdx.x != 0) return;
  const int it = iters[k] + (initial ? 0 : 1);
  iters[k] = it;
  const double nrk = sqrt(a);
  resn[k] = nrk;
  if ((taud && nrk <= taud[k]) || it >= kmax) {
    stop[k] = 1;
    rule[k] = (taud && it != kmax) ? 2 : 0;
    atomicSub(&st->active, 1);
  }
}

__global__ void k_mr_advance(MultiState *st, const double *relax_table, double relaxpar,
                             int64_t kmax, int initial) {
  if (threadIdx.x || blockIdx.x) return;
  const int it = st->iter + (initial ? 0 : 1);
  st->iter = it;
  // relaxpar of iteration it + 1 (relax_table holds kmax entries)
  if (it < kmax) st->lam = relax_table ? relax_table[it] : relaxpar;
}

// [K][len] instance-major <-> [len][Kp] interleaved, through 32 x 32 tiles.
__global__ void k_to_interleaved(int64_t len, int K, int Kp, const double *__restrict__ src,
                                 double *__restrict__ dst, float *__restrict__ dst32) {
  __shared__ double t[32][33];
  const int64_t i0 = (int64_t)blockIdx.x * 32;
  const int k0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int k = k0 + r;
    const int64_t i = i0 + threadIdx.x;
    t[r][threadIdx.x] = (k < K && i < len) ? (src ? src[(int64_t)k * len + i] : 0.0) : 0.0;
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int64_t i = i0 + r;
    const int k = k0 + threadIdx.x;
    if (i < len && k < Kp) {
      const double v = t[threadIdx.x][r];
      dst[i * Kp + k] = v;
      if (dst32) dst32[i * Kp + k] = (float)v;
    }
  }
}

__global__ void k_from_interleaved(int64_t len, int K, int Kp, const double *__restrict__ src,
                                   double *__restrict__ dst, const int *__restrict__ kmap) {
  __shared__ double t[32][33];
  const int64_t i0 = (int64_t)blockIdx.x * 32;
  const int k0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int64_t i = i0 + r;
    const int k = k0 + threadIdx.x;
    t[r][threadIdx.x] = (i < len && k < Kp) ? src[i * Kp + k] : 0.0;
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int k = k0 + r;
    const int64_t i = i0 + threadIdx.x;
    if (k < K && i < len) dst[(int64_t)(kmap ? kmap[k] : k) * len + i] = t[threadIdx.x][r];
  }
}

// Compaction of the interleaved layout to the running instances:
// dst[i][q] = src[i][map[q]] ([len][Kq] from [len][Kp]; map[q] < 0: 0),
// and, for FP64 sources, the FP32 copy.
template <typename T>
__global__ void k_mr_compact(int64_t len, int Kp, int Kq, const int *__restrict__ map,
                             const T *__restrict__ src, T *__restrict__ dst,
                             float *__restrict__ dst32) {
  const int64_t total = len * Kq;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = e / Kq;
    const int q = (int)(e - i * Kq);
    const int k = map[q];
    const T v = k >= 0 ? src[i * Kp + k] : (T)0;
    dst[e] = v;
    if (dst32) dst32[e] = (float)v;
  }
}

// Final iterates of the listed slots to their instance-major rows:
// X[dst_k[c]][j] = x64[j][slot[c]].
__global__ void k_mr_extract(int64_t n, int Kp, int cnt, const int *__restrict__ slot,
                             const int *__restrict__ dst_k, const double *__restrict__ x64,
                             double *__restrict__ X) {
  const int64_t total = (int64_t)cnt * n;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(e / n);
    const int64_t j = e - (int64_t)c * n;
    X[(int64_t)dst_k[c] * n + j] = x64[j * Kp + slot[c]];
  }
}

// After the control step of iteration st->iter: if that iteration is in the
// save list, copy every instance's iterate to its slot (instance-major;
// an instance that has stopped keeps its final iterate).
__global__ void k_mr_save(int64_t n, int K, int Kp, const MultiState *st,
                          const int *__restrict__ save_slot, const double *__restrict__ x64,
                          double *__restrict__ Xs, int64_t slot_stride) {
  const int slot = save_slot[st->iter];
  if (slot < 0) return;
  double *dst = Xs + (int64_t)slot * slot_stride;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < (int64_t)K * n;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int k = (int)(e / n);
    const int64_t j = e - (int64_t)k * n;
    dst[e] = x64[j * Kp + k];
  }
}

int group_for(int Kp) {
  int G = 1;
  while (8 * G < Kp) G <<= 1;
  return G;
}

// One pass: K <= kMaxK instances.  Once the running instances fit in half
// the slots (DP rule, no save list), the pass drains the stream, writes the
// stopped instances' iterates out and compacts the layout to the running
// ones, so an iteration's gathers shrink with the instances still running.
// Every instance's own sums keep their order, so its iterates do not depend
// on the slot it occupies.
void multi_pass(Problem &P, const airt_sirt_opts &o, int K0, const double *d_B, const double *d_X0,
                const double *taud_host, const double *lam_host, const int *save_slot,
                double *d_Xs, int64_t slot_stride, double *d_X, int64_t *finaliter,
                int *stoprule) {
  cudaStream_t s = P.stream;
  const int64_t m = P.m, n = P.n, kmax = o.kmax;
  // every lane of a group owns 8 slots, so the slot count is 8G (G a power
  // of two): no lane reads or writes past its row
  int K = K0;
  int G = group_for((K + 7) / 8 * 8);
  int Kp = 8 * G;
  P.mr_b.ensure((size_t)m * Kp);
  P.mr_x64.ensure((size_t)n * Kp);
  P.mr_x32.ensure((size_t)n * Kp);
  P.mr_r32.ensure((size_t)m * Kp);
  const dim3 tb(32, 8);
  k_to_interleaved<<<dim3((unsigned)((m + 31) / 32), (unsigned)((Kp + 31) / 32)), tb, 0, s>>>(
      m, K, Kp, d_B, P.mr_b.p, nullptr);
  k_to_interleaved<<<dim3((unsigned)((n + 31) / 32), (unsigned)((Kp + 31) / 32)), tb, 0, s>>>(
      n, K, Kp, d_X0, P.mr_x64.p, P.mr_x32.p);
  AIRT_LAUNCH_CHECK();
  auto grids = [&](unsigned &gf, unsigned &gb) {
    gf = std::min<unsigned>(grid_for(m * G, kMrThreads, 8), (unsigned)num_sms() * 8);
    gb = std::min<unsigned>(grid_for(n * G, kMrThreads, 8), (unsigned)num_sms() * 8);
  };
  unsigned gf, gb;
  grids(gf, gb);
  P.mr_part.ensure((size_t)gf * Kp);
  P.mr_stop.ensure(Kp);
  P.mr_iters.ensure(Kp);
  P.mr_rule.ensure(Kp);
  P.mr_resn.ensure(Kp);
  P.mr_state.ensure(1);
  AIRT_CHECK_CUDA(cudaMemsetAsync(P.mr_stop.p, 0, Kp * sizeof(int), s));
  AIRT_CHECK_CUDA(cudaMemsetAsync(P.mr_iters.p, 0, Kp * sizeof(int), s));
  AIRT_CHECK_CUDA(cudaMemsetAsync(P.mr_rule.p, 0, Kp * sizeof(int), s));
  MultiState st0{0, K, o.relaxpar};
  P.mr_state.upload(&st0, 1, s);
  // per-slot copies of the per-instance inputs (slot q holds instance orig[q])
  std::vector<int> orig(K);
  for (int k = 0; k < K; ++k) orig[k] = k;
  std::vector<double> hlam, htaud;
  if (lam_host) {
    hlam.assign(lam_host, lam_host + K);
    hlam.resize(Kp, 0.0);
    P.mr_lam.upload(hlam.data(), Kp, s);
  }
  if (taud_host) {
    htaud.assign(taud_host, taud_host + K);
    P.mr_taud.upload(htaud.data(), K, s);
  }
  const double *taud = taud_host ? P.mr_taud.p : nullptr;
  if (o.relax_kind == AIRT_RELAX_TABLE && kmax > 0) P.table.upload(o.relax_table, kmax, s);
  const double *table = o.relax_kind == AIRT_RELAX_TABLE ? P.table.p : nullptr;

  auto args = [&]() {
    return MrArgs{K, Kp, P.mr_b.p, P.M.p, P.D.p, P.mr_x64.p, P.mr_x32.p, P.mr_r32.p, P.mr_stop.p,
                  P.mr_part.p, o.lb_kind, o.ub_kind, o.lb, o.ub, P.mr_state.p,
                  lam_host ? P.mr_lam.p : nullptr};
  };
  MrArgs a = args();
  auto fwd = [&]() {
    switch (G) {
      case 1: k_mr_fwd<1><<<gf, kMrThreads, 0, s>>>(m, P.rp.p, P.ci.p, P.rv.p, a); break;
      case 2: k_mr_fwd<2><<<gf, kMrThreads, 0, s>>>(m, P.rp.p, P.ci.p, P.rv.p, a); break;
      case 4: k_mr_fwd<4><<<gf, kMrThreads, 0, s>>>(m, P.rp.p, P.ci.p, P.rv.p, a); break;
      case 8: k_mr_fwd<8><<<gf, kMrThreads, 0, s>>>(m, P.rp.p, P.ci.p, P.rv.p, a); break;
      case 16: k_mr_fwd<16><<<gf, kMrThreads, 0, s>>>(m, P.rp.p, P.ci.p, P.rv.p, a); break;
      default: k_mr_fwd<32><<<gf, kMrThreads, 0, s>>>(m, P.rp.p, P.ci.p, P.rv.p, a); break;
    }
  };
  auto bwd = [&]() {
    switch (G) {
      case 1: k_mr_bwd<1><<<gb, kMrThreads, 0, s>>>(n, P.cp.p, P.ri.p, P.cv.p, a); break;
      case 2: k_mr_bwd<2><<<gb, kMrThreads, 0, s>>>(n, P.cp.p, P.ri.p, P.cv.p, a); break;
      case 4: k_mr_bwd<4><<<gb, kMrThreads, 0, s>>>(n, P.cp.p, P.ri.p, P.cv.p, a); break;
      case 8: k_mr_bwd<8><<<gb, kMrThreads, 0, s>>>(n, P.cp.p, P.ri.p, P.cv.p, a); break;
      case 16: k_mr_bwd<16><<<gb, kMrThreads, 0, s>>>(n, P.cp.p, P.ri.p, P.cv.p, a); break;
      default: k_mr_bwd<32><<<gb, kMrThreads, 0, s>>>(n, P.cp.p, P.ri.p, P.cv.p, a); break;
    }
  };
  auto ctrl = [&](int initial) {
    k_mr_ctrl<<<K, 256, 0, s>>>(K, Kp, (int)gf, initial, kmax, P.mr_part.p, taud, P.mr_stop.p,
                                P.mr_iters.p, P.mr_rule.p, P.mr_resn.p, P.mr_state.p);
    k_mr_advance<<<1, 32, 0, s>>>(P.mr_state.p, table, o.relaxpar, kmax, initial);
    if (save_slot && !initial)
      k_mr_save<<<grid_for((int64_t)K * n, 256), 256, 0, s>>>(n, K, Kp, P.mr_state.p, save_slot,
                                                              P.mr_x64.p, d_Xs, slot_stride);
  };
  fwd();
  ctrl(1);
  AIRT_LAUNCH_CHECK();
  // Chunks of iterations captured once as a CUDA graph (again after each
  // compaction).  With the DP rule the host reads the active count after
  // every chunk of 4 (no lag): a drained stream costs tens of microseconds
  // against a chunk of several milliseconds, and an exact, current count
  // lets the layout compact in time for warm-started solves of 10-20
  // iterations, which a count two chunks late would miss.
  const int64_t chunk = taud_host ? 4 : 8;
  const int lag = 0;
  cudaGraphExec_t gexec = nullptr;
  auto capture = [&]() {
    if (gexec) cudaGraphExecDestroy(gexec);
    gexec = nullptr;
    if (kmax < chunk) return;
    cudaGraph_t g = nullptr;
    AIRT_CHECK_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    for (int64_t j = 0; j < chunk; ++j) {
      bwd();
      fwd();
      ctrl(0);
    }
    const cudaError_t ec = cudaStreamEndCapture(s, &g);
    if (ec == cudaSuccess && g) {
      if (cudaGraphInstantiate(&gexec, g, 0) != cudaSuccess) gexec = nullptr;
      cudaGraphDestroy(g);
    }
    cudaGetLastError();
  };
  capture();
  if (!P.h_state) AIRT_CHECK_CUDA(cudaMallocHost(&P.h_state, 3 * sizeof(SirtState)));
  static_assert(sizeof(MultiState) <= sizeof(SirtState), "poll slots");
  MultiState *hs = reinterpret_cast<MultiState *>(P.h_state);  // 3 slots in the pinned mirror
  cudaEvent_t ev[3];
  for (int q = 0; q < 3; ++q) AIRT_CHECK_CUDA(cudaEventCreateWithFlags(&ev[q], cudaEventDisableTiming));
  std::vector<int> hstop, hit, hrule;
  auto record = [&](int q) {  // finaliter / stoprule of slot q's instance
    if (finaliter) finaliter[orig[q]] = hit[q];
    if (stoprule) stoprule[orig[q]] = hrule[q];
  };
  auto read_slots = [&]() {
    hstop.resize(K);
    hit.resize(K);
    hrule.resize(K);
    AIRT_CHECK_CUDA(cudaMemcpyAsync(hstop.data(), P.mr_stop.p, K * sizeof(int), cudaMemcpyDeviceToHost, s));
    AIRT_CHECK_CUDA(cudaMemcpyAsync(hit.data(), P.mr_iters.p, K * sizeof(int), cudaMemcpyDeviceToHost, s));
    AIRT_CHECK_CUDA(cudaMemcpyAsync(hrule.data(), P.mr_rule.p, K * sizeof(int), cudaMemcpyDeviceToHost, s));
    AIRT_CHECK_CUDA(cudaStreamSynchronize(s));
  };
  DevBuf<int> dmap, dslot, ddst;
  DevBuf<double> tmp64;
  DevBuf<float> tmp32;
  // Compacts to the running slots; returns false when none is left.
  auto compact = [&]() {
    read_slots();
    std::vector<int> keep, done_slot, done_k;
    for (int q = 0; q < K; ++q) {
      if (hstop[q]) {
        done_slot.push_back(q);
        done_k.push_back(orig[q]);
        record(q);
      } else {
        keep.push_back(q);
      }
    }
    if (!done_slot.empty()) {
      dslot.upload(done_slot.data(), done_slot.size(), s);
      ddst.upload(done_k.data(), done_k.size(), s);
      k_mr_extract<<<grid_for((int64_t)done_slot.size() * n, 256), 256, 0, s>>>(
          n, Kp, (int)done_slot.size(), dslot.p, ddst.p, P.mr_x64.p, d_X);
    }
    const int Kn = (int)keep.size();
    if (Kn == 0) return false;
    const int Gn = group_for((Kn + 7) / 8 * 8), Kq = 8 * Gn;
    std::vector<int> map(Kq, -1), norig(Kn);
    for (int q = 0; q < Kn; ++q) {
      map[q] = keep[q];
      norig[q] = orig[keep[q]];
    }
    dmap.upload(map.data(), Kq, s);
    // iterates, FP32 copies and right-hand sides
    tmp64.ensure((size_t)n * Kq);
    tmp32.ensure((size_t)n * Kq);
    k_mr_compact<double><<<grid_for(n * Kq, 256), 256, 0, s>>>(n, Kp, Kq, dmap.p, P.mr_x64.p, tmp64.p,
                                                             tmp32.p);
    std::swap(P.mr_x64, tmp64);
    std::swap(P.mr_x32, tmp32);
    tmp64.ensure((size_t)m * Kq);
    k_mr_compact<double><<<grid_for(m * Kq, 256), 256, 0, s>>>(m, Kp, Kq, dmap.p, P.mr_b.p, tmp64.p,
                                                             nullptr);
    std::swap(P.mr_b, tmp64);
    // M.*R of the last forward pass: the next transpose pass reads it
    tmp32.ensure((size_t)m * Kq);
    k_mr_compact<float><<<grid_for(m * Kq, 256), 256, 0, s>>>(m, Kp, Kq, dmap.p, P.mr_r32.p, tmp32.p,
                                                             nullptr);
    std::swap(P.mr_r32, tmp32);
    AIRT_LAUNCH_CHECK();
    // per-slot state: every running instance has the same iteration count
    std::vector<int> zero(Kq, 0), its(Kq, 0);
    for (int q = 0; q < Kn; ++q) its[q] = hit[keep[q]];
    P.mr_stop.upload(zero.data(), Kq, s);
    P.mr_rule.upload(zero.data(), Kq, s);
    P.mr_iters.upload(its.data(), Kq, s);
    if (lam_host) {
      std::vector<double> l(Kq, 0.0);
      for (int q = 0; q < Kn; ++q) l[q] = hlam[keep[q]];
      hlam = l;
      P.mr_lam.upload(hlam.data(), Kq, s);
    }
    if (taud_host) {
      std::vector<double> t(Kn);
      for (int q = 0; q < Kn; ++q) t[q] = htaud[keep[q]];
      htaud = t;
      P.mr_taud.upload(htaud.data(), Kn, s);
    }
    orig = norig;
    K = Kn;
    G = Gn;
    Kp = Kq;
    grids(gf, gb);
    P.mr_part.ensure((size_t)gf * Kp);
    a = args();
    capture();
    return true;
  };
  int64_t c = 0;
  bool live = true;
  for (int64_t it = 1; it <= kmax; ++c) {
    const int64_t cnt = std::min<int64_t>(chunk, kmax - it + 1);
    if (cnt == chunk && gexec) {
      AIRT_CHECK_CUDA(cudaGraphLaunch(gexec, s));
    } else {
      for (int64_t j = 0; j < cnt; ++j) {
        bwd();
        fwd();
        ctrl(0);
      }
    }
    AIRT_LAUNCH_CHECK();
    it += cnt;
    if (!taud) continue;
    AIRT_CHECK_CUDA(cudaMemcpyAsync(hs + (c % 3), P.mr_state.p, sizeof(MultiState),
                                    cudaMemcpyDeviceToHost, s));
    AIRT_CHECK_CUDA(cudaEventRecord(ev[c % 3], s));
    if (c >= lag) {
      AIRT_CHECK_CUDA(cudaEventSynchronize(ev[(c - lag) % 3]));
      const int act = hs[(c - lag) % 3].active;
      if (act == 0) break;
      if (!save_slot && it <= kmax && G > 1 && group_for((act + 7) / 8 * 8) < G) {
        if (!compact()) {
          live = false;
          break;
        }
        c = -1;  // fresh poll slots after the drain
      }
    }
  }
  if (gexec) cudaGraphExecDestroy(gexec);
  for (int q = 0; q < 3; ++q) cudaEventDestroy(ev[q]);
  if (live) {
    const bool ident = K == K0;
    if (!ident) dmap.upload(orig.data(), K, s);
    k_from_interleaved<<<dim3((unsigned)((n + 31) / 32), (unsigned)((Kp + 31) / 32)), tb, 0, s>>>(
        n, K, Kp, P.mr_x64.p, d_X, ident ? nullptr : dmap.p);
    AIRT_LAUNCH_CHECK();
    read_slots();
    for (int q = 0; q < K; ++q) record(q);
  } else {
    AIRT_CHECK_CUDA(cudaStreamSynchronize(s));
  }
}

}  // namespace

void run_sirt_multi(Problem &P, const airt_sirt_opts &o, int K, const double *d_B,
                    const double *d_X0, const double *taud_host, const double *lam_host,
                    const int64_t *Ksave, int64_t nsave, double *d_Xs, double *d_X,
                    int64_t *finaliter, int *stoprule, double *gpu_ms) {
  AIRT_REQUIRE(!P.matrix_free, "multi-right-hand-side SIRT needs the stored matrix");
  AIRT_REQUIRE(K >= 1, "K must be positive");
  AIRT_REQUIRE(o.method >= AIRT_LANDWEBER && o.method <= AIRT_SART,
               "multi-right-hand-side SIRT takes the built-in methods");
  AIRT_REQUIRE(o.relax_kind == AIRT_RELAX_CONST || o.relax_kind == AIRT_RELAX_TABLE,
               "multi-right-hand-side SIRT takes a constant or tabulated relaxpar");
  AIRT_REQUIRE(o.relax_kind != AIRT_RELAX_TABLE || o.relax_table, "relax_table required");
  AIRT_REQUIRE(o.stoprule == AIRT_STOP_NONE || o.stoprule == AIRT_STOP_DP,
               "multi-right-hand-side SIRT takes the DP rule or none");
  AIRT_REQUIRE(o.stoprule != AIRT_STOP_DP || taud_host, "DP needs a taudelta per right-hand side");
  AIRT_REQUIRE(o.lb_kind != AIRT_BOUND_VECTOR && o.ub_kind != AIRT_BOUND_VECTOR,
               "multi-right-hand-side SIRT takes scalar bounds");
  AIRT_REQUIRE(o.kmax >= 0 && o.kmax < (int64_t)INT32_MAX, "kmax out of range");
  AIRT_REQUIRE(nsave == 0 || (Ksave && d_Xs), "save list without an output array");
  cudaStream_t s = P.stream;
  for (int64_t l = 0; l < nsave; ++l) {
    AIRT_REQUIRE(Ksave[l] >= 1 && Ksave[l] <= o.kmax, "saved iterations must lie in 1..kmax");
    AIRT_REQUIRE(l == 0 || Ksave[l] > Ksave[l - 1], "Elements of K must be strictly increasing.");
  }
  if (nsave > 0) {
    std::vector<int> slots(o.kmax + 1, -1);
    for (int64_t l = 0; l < nsave; ++l) slots[Ksave[l]] = (int)l;
    P.save_slot.upload(slots.data(), slots.size(), s);
  }
  cudaEvent_t t0, t1;
  AIRT_CHECK_CUDA(cudaEventCreate(&t0));
  AIRT_CHECK_CUDA(cudaEventCreate(&t1));
  AIRT_CHECK_CUDA(cudaEventRecord(t0, s));
  P.M.ensure(P.m);
  P.D.ensure(P.n);
  compute_weights(P, o.method, P.M.p, P.D.p);
  const double *taud = o.stoprule == AIRT_STOP_DP ? taud_host : nullptr;
  for (int k0 = 0; k0 < K; k0 += kMaxK) {
    const int kc = std::min(kMaxK, K - k0);
    multi_pass(P, o, kc, d_B + (int64_t)k0 * P.m, d_X0 ? d_X0 + (int64_t)k0 * P.n : nullptr,
               taud ? taud + k0 : nullptr, lam_host ? lam_host + k0 : nullptr,
               nsave > 0 ? P.save_slot.p : nullptr, nsave > 0 ? d_Xs + (int64_t)k0 * P.n : nullptr,
               (int64_t)K * P.n, d_X + (int64_t)k0 * P.n, finaliter ? finaliter + k0 : nullptr,
               stoprule ? stoprule + k0 : nullptr);
  }
  AIRT_CHECK_CUDA(cudaEventRecord(t1, s));
  AIRT_CHECK_CUDA(cudaEventSynchronize(t1));
  float ms = 0;
  cudaEventElapsedTime(&ms, t0, t1);
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  if (gpu_ms) *gpu_ms = ms;
}

}  // namespace airt
