// Batched independent SIRT / Kaczmarz problems (no counterpart in the
// reference, which solves one problem per sirt/art call).
//
// The batch is one block-diagonal system: instance k owns rows
// [row_off[k], row_off[k+1]) and columns [col_off[k], col_off[k+1]); all
// matrices are generated on the GPU in one pass over every ray of every
// instance and stored as one FP32 CSR + CSC.  An iteration is therefore a
// handful of full-bandwidth launches over all instances:
//   bwd (per lane class)  x += lambda_k * D.*A'(M.*r), box clamp
//   fwd (per lane class)  r = b - A*x, M.*r, r.^2 per row
//   reduce                ||r_k||^2 per instance (one block per instance)
//   ctrl                  per-instance DP / max-iteration rule
//   tiles                 lists of the segment tiles still holding an
//                         unstopped instance
// Per-instance scalars (lambda, tau*delta, stop flag, iteration count) are
// read through the row->instance and column->instance maps; stopped
// instances skip their rows and columns entirely.  Rows and columns are cut
// into tiles of 2048 segments; a tile's lane class follows its mean segment
// length (<= 16, 48, 96, 128, > 128 nonzeros), so instances of any size mix in
// any order still give at most five launches per direction.  An autotuner times
// the candidate lane widths on every class once.  A chunk of iterations is
// captured as one CUDA graph (all loop state lives in device memory).
// Kaczmarz runs one CTA per instance over a level schedule of the
// instance's row order, built on the device once per batch.
#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"
#include "ncp.cuh"
#include "spmv.cuh"
#include "trace.cuh"

namespace airt {

struct InstGeom {
  int N, nA, p;
  int ang0;      // first entry of the instance in the angle tables
  int off0;      // first entry in the offset table
  int64_t ray0;  // first global row
  int64_t col0;  // first global column
};

// Segment tiles of the active-tile lists: 2048 rows or columns, in
// kClasses lane classes by mean segment length.
constexpr int kTileShift = 11;
// Resident CTAs per SM of the batch walkers (register budget 48 per thread):
// they are latency bound, so resident warps set their bandwidth.
constexpr int kBatchCtas = 5;
constexpr int kClasses = 5;

// Per-direction tile bookkeeping: class of every tile, tiles per class, and
// the region of each class in the active list.
struct TileSet {
  int ntiles = 0;
  DevBuf<int> cls, list;
  int count[kClasses] = {};
  int off[kClasses] = {};
  int lanes[kClasses] = {2, 4, 4, 8, 8};
};

struct ClassOffsets {
  int off[kClasses];
};

struct Batch {
  Problem P;                 // block-diagonal CSR/CSC and work vectors
  int ninst = 0;
  std::vector<InstGeom> hg;
  std::vector<int64_t> row_off, col_off;
  TileSet rt, ct;  // row (CSR) and column (CSC) tiles
  DevBuf<InstGeom> g;
  DevBuf<int64_t> d_row_off, d_col_off;
  DevBuf<int> inst_row, inst_col, stop, iters, rule, active;
  // 16-bit local column (CSR) and row (CSC) indices, when every instance has
  // at most 65,536 pixels and rays (empty otherwise: the SpMVs then read the
  // 32-bit indices)
  DevBuf<uint16_t> ci16, ri16;
  DevBuf<double> rsq, nrm2, lam, taud, resn_last;
  bool tuned = false;
  // active tiles per class, rebuilt after every stop-rule update:
  // tcount[c] row tiles, tcount[kClasses + c] column tiles of class c
  DevBuf<int> tcount;
  int wmethod = -1;  // method whose M and D are in P.M / P.D (the matrix never changes)
  // M and D of methods used earlier on this batch, saved when the batch
  // switches to another method (the warm start alternates a SART step and
  // cimmino solves: a copy instead of two passes over the matrix per switch)
  static constexpr int kWCache = 8;
  DevBuf<double> wc_M[kWCache], wc_D[kWCache];
  bool wc_ok[kWCache] = {};
  // Kaczmarz level schedules (built on first use): per instance k, levels
  // kz_lev_ptr[base_k .. base_k + kz_nlev[k]] with base_k = row_off[k] + k,
  // row steps of level L at kz_steps[kz_lev_ptr[base_k + L] ..)
  bool kz_ready = false;
  DevBuf<int> kz_lev_ptr, kz_steps, kz_nlev;
  // ME / NCP stopping rules per instance: the previous residual and the
  // per-row products of the ME sums; NCP's projection columns (one per angle
  // of every instance, length p_k), their twiddle tables per distinct p,
  // periodograms, distances and the ncp_smooth history per instance
  DevBuf<double> rprev, pp, ppr, p2, pr;
  bool ncp_ready = false;
  int ncols = 0;
  DevBuf<int64_t> ncp_row0, ncp_tw0, ncp_pk0;
  DevBuf<int> ncp_L, ncp_inst, ncp_col0;
  DevBuf<double> ncp_tw, ncp_pk, ncp_ccol, ncp_dk;
  // the lane classes of one direction run side by side: two more streams,
  // forked from and joined to P.stream by events (graph-capturable)
  cudaStream_t aux[kClasses - 1] = {};
  cudaEvent_t ev_fork = nullptr, ev_join[kClasses - 1] = {};
  ~Batch() {
    for (int i = 0; i < kClasses - 1; ++i) {
      if (aux[i]) cudaStreamDestroy(aux[i]);
      if (ev_join[i]) cudaEventDestroy(ev_join[i]);
    }
    if (ev_fork) cudaEventDestroy(ev_fork);
  }
};

namespace {

__device__ __forceinline__ int find_inst(const int64_t *off, int ninst, int64_t r) {
  int lo = 0, hi = ninst;  // off[lo] <= r < off[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (off[mid] <= r) lo = mid;
    else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ Ray batch_ray(const InstGeom &gk, const double *cos_t, const double *sin_t,
                                         const double *offs, int64_t local) {
  RayGeom g;
  g.kind = GEO_PARALLEL;
  g.N = gk.N;
  g.nA = gk.nA;
  g.p = gk.p;
  g.R = 0;
  g.cos_t = cos_t + gk.ang0;
  g.sin_t = sin_t + gk.ang0;
  g.offsets = offs + gk.off0;
  g.cos_w = g.sin_w = nullptr;
  g.src_x = g.src_y = g.rcv_x = g.rcv_y = nullptr;
  g.radius = g.cscale = g.cos_k = g.sin_k = nullptr;
  g.koff = nullptr;
  g.dx = 0;
  g.center = 0;
  return ray_of(g, local);
}

__global__ void k_batch_count(int ninst, const InstGeom *__restrict__ G, const int64_t *__restrict__ roff,
                              const double *cos_t, const double *sin_t, const double *offs,
                              int64_t nrays, int64_t *__restrict__ counts, int *__restrict__ bad) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < nrays;
       r += (int64_t)gridDim.x * blockDim.x) {
    const int k = find_inst(roff, ninst, r);
    const InstGeom gk = G[k];
    const Ray q = batch_ray(gk, cos_t, sin_t, offs, r - gk.ray0);
    const int64_t nn = (int64_t)gk.N * gk.N;
    int64_t c = 0;
    trace_entries(gk.N, q, true, [&](int col, double) {
      if (col < 0 || col >= nn) atomicExch(bad, 1);
      else ++c;
    });
    counts[r] = c;
  }
}

__global__ void k_batch_fill(int ninst, const InstGeom *__restrict__ G, const int64_t *__restrict__ roff,
                             const double *cos_t, const double *sin_t, const double *offs,
                             int64_t nrays, const int64_t *__restrict__ rp, int *__restrict__ ci,
                             float *__restrict__ rv) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < nrays;
       r += (int64_t)gridDim.x * blockDim.x) {
    const int k = find_inst(roff, ninst, r);
    const InstGeom gk = G[k];
    const Ray q = batch_ray(gk, cos_t, sin_t, offs, r - gk.ray0);
    const int64_t nn = (int64_t)gk.N * gk.N;
    int64_t pos = rp[r];
    const int64_t end = rp[r + 1];
    trace_entries(gk.N, q, true, [&](int col, double v) {
      if (col >= 0 && col < nn && pos < end) {
        ci[pos] = (int)(gk.col0 + col);
        rv[pos] = (float)v;
        ++pos;
      }
    });
  }
}

__global__ void k_fill_inst(int ninst, const int64_t *__restrict__ off, int64_t total,
                            int *__restrict__ inst) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x)
    inst[i] = find_inst(off, ninst, i);
}

// cimmino: M_i = 1/m_k * (1./||a_i||^2) with m_k the rows of i's instance.
__global__ void k_cimmino_batch(int64_t m, const double *__restrict__ s2, const int *__restrict__ inst_row,
                                const int64_t *__restrict__ roff, double *__restrict__ M) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int k = inst_row[i];
    const double mk = (double)(roff[k + 1] - roff[k]);
    const double v = (1.0 / mk) * (1.0 / s2[i]);
    M[i] = isinf(v) ? 0.0 : v;
  }
}

struct BFwd {
  const double *b, *M;
  float *mr32;
  double *rsq;
  const int *inst_row, *stop;
  int64_t r0;
  double *rprev;  // ME / NCP: the residual is kept (previous one read first)
  double *pp;     // ME: rprev.^2 and rprev.*(rprev + r) per row
  double *ppr;
};

// Residual pass; with idx16 (16-bit local column indices, voff = the
// instances' first columns) the nonzeros stream at 6 bytes instead of 8.
template <int L>
__global__ void __launch_bounds__(256, kBatchCtas)
    k_batch_fwd(int64_t nseg, const int *__restrict__ tiles, const int *__restrict__ ntiles,
                const int64_t *__restrict__ rp, const int *__restrict__ ci, const float *__restrict__ rv,
                const float *__restrict__ x32, BFwd o, const uint16_t *__restrict__ idx16,
                const int64_t *__restrict__ voff) {
  auto pre = [&](int64_t i) { return make_double2(o.b[o.r0 + i], o.M[o.r0 + i]); };
  auto epi = [&](int64_t i, double s, bool lead, double2 bm) {
        if (!lead) return;
        const int64_t r = o.r0 + i;
        const double ri = bm.x - s;
        o.mr32[r] = (float)(bm.y * ri);
        o.rsq[r] = ri * ri;
        if (o.rprev) {
          if (o.pp) {
            const double pv = o.rprev[r];
            o.pp[r] = pv * pv;
            o.ppr[r] = pv * (pv + ri);
          }
          o.rprev[r] = ri;
        }
      };
  if (idx16)
    for_each_segment_vt16<L>(nseg, tiles, ntiles, kTileShift, rp + o.r0, idx16, rv, x32, o.inst_row + o.r0, o.stop,
                             voff, pre, epi);
  else
    for_each_segment_vt<L>(
        nseg, tiles, ntiles, kTileShift, rp + o.r0, ci, rv, x32,
        [&](int64_t i) { return o.stop[o.inst_row[o.r0 + i]] == 0; }, pre, epi);
}

struct BUpd {
  const double *D, *lam;
  double *x64;
  float *x32;
  const int *inst_col, *stop;
  int lbk, ubk;
  double lb, ub;
  int64_t c0;
};

// Update pass; idx16 / voff as in k_batch_fwd (16-bit local row indices,
// the instances' first rows).
template <int L>
__global__ void __launch_bounds__(256, kBatchCtas)
    k_batch_bwd(int64_t nseg, const int *__restrict__ tiles, const int *__restrict__ ntiles,
                const int64_t *__restrict__ cp, const int *__restrict__ ri, const float *__restrict__ cv,
                const float *__restrict__ mr32, BUpd u, const uint16_t *__restrict__ idx16,
                const int64_t *__restrict__ voff) {
  auto pre = [&](int64_t j) {
    const int64_t c = u.c0 + j;
    return make_double3(u.x64[c], u.lam[u.inst_col[c]], u.D[c]);
  };
  auto epi = [&](int64_t j, double g, bool lead, double3 xld) {
        if (!lead) return;
        const int64_t c = u.c0 + j;
        double x = xld.x + xld.y * (xld.z * g);
        if (u.lbk) x = fmax(x, u.lb);
        if (u.ubk) x = fmin(x, u.ub);
        u.x64[c] = x;
        u.x32[c] = (float)x;
      };
  if (idx16)
    for_each_segment_vt16<L>(nseg, tiles, ntiles, kTileShift, cp + u.c0, idx16, cv, mr32, u.inst_col + u.c0, u.stop,
                             voff, pre, epi);
  else
    for_each_segment_vt<L>(
        nseg, tiles, ntiles, kTileShift, cp + u.c0, ri, cv, mr32,
        [&](int64_t j) { return u.stop[u.inst_col[u.c0 + j]] == 0; }, pre, epi);
}

// 16-bit local indices of a block-diagonal matrix: out[q] = idx[q] -
// off[inst_of[segment of q]], a warp per segment.
__global__ void k_local16(int64_t nseg, const int64_t *__restrict__ ptr, const int *__restrict__ idx,
                          const int *__restrict__ inst_of, const int64_t *__restrict__ off,
                          uint16_t *__restrict__ out) {
  const int lane = threadIdx.x & 31;
  for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; i < nseg;
       i += ((int64_t)gridDim.x * blockDim.x) >> 5) {
    const int64_t base = off[inst_of[i]];
    for (int64_t q = ptr[i] + lane; q < ptr[i + 1]; q += 32) out[q] = (uint16_t)(idx[q] - base);
  }
}

// Class of every tile of segments [0, nseg): its mean segment length from
// the pointer array.
__global__ void k_tile_class(int ntiles, int64_t nseg, const int64_t *__restrict__ ptr, int *__restrict__ cls) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ntiles) return;
  const int64_t s0 = (int64_t)t << kTileShift;
  const int64_t s1 = min(nseg, s0 + ((int64_t)1 << kTileShift));
  const double avg = (double)(ptr[s1] - ptr[s0]) / (double)(s1 - s0);
  cls[t] = avg > 128.0 ? 4 : avg > 96.0 ? 3 : avg > 48.0 ? 2 : avg > 16.0 ? 1 : 0;
}

// List the tiles (2^kTileShift segments each) that hold at least one
// instance with stop == 0, in the region of the tile's class; inst_of maps a
// segment to its instance (instances are contiguous, so a tile spans
// inst_of[first] .. inst_of[last]).  count[] must start at zero; the order
// within a class is arbitrary.
__global__ void k_active_tiles(int ntiles, int64_t nseg, const int *__restrict__ inst_of,
                               const int *__restrict__ stop, const int *__restrict__ cls, ClassOffsets co,
                               int *__restrict__ list, int *__restrict__ count) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ntiles) return;
  const int64_t s0 = (int64_t)t << kTileShift;
  const int64_t s1 = min(nseg, s0 + ((int64_t)1 << kTileShift));
  for (int k = inst_of[s0]; k <= inst_of[s1 - 1]; ++k)
    if (!stop[k]) {
      const int c = cls[t];
      list[co.off[c] + atomicAdd(count + c, 1)] = t;
      return;
    }
}

// Both directions' active-tile lists in one launch (threads [0, nt_r) the
// row tiles, the rest the column tiles); the counts were zeroed by the step
// kernel that ran before.
struct TileArgs {
  int ntiles;
  int64_t nseg;
  const int *inst_of, *cls;
  ClassOffsets co;
  int *list, *count;
};

__global__ void k_active_tiles2(TileArgs r, TileArgs c, const int *__restrict__ stop) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  const TileArgs *a = &r;
  if (t >= r.ntiles) {
    t -= r.ntiles;
    a = &c;
    if (t >= c.ntiles) return;
  }
  const int64_t s0 = (int64_t)t << kTileShift;
  const int64_t s1 = min(a->nseg, s0 + ((int64_t)1 << kTileShift));
  for (int k = a->inst_of[s0]; k <= a->inst_of[s1 - 1]; ++k)
    if (!stop[k]) {
      const int cl = a->cls[t];
      a->list[a->co.off[cl] + atomicAdd(a->count + cl, 1)] = t;
      return;
    }
}

// NCP per instance, part 1: the periodogram of every projection column of
// the active instances (block = column; frequencies 1..floor(L/2) over the
// threads), by direct summation with the twiddle table of the column's
// length, as k_ncp_power does for one problem.
__global__ void __launch_bounds__(128) k_batch_ncp_power(const int64_t *__restrict__ row0,
                                                         const int *__restrict__ Ls,
                                                         const int64_t *__restrict__ tw0,
                                                         const int64_t *__restrict__ pk0,
                                                         const int *__restrict__ inst,
                                                         const int *__restrict__ stop,
                                                         const double *__restrict__ r,
                                                         const double *__restrict__ tw,
                                                         double *__restrict__ pk) {
  const int j = blockIdx.x;
  if (stop[inst[j]]) return;
  const int L = Ls[j], q = L / 2;
  const double *rc = r + row0[j];
  const double *t = tw + tw0[j];
  for (int f = threadIdx.x + 1; f <= q; f += blockDim.x) {
    double re = 0.0, im = 0.0;
    int idx = 0;
    for (int n = 0; n < L; ++n) {
      const double v = __ldg(rc + n);
      re = fma(v, __ldg(t + 2 * idx), re);
      im = fma(v, __ldg(t + 2 * idx + 1), im);
      idx += f;
      if (idx >= L) idx -= L;
    }
    pk[pk0[j] + (f - 1)] = re * re + im * im;
  }
}

// NCP per instance, part 2: every active column's distance to the white-
// noise cumulative line.
__global__ void __launch_bounds__(256) k_batch_ncp_col(const int *__restrict__ Ls,
                                                       const int64_t *__restrict__ pk0,
                                                       const int *__restrict__ inst,
                                                       const int *__restrict__ stop,
                                                       const double *__restrict__ pk,
                                                       double *__restrict__ ccol) {
  const int j = blockIdx.x;
  if (stop[inst[j]]) return;
  const double d = ncp_distance(Ls[j] / 2, pk + pk0[j]);
  if (threadIdx.x == 0) ccol[j] = d;
}

// Per-instance rule of check_stoprules.m: DP (56-72), ME (74-94), NCP
// (96-151, the residual reshaped to the instance's p x nA projections,
// history of ncp_smooth values per instance) or NONE (153-161).
struct BCtrl {
  int rule;  // AIRT_STOP_*
  const double *taud;
  const double *p2, *pr;                 // ME
  const double *ccol;                    // NCP: distances per column
  const int *col0;                       // NCP: first column of each instance (ninst + 1)
  double *dk;                            // NCP: ncp_smooth values per instance
  int ns;
};

// The rule for instance k after its ||r_k||^2 is known; returns true when k stops.
__device__ __forceinline__ bool batch_rule(int k, int initial, int64_t kmax, const BCtrl &c,
                                           double nrm2, int *__restrict__ iters,
                                           int *__restrict__ rule, double *__restrict__ resn) {
  const int it = iters[k] + (initial ? 0 : 1);
  iters[k] = it;
  const double nrk = sqrt(nrm2);
  resn[k] = nrk;
  bool st = false;
  int why = 0;
  switch (c.rule) {
    case AIRT_STOP_DP:
      if (nrk <= c.taud[k] || it >= kmax) {
        st = true;
        why = it != kmax ? 2 : 0;
      }
      break;
    case AIRT_STOP_ME: {
      const double dme = c.pr[k] / 2.0;
      if (it > 0 && dme / sqrt(c.p2[k]) <= c.taud[k]) {
        st = true;
        why = 3;
      } else if (it >= kmax) {
        st = true;
      }
      break;
    }
    case AIRT_STOP_NCP: {
      double sum = 0.0;
      const int j0 = c.col0[k], j1 = c.col0[k + 1];
      for (int j = j0; j < j1; ++j) sum += c.ccol[j];
      const double ncc = sum / (double)(j1 - j0);
      double *dk = c.dk + (int64_t)k * c.ns;
      double mx = -INFINITY, mxn = ncc;
      for (int i = 0; i < c.ns; ++i) mx = fmax(mx, dk[i]);
      for (int i = 1; i < c.ns; ++i) mxn = fmax(mxn, dk[i]);
      if (mx < mxn || it >= kmax) {
        st = true;
        why = it != kmax ? 1 : 0;
      } else {
        for (int i = 0; i + 1 < c.ns; ++i) dk[i] = dk[i + 1];
        dk[c.ns - 1] = ncc;
      }
      break;
    }
    default:
      st = it >= kmax;
  }
  if (st) rule[k] = why;
  return st;
}

// One block per unstopped instance: ||r_k||^2 (and the ME sums) in a fixed
// order, then the instance's stopping rule; a stopping instance raises its
// flag and takes itself off the active count the host polls.
__global__ void __launch_bounds__(256) k_batch_step(const int64_t *__restrict__ roff,
                                                    const double *__restrict__ rsq,
                                                    const double *__restrict__ pp,
                                                    const double *__restrict__ ppr,
                                                    double *__restrict__ p2,
                                                    double *__restrict__ pr, int initial,
                                                    int64_t kmax, BCtrl c, int *__restrict__ stop,
                                                    int *__restrict__ iters, int *__restrict__ rule,
                                                    double *__restrict__ resn, int *active,
                                                    int *__restrict__ tcount) {
  const int k = blockIdx.x;
  // the active-tile counts of the rebuild that follows this step
  if (tcount && k == 0 && threadIdx.x < 2 * kClasses) tcount[threadIdx.x] = 0;
  if (stop[k]) return;
  double a = 0, e = 0, d = 0;
  for (int64_t i = roff[k] + threadIdx.x; i < roff[k + 1]; i += blockDim.x) {
    a += rsq[i];
    if (pp) {
      e += pp[i];
      d += ppr[i];
    }
  }
  a = block_sum<256>(a);
  if (pp) {
    e = block_sum<256>(e);
    d = block_sum<256>(d);
  }
  if (threadIdx.x != 0) return;
  if (pp) {
    p2[k] = e;
    pr[k] = d;
  }
  if (batch_rule(k, initial, kmax, c, a, iters, rule, resn)) {
    stop[k] = 1;
    atomicSub(active, 1);
  }
}

__global__ void k_copy_f32(int64_t n, const double *__restrict__ a, float *__restrict__ b) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}

// Per-instance power-iteration pieces on column ranges.
__global__ void __launch_bounds__(256) k_inst_dot2(const int64_t *__restrict__ coff,
                                                   const double *__restrict__ u,
                                                   const double *__restrict__ w,
                                                   double *__restrict__ uw, double *__restrict__ ww) {
  const int k = blockIdx.x;
  double a = 0, b2 = 0;
  for (int64_t j = coff[k] + threadIdx.x; j < coff[k + 1]; j += blockDim.x) {
    a += u[j] * w[j];
    b2 += w[j] * w[j];
  }
  a = block_sum<256>(a);
  b2 = block_sum<256>(b2);
  if (threadIdx.x == 0) {
    uw[k] = a;
    ww[k] = b2;
  }
}

__global__ void k_inst_normalize(int64_t n, const int *__restrict__ inst_col, const double *__restrict__ w,
                                 const double *__restrict__ ww, double *__restrict__ u) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n;
       j += (int64_t)gridDim.x * blockDim.x) {
    const double s = ww[inst_col[j]];
    u[j] = s > 0 ? w[j] / sqrt(s) : 0.0;
  }
}

__global__ void k_inst_init(int64_t n, const int *__restrict__ inst_col, const int64_t *__restrict__ coff,
                            double *__restrict__ u) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n;
       j += (int64_t)gridDim.x * blockDim.x) {
    const int k = inst_col[j];
    u[j] = 1.0 / sqrt((double)(coff[k + 1] - coff[k]));
  }
}

__global__ void k_vmul(int64_t n, const double *__restrict__ a, const double *__restrict__ b,
                       double *__restrict__ c) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    c[i] = a[i] * b[i];
}

__global__ void k_vsqrt(int64_t n, const double *__restrict__ a, double *__restrict__ b) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    b[i] = sqrt(a[i] > 0 ? a[i] : 0.0);
}

// ---------------------------------------------------------------- launchers
template <class F>
float time_launch(cudaStream_t s, F &&f, int reps = 3) {
  cudaEvent_t e0, e1;
  AIRT_CHECK_CUDA(cudaEventCreate(&e0));
  AIRT_CHECK_CUDA(cudaEventCreate(&e1));
  f();
  AIRT_CHECK_CUDA(cudaEventRecord(e0, s));
  for (int r = 0; r < reps; ++r) f();
  AIRT_CHECK_CUDA(cudaEventRecord(e1, s));
  AIRT_CHECK_CUDA(cudaEventSynchronize(e1));
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return ms / reps;
}

// Launch class c of the forward / transpose kernel with L lanes per
// segment; the grid covers every tile of the class (graph-capturable), the
// kernel walks only the listed ones.
void launch_bfwd(Batch &B, int c, int L, const BFwd &o, const float *x32 = nullptr,
                 cudaStream_t st = nullptr) {
  Problem &P = B.P;
  if (!x32) x32 = P.x32.p;
  if (B.rt.count[c] == 0) return;
  cudaStream_t s = st ? st : P.stream;
  const int64_t ns = P.m;
  const unsigned g = grid_for((int64_t)B.rt.count[c] * (1 << kTileShift) * L, 256, kBatchCtas);
  const int *tl = B.rt.list.p + B.rt.off[c], *cnt = B.tcount.p + c;
  // 16-bit indices for the two longest-segment classes (mean above 96
  // nonzeros) only: on shorter segments the 8-aligned head and tail (up to 7
  // elements each, element-wise) cost more than the index bytes save
  // (measured on the 512-instance batch: all-active iterations 5 % faster,
  // the short-segment tail 5 % slower when every class used them; the
  // 97-128 class as well as the longest: the whole batch 0.8 % faster)
  const uint16_t *i16 = c >= kClasses - 2 ? B.ci16.p : nullptr;
  switch (L) {
#define AIRT_F(LV) \
  k_batch_fwd<LV><<<g, 256, 0, s>>>(ns, tl, cnt, P.rp.p, P.ci.p, P.rv.p, x32, o, i16, B.d_col_off.p)
    case 16: AIRT_F(16); break;
    case 8: AIRT_F(8); break;
    case 4: AIRT_F(4); break;
    default: AIRT_F(2); break;
#undef AIRT_F
  }
}

void launch_bbwd(Batch &B, int c, int L, const BUpd &u, const float *mr32 = nullptr,
                 cudaStream_t st = nullptr) {
  Problem &P = B.P;
  if (!mr32) mr32 = P.mr32.p;
  if (B.ct.count[c] == 0) return;
  cudaStream_t s = st ? st : P.stream;
  const int64_t ns = P.n;
  const unsigned g = grid_for((int64_t)B.ct.count[c] * (1 << kTileShift) * L, 256, kBatchCtas);
  const int *tl = B.ct.list.p + B.ct.off[c], *cnt = B.tcount.p + kClasses + c;
  const uint16_t *i16 = c >= kClasses - 2 ? B.ri16.p : nullptr;  // as in launch_bfwd
  switch (L) {
#define AIRT_B(LV) \
  k_batch_bwd<LV><<<g, 256, 0, s>>>(ns, tl, cnt, P.cp.p, P.ri.p, P.cv.p, mr32, u, i16, B.d_row_off.p)
    case 16: AIRT_B(16); break;
    case 8: AIRT_B(8); break;
    case 4: AIRT_B(4); break;
    default: AIRT_B(2); break;
#undef AIRT_B
  }
}

// The classes with tiles run concurrently: the largest on P.stream, the
// others on the auxiliary streams, joined back before the next step.
template <class F>
void run_classes(Batch &B, const TileSet &T, F &&launch) {
  cudaStream_t s = B.P.stream;
  int big = 0;
  for (int c = 1; c < kClasses; ++c)
    if (T.count[c] > T.count[big]) big = c;
  int na = 0;
  for (int c = 0; c < kClasses; ++c)
    if (c != big && T.count[c] > 0) ++na;
  if (na > 0) AIRT_CHECK_CUDA(cudaEventRecord(B.ev_fork, s));
  int q = 0;
  for (int c = 0; c < kClasses; ++c) {
    if (c == big || T.count[c] == 0) continue;
    AIRT_CHECK_CUDA(cudaStreamWaitEvent(B.aux[q], B.ev_fork, 0));
    launch(c, B.aux[q]);
    AIRT_CHECK_CUDA(cudaEventRecord(B.ev_join[q], B.aux[q]));
    ++q;
  }
  launch(big, s);
  for (int i = 0; i < q; ++i) AIRT_CHECK_CUDA(cudaStreamWaitEvent(s, B.ev_join[i], 0));
}

void fwd_classes(Batch &B, const BFwd &o) {
  run_classes(B, B.rt, [&](int c, cudaStream_t st) { launch_bfwd(B, c, B.rt.lanes[c], o, nullptr, st); });
}

void bwd_classes(Batch &B, const BUpd &u) {
  run_classes(B, B.ct, [&](int c, cudaStream_t st) { launch_bbwd(B, c, B.ct.lanes[c], u, nullptr, st); });
}

// Rebuild the active row and column tile lists from stop[].
void build_tiles(Batch &B, const int *stop) {
  Problem &P = B.P;
  cudaStream_t s = P.stream;
  AIRT_CHECK_CUDA(cudaMemsetAsync(B.tcount.p, 0, 2 * kClasses * sizeof(int), s));
  ClassOffsets ro, co;
  for (int c = 0; c < kClasses; ++c) {
    ro.off[c] = B.rt.off[c];
    co.off[c] = B.ct.off[c];
  }
  k_active_tiles<<<(B.rt.ntiles + 127) / 128, 128, 0, s>>>(B.rt.ntiles, P.m, B.inst_row.p, stop, B.rt.cls.p, ro,
                                                           B.rt.list.p, B.tcount.p);
  k_active_tiles<<<(B.ct.ntiles + 127) / 128, 128, 0, s>>>(B.ct.ntiles, P.n, B.inst_col.p, stop, B.ct.cls.p, co,
                                                           B.ct.list.p, B.tcount.p + kClasses);
  AIRT_LAUNCH_CHECK();
}

// Rebuild after k_batch_step (which zeroed the counts): one launch.
void build_tiles_after_step(Batch &B, const int *stop) {
  Problem &P = B.P;
  TileArgs r{B.rt.ntiles, P.m, B.inst_row.p, B.rt.cls.p, {}, B.rt.list.p, B.tcount.p};
  TileArgs c{B.ct.ntiles, P.n, B.inst_col.p, B.ct.cls.p, {}, B.ct.list.p, B.tcount.p + kClasses};
  for (int q = 0; q < kClasses; ++q) {
    r.co.off[q] = B.rt.off[q];
    c.co.off[q] = B.ct.off[q];
  }
  const int nt = B.rt.ntiles + B.ct.ntiles;
  k_active_tiles2<<<(nt + 127) / 128, 128, 0, P.stream>>>(r, c, stop);
  AIRT_LAUNCH_CHECK();
}

// Tiles of one direction: classes on the device, counts and list regions on
// the host.
void setup_tileset(TileSet &T, int64_t nseg, const int64_t *ptr, cudaStream_t s) {
  T.ntiles = (int)((nseg + (1 << kTileShift) - 1) >> kTileShift);
  T.cls.ensure(T.ntiles > 0 ? T.ntiles : 1);
  T.list.ensure(T.ntiles > 0 ? T.ntiles : 1);
  for (int c = 0; c < kClasses; ++c) T.count[c] = 0;
  if (T.ntiles == 0) return;
  k_tile_class<<<(T.ntiles + 127) / 128, 128, 0, s>>>(T.ntiles, nseg, ptr, T.cls.p);
  AIRT_LAUNCH_CHECK();
  std::vector<int> h(T.ntiles);
  AIRT_CHECK_CUDA(cudaMemcpyAsync(h.data(), T.cls.p, T.ntiles * sizeof(int), cudaMemcpyDeviceToHost, s));
  AIRT_CHECK_CUDA(cudaStreamSynchronize(s));
  for (int v : h) ++T.count[v];
  int off = 0;
  for (int c = 0; c < kClasses; ++c) {
    T.off[c] = off;
    off += T.count[c];
  }
}

}  // namespace

// ---------------------------------------------------------------- building
Batch *batch_build(int ninst, const int *N, const int *nA, const int *p, const double *cos_t,
                   const double *sin_t, const double *offsets) {
  Batch *B = new Batch();
  try {
    AIRT_CHECK_CUDA(cudaStreamCreateWithFlags(&B->P.stream, cudaStreamNonBlocking));
    for (int i = 0; i < kClasses - 1; ++i) {
      AIRT_CHECK_CUDA(cudaStreamCreateWithFlags(&B->aux[i], cudaStreamNonBlocking));
      AIRT_CHECK_CUDA(cudaEventCreateWithFlags(&B->ev_join[i], cudaEventDisableTiming));
    }
    AIRT_CHECK_CUDA(cudaEventCreateWithFlags(&B->ev_fork, cudaEventDisableTiming));
    Problem &P = B->P;
    cudaStream_t s = P.stream;
    B->ninst = ninst;
    B->hg.resize(ninst);
    B->row_off.assign(ninst + 1, 0);
    B->col_off.assign(ninst + 1, 0);
    int64_t angs = 0, offs = 0;
    for (int k = 0; k < ninst; ++k) {
      AIRT_REQUIRE(N[k] >= 1 && N[k] <= 46340 && nA[k] >= 0 && p[k] >= 0, "instance %d: bad size", k);
      InstGeom &gk = B->hg[k];
      gk.N = N[k];
      gk.nA = nA[k];
      gk.p = p[k];
      gk.ang0 = (int)angs;
      gk.off0 = (int)offs;
      gk.ray0 = B->row_off[k];
      gk.col0 = B->col_off[k];
      angs += nA[k];
      offs += p[k];
      B->row_off[k + 1] = B->row_off[k] + (int64_t)nA[k] * p[k];
      B->col_off[k + 1] = B->col_off[k] + (int64_t)N[k] * N[k];
    }
    P.m = B->row_off[ninst];
    P.n = B->col_off[ninst];
    AIRT_REQUIRE(P.m < INT32_MAX && P.n < INT32_MAX, "batch too large (rows or columns >= 2^31)");
    P.geo_kind = GEO_PARALLEL;
    P.cos_t.upload(cos_t, angs, s);
    P.sin_t.upload(sin_t, angs, s);
    P.offsets.upload(offsets, offs, s);
    B->g.upload(B->hg.data(), ninst, s);
    B->d_row_off.upload(B->row_off.data(), ninst + 1, s);
    B->d_col_off.upload(B->col_off.data(), ninst + 1, s);
    // generation: count, scan, fill, transpose (as generate_matrix)
    DevBuf<int64_t> counts;
    DevBuf<int> bad;
    counts.ensure(P.m);
    bad.ensure(1);
    AIRT_CHECK_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int), s));
    const unsigned grid = grid_for(P.m, 128, 16);
    k_batch_count<<<grid, 128, 0, s>>>(ninst, B->g.p, B->d_row_off.p, P.cos_t.p, P.sin_t.p,
                                       P.offsets.p, P.m, counts.p, bad.p);
    AIRT_LAUNCH_CHECK();
    P.rp.ensure(P.m + 1 + 4);
    AIRT_CHECK_CUDA(cudaMemsetAsync(P.rp.p + P.m + 1, 0, 4 * sizeof(int64_t), s));
    exclusive_scan_i64(counts.p, P.rp.p, P.m, s);
    int hbad = 0;
    AIRT_CHECK_CUDA(cudaMemcpyAsync(&P.nnz, P.rp.p + P.m, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    AIRT_CHECK_CUDA(cudaMemcpyAsync(&hbad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    AIRT_CHECK_CUDA(cudaStreamSynchronize(s));
    AIRT_REQUIRE(!hbad, "ray trace produced a pixel index outside the image");
    P.ci.ensure(P.nnz + 8);
    P.rv.ensure(P.nnz + 8);
    AIRT_CHECK_CUDA(cudaMemsetAsync(P.ci.p + P.nnz, 0, 8 * sizeof(int), s));
    AIRT_CHECK_CUDA(cudaMemsetAsync(P.rv.p + P.nnz, 0, 8 * sizeof(float), s));
    k_batch_fill<<<grid, 128, 0, s>>>(ninst, B->g.p, B->d_row_off.p, P.cos_t.p, P.sin_t.p,
                                      P.offsets.p, P.m, P.rp.p, P.ci.p, P.rv.p);
    AIRT_LAUNCH_CHECK();
    counts.release();
    build_csc_from_csr(P);
    B->inst_row.ensure(P.m);
    B->inst_col.ensure(P.n);
    k_fill_inst<<<grid_for(P.m, 256), 256, 0, s>>>(ninst, B->d_row_off.p, P.m, B->inst_row.p);
    k_fill_inst<<<grid_for(P.n, 256), 256, 0, s>>>(ninst, B->d_col_off.p, P.n, B->inst_col.p);
    AIRT_LAUNCH_CHECK();
    bool fits16 = true;
    for (int k = 0; k < ninst; ++k)
      fits16 = fits16 && B->row_off[k + 1] - B->row_off[k] <= 65536 && B->col_off[k + 1] - B->col_off[k] <= 65536;
    if (fits16 && P.nnz > 0) {
      B->ci16.ensure(P.nnz);
      B->ri16.ensure(P.nnz);
      k_local16<<<grid_for(P.m * 32, 256), 256, 0, s>>>(P.m, P.rp.p, P.ci.p, B->inst_row.p, B->d_col_off.p,
                                                        B->ci16.p);
      k_local16<<<grid_for(P.n * 32, 256), 256, 0, s>>>(P.n, P.cp.p, P.ri.p, B->inst_col.p, B->d_row_off.p,
                                                        B->ri16.p);
      AIRT_LAUNCH_CHECK();
    }
    setup_tileset(B->rt, P.m, P.rp.p, s);
    setup_tileset(B->ct, P.n, P.cp.p, s);
    B->tcount.ensure(2 * kClasses);
    AIRT_CHECK_CUDA(cudaStreamSynchronize(s));
  } catch (...) {
    if (B->P.stream) cudaStreamSynchronize(B->P.stream);
    cudaStream_t st = B->P.stream;
    delete B;
    if (st) cudaStreamDestroy(st);
    throw;
  }
  return B;
}

Problem &batch_problem(Batch &B) { return B.P; }
int batch_ninst(const Batch &B) { return B.ninst; }
const int64_t *batch_row_off(const Batch &B) { return B.row_off.data(); }
const int64_t *batch_col_off(const Batch &B) { return B.col_off.data(); }

void batch_destroy(Batch *B) {
  if (!B) return;
  cudaStream_t s = B->P.stream;
  if (s) cudaStreamSynchronize(s);
  if (B->P.h_state) cudaFreeHost(B->P.h_state);
  B->P.h_state = nullptr;
  delete B;
  if (s) cudaStreamDestroy(s);
}

namespace {
__global__ void k_batch_mb(int64_t m, const double *__restrict__ M, const double *__restrict__ b,
                           float *__restrict__ mr32) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x)
    mr32[i] = (float)(M[i] * b[i]);
}

__global__ void k_fill1(int64_t n, double *__restrict__ a) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    a[i] = 1.0;
}
}  // namespace

// Weights of get_mfun_dfun.m per instance: only cimmino's 1/m factor depends on
// the instance; every other weight is a per-row or per-column quantity.
void batch_weights(Batch &B, int method) {
  Problem &P = B.P;
  if (B.wmethod == method) return;
  cudaStream_t s = P.stream;
  const int prev = B.wmethod;
  if (prev >= 0 && prev < Batch::kWCache && !B.wc_ok[prev]) {
    B.wc_M[prev].ensure(P.m);
    B.wc_D[prev].ensure(P.n);
    AIRT_CHECK_CUDA(cudaMemcpyAsync(B.wc_M[prev].p, P.M.p, P.m * sizeof(double), cudaMemcpyDeviceToDevice, s));
    AIRT_CHECK_CUDA(cudaMemcpyAsync(B.wc_D[prev].p, P.D.p, P.n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    B.wc_ok[prev] = true;
  }
  P.M.ensure(P.m);
  P.D.ensure(P.n);
  B.wmethod = method;
  if (method >= 0 && method < Batch::kWCache && B.wc_ok[method]) {
    AIRT_CHECK_CUDA(cudaMemcpyAsync(P.M.p, B.wc_M[method].p, P.m * sizeof(double), cudaMemcpyDeviceToDevice, s));
    AIRT_CHECK_CUDA(cudaMemcpyAsync(P.D.p, B.wc_D[method].p, P.n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    return;
  }
  if (method != AIRT_CIMMINO) {
    compute_weights(P, method, P.M.p, P.D.p);
    return;
  }
  P.w2.ensure(P.m > P.n ? P.m : P.n);
  row_sums_sq(P, P.w2.p);
  k_cimmino_batch<<<grid_for(P.m, 256), 256, 0, P.stream>>>(P.m, P.w2.p, B.inst_row.p,
                                                            B.d_row_off.p, P.M.p);
  k_fill1<<<grid_for(P.n, 256), 256, 0, P.stream>>>(P.n, P.D.p);
  AIRT_LAUNCH_CHECK();
}

void batch_rho(Batch &B, int method, double tol, int maxit, double *rho_host) {
  Problem &P = B.P;
  cudaStream_t s = P.stream;
  batch_weights(B, method);
  const int K = B.ninst;
  DevBuf<double> sd, u, t, y, w, uw, ww;
  sd.ensure(P.n);
  u.ensure(P.n);
  t.ensure(P.n);
  y.ensure(P.m);
  w.ensure(P.n);
  uw.ensure(K);
  ww.ensure(K);
  const unsigned gn = grid_for(P.n, 256), gm = grid_for(P.m, 256);
  k_vsqrt<<<gn, 256, 0, s>>>(P.n, P.D.p, sd.p);
  k_inst_init<<<gn, 256, 0, s>>>(P.n, B.inst_col.p, B.d_col_off.p, u.p);
  std::vector<double> lam(K, 0.0), prev(K, 0.0);
  for (int it = 0; it < maxit; ++it) {
    k_vmul<<<gn, 256, 0, s>>>(P.n, sd.p, u.p, t.p);
    apply_operator(P, t.p, y.p, 0);
    k_vmul<<<gm, 256, 0, s>>>(P.m, P.M.p, y.p, y.p);
    apply_operator(P, y.p, t.p, 1);
    k_vmul<<<gn, 256, 0, s>>>(P.n, sd.p, t.p, w.p);
    k_inst_dot2<<<K, 256, 0, s>>>(B.d_col_off.p, u.p, w.p, uw.p, ww.p);
    k_inst_normalize<<<gn, 256, 0, s>>>(P.n, B.inst_col.p, w.p, ww.p, u.p);
    AIRT_LAUNCH_CHECK();
    AIRT_CHECK_CUDA(cudaMemcpyAsync(lam.data(), uw.p, K * sizeof(double), cudaMemcpyDeviceToHost, s));
    AIRT_CHECK_CUDA(cudaStreamSynchronize(s));
    bool done = it > 0;
    for (int k = 0; k < K && done; ++k)
      if (std::fabs(lam[k] - prev[k]) > tol * std::fabs(lam[k])) done = false;
    prev = lam;
    if (done) break;
  }
  for (int k = 0; k < K; ++k) rho_host[k] = lam[k];
}

// Times the candidate lane widths per bucket once (the autotuner).
void batch_tune(Batch &B) {
  if (B.tuned) return;
  Problem &P = B.P;
  cudaStream_t s = P.stream;
  DevBuf<double> yr, yc;
  DevBuf<float> xr, xc;
  yr.ensure(P.m);
  yc.ensure(P.n);
  xr.ensure(P.m);
  xc.ensure(P.n);
  AIRT_CHECK_CUDA(cudaMemsetAsync(xr.p, 0, P.m * sizeof(float), s));
  AIRT_CHECK_CUDA(cudaMemsetAsync(xc.p, 0, P.n * sizeof(float), s));
  DevBuf<int> nostop;
  nostop.ensure(B.ninst);
  AIRT_CHECK_CUDA(cudaMemsetAsync(nostop.p, 0, B.ninst * sizeof(int), s));
  build_tiles(B, nostop.p);
  DevBuf<double> zero;
  zero.ensure(P.m > P.n ? P.m : P.n);
  AIRT_CHECK_CUDA(cudaMemsetAsync(zero.p, 0, zero.n * sizeof(double), s));
  DevBuf<double> xtmp;
  xtmp.ensure(P.n);
  DevBuf<float> mtmp, x32tmp;
  mtmp.ensure(P.m);
  x32tmp.ensure(P.n);
  const int cands[4] = {2, 4, 8, 16};
  for (int c = 0; c < kClasses; ++c) {
    float best_f = 1e30f, best_b = 1e30f;
    for (int L : cands) {
      if (B.rt.count[c] > 0) {
        BFwd o{zero.p, zero.p, mtmp.p, yr.p, B.inst_row.p, nostop.p, 0};
        const float tf = time_launch(s, [&] { launch_bfwd(B, c, L, o, xc.p); });
        if (tf < best_f) {
          best_f = tf;
          B.rt.lanes[c] = L;
        }
      }
      if (B.ct.count[c] > 0) {
        BUpd u{zero.p, zero.p, xtmp.p, x32tmp.p, B.inst_col.p, nostop.p, 0, 0, 0.0, 0.0, 0};
        const float tb = time_launch(s, [&] { launch_bbwd(B, c, L, u, xr.p); });
        if (tb < best_b) {
          best_b = tb;
          B.ct.lanes[c] = L;
        }
      }
      AIRT_LAUNCH_CHECK();
    }
  }
  B.tuned = true;
}

namespace {
// NCP column tables of a batch (built once): one column per projection of
// every instance (instance k: nA_k columns of p_k rows), twiddles per
// distinct column length.
void batch_ncp_setup(Batch &B) {
  if (B.ncp_ready) return;
  cudaStream_t s = B.P.stream;
  const int K = B.ninst;
  std::vector<int64_t> row0, tw0, pk0;
  std::vector<int> L, inst, col0(K + 1, 0);
  std::vector<double> tw;
  std::vector<std::pair<int, int64_t>> tabs;  // (length, offset) of the twiddle tables
  int64_t pkoff = 0;
  for (int k = 0; k < K; ++k) {
    const InstGeom &g = B.hg[k];
    AIRT_REQUIRE(g.nA == 0 || g.p >= 2, "NCP: instance %d has fewer than 2 rays per projection", k);
    int64_t toff = -1;
    for (auto &t : tabs)
      if (t.first == g.p) toff = t.second;
    if (toff < 0 && g.nA > 0) {
      toff = (int64_t)tw.size();
      const std::vector<double> t = ncp_twiddles(g.p);
      tw.insert(tw.end(), t.begin(), t.end());
      tabs.push_back({g.p, toff});
    }
    col0[k + 1] = col0[k] + g.nA;
    for (int c = 0; c < g.nA; ++c) {
      row0.push_back(B.row_off[k] + (int64_t)c * g.p);
      L.push_back(g.p);
      tw0.push_back(toff);
      pk0.push_back(pkoff);
      inst.push_back(k);
      pkoff += g.p / 2;
    }
  }
  B.ncols = (int)row0.size();
  const size_t nc = std::max<size_t>(row0.size(), 1);
  B.ncp_row0.ensure(nc);
  B.ncp_tw0.ensure(nc);
  B.ncp_pk0.ensure(nc);
  B.ncp_L.ensure(nc);
  B.ncp_inst.ensure(nc);
  if (!row0.empty()) {
    B.ncp_row0.upload(row0.data(), row0.size(), s);
    B.ncp_tw0.upload(tw0.data(), tw0.size(), s);
    B.ncp_pk0.upload(pk0.data(), pk0.size(), s);
    B.ncp_L.upload(L.data(), L.size(), s);
    B.ncp_inst.upload(inst.data(), inst.size(), s);
  }
  B.ncp_col0.upload(col0.data(), col0.size(), s);
  if (tw.empty()) B.ncp_tw.ensure(1);
  else B.ncp_tw.upload(tw.data(), tw.size(), s);
  B.ncp_pk.ensure(std::max<int64_t>(pkoff, 1));
  B.ncp_ccol.ensure(nc);
  AIRT_CHECK_CUDA(cudaStreamSynchronize(s));
  B.ncp_ready = true;
}
}  // namespace

// SIRT over the whole batch with per-instance relaxpar and a per-instance
// stopping rule (rule: AIRT_STOP_NONE, DP, ME or NCP; taud_host per
// instance for DP / ME; ncp_smooth values for NCP).
void batch_sirt(Batch &B, int method, const double *lam_host, const double *d_b, int rule,
                const double *taud_host, int ncp_smooth, int64_t kmax, int lbk, double lb, int ubk,
                double ub, const double *d_x0, double *d_x, int64_t *finaliter, int *stoprule,
                double *gpu_ms) {
  Problem &P = B.P;
  cudaStream_t s = P.stream;
  const int K = B.ninst;
  AIRT_REQUIRE(kmax >= 0 && kmax < INT32_MAX, "kmax out of range");
  AIRT_REQUIRE(rule == AIRT_STOP_NONE || rule == AIRT_STOP_DP || rule == AIRT_STOP_ME ||
                   rule == AIRT_STOP_NCP,
               "The chosen stopping rule is not valid.");
  AIRT_REQUIRE((rule != AIRT_STOP_DP && rule != AIRT_STOP_ME) || taud_host,
               "For stopping rules DP and ME a taudelta per instance must be given.");
  AIRT_REQUIRE(rule != AIRT_STOP_NCP || (ncp_smooth >= 1 && ncp_smooth <= 4096),
               "NCP: ncp_smooth must be in 1..4096");
  const bool me = rule == AIRT_STOP_ME, ncp = rule == AIRT_STOP_NCP;
  if (ncp) batch_ncp_setup(B);
  cudaEvent_t t0, t1;
  AIRT_CHECK_CUDA(cudaEventCreate(&t0));
  AIRT_CHECK_CUDA(cudaEventCreate(&t1));
  batch_tune(B);
  AIRT_CHECK_CUDA(cudaEventRecord(t0, s));
  batch_weights(B, method);
  P.x64.ensure(P.n);
  P.x32.ensure(P.n);
  P.mr32.ensure(P.m);
  B.rsq.ensure(P.m);
  B.nrm2.ensure(K);
  B.stop.ensure(K);
  B.iters.ensure(K);
  B.rule.ensure(K);
  B.resn_last.ensure(K);
  B.lam.upload(lam_host, K, s);
  if (taud_host && (rule == AIRT_STOP_DP || me)) B.taud.upload(taud_host, K, s);
  if (me || ncp) {
    B.rprev.ensure(P.m);
    AIRT_CHECK_CUDA(cudaMemsetAsync(B.rprev.p, 0, P.m * sizeof(double), s));
  }
  if (me) {
    B.pp.ensure(P.m);
    B.ppr.ensure(P.m);
    B.p2.ensure(K);
    B.pr.ensure(K);
  }
  if (ncp) {
    const std::vector<double> inf((size_t)K * ncp_smooth, INFINITY);
    B.ncp_dk.upload(inf.data(), inf.size(), s);
  }
  if (d_x0)
    AIRT_CHECK_CUDA(cudaMemcpyAsync(P.x64.p, d_x0, P.n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  else
    AIRT_CHECK_CUDA(cudaMemsetAsync(P.x64.p, 0, P.n * sizeof(double), s));
  k_copy_f32<<<grid_for(P.n, 256), 256, 0, s>>>(P.n, P.x64.p, P.x32.p);
  AIRT_CHECK_CUDA(cudaMemsetAsync(B.stop.p, 0, K * sizeof(int), s));
  AIRT_CHECK_CUDA(cudaMemsetAsync(B.iters.p, 0, K * sizeof(int), s));
  AIRT_CHECK_CUDA(cudaMemsetAsync(B.rule.p, 0, K * sizeof(int), s));
  build_tiles(B, B.stop.p);
  BFwd fo{d_b, P.M.p, P.mr32.p, B.rsq.p, B.inst_row.p, B.stop.p, 0,
          (me || ncp) ? B.rprev.p : nullptr, me ? B.pp.p : nullptr, me ? B.ppr.p : nullptr};
  BUpd uo{P.D.p, B.lam.p, P.x64.p, P.x32.p, B.inst_col.p, B.stop.p, lbk, ubk, lb, ub, 0};
  BCtrl co{rule, (rule == AIRT_STOP_DP || me) ? B.taud.p : nullptr, me ? B.p2.p : nullptr,
           me ? B.pr.p : nullptr, ncp ? B.ncp_ccol.p : nullptr, ncp ? B.ncp_col0.p : nullptr,
           ncp ? B.ncp_dk.p : nullptr, ncp_smooth};
  const bool poll = rule != AIRT_STOP_NONE;
  B.active.ensure(1);
  AIRT_CHECK_CUDA(cudaMemcpyAsync(B.active.p, &K, sizeof(int), cudaMemcpyHostToDevice, s));
  // forward pass, NCP periodograms, then per instance the norm and the rule
  auto fwd_step = [&](int initial) {
    fwd_classes(B, fo);
    if (ncp && B.ncols > 0) {
      k_batch_ncp_power<<<B.ncols, 128, 0, s>>>(B.ncp_row0.p, B.ncp_L.p, B.ncp_tw0.p, B.ncp_pk0.p,
                                                B.ncp_inst.p, B.stop.p, B.rprev.p, B.ncp_tw.p,
                                                B.ncp_pk.p);
      k_batch_ncp_col<<<B.ncols, 256, 0, s>>>(B.ncp_L.p, B.ncp_pk0.p, B.ncp_inst.p, B.stop.p,
                                              B.ncp_pk.p, B.ncp_ccol.p);
    }
    k_batch_step<<<K, 256, 0, s>>>(B.d_row_off.p, B.rsq.p, me ? B.pp.p : nullptr,
                                   me ? B.ppr.p : nullptr, me ? B.p2.p : nullptr,
                                   me ? B.pr.p : nullptr, initial, kmax, co, B.stop.p, B.iters.p,
                                   B.rule.p, B.resn_last.p, B.active.p, B.tcount.p);
  };
  auto iteration = [&]() {
    bwd_classes(B, uo);
    fwd_step(0);
    build_tiles_after_step(B, B.stop.p);
  };
  fwd_step(1);
  AIRT_LAUNCH_CHECK();
  build_tiles_after_step(B, B.stop.p);
  // A chunk of iterations is captured once as a CUDA graph and replayed:
  // every argument is fixed for the solve and the loop state lives in device
  // memory.  The host reads the active count of chunk c once chunk c+2 is
  // queued (lagged poll), so the device never idles on the poll.
  const int64_t chunk = 8;
  const int lag = 2;
  cudaGraphExec_t gexec = nullptr;
  if (kmax >= chunk) {
    cudaGraph_t g = nullptr;
    AIRT_CHECK_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    for (int64_t j = 0; j < chunk; ++j) iteration();
    const cudaError_t ec = cudaStreamEndCapture(s, &g);
    if (ec == cudaSuccess && g) {
      if (cudaGraphInstantiate(&gexec, g, 0) != cudaSuccess) gexec = nullptr;
      cudaGraphDestroy(g);
    }
    cudaGetLastError();
  }
  if (!P.h_state) AIRT_CHECK_CUDA(cudaMallocHost(&P.h_state, 3 * sizeof(SirtState)));
  int *hact = reinterpret_cast<int *>(P.h_state);  // 3 poll slots in the pinned mirror
  cudaEvent_t ev[3];
  for (int q = 0; q < 3; ++q) AIRT_CHECK_CUDA(cudaEventCreateWithFlags(&ev[q], cudaEventDisableTiming));
  int64_t c = 0;
  for (int64_t it = 1; it <= kmax; ++c) {
    const int64_t cnt = std::min<int64_t>(chunk, kmax - it + 1);
    if (cnt == chunk && gexec) {
      AIRT_CHECK_CUDA(cudaGraphLaunch(gexec, s));
    } else {
      for (int64_t j = 0; j < cnt; ++j) iteration();
    }
    AIRT_LAUNCH_CHECK();
    it += cnt;
    if (!poll) continue;
    AIRT_CHECK_CUDA(cudaMemcpyAsync(hact + (c % 3), B.active.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    AIRT_CHECK_CUDA(cudaEventRecord(ev[c % 3], s));
    if (c >= lag) {
      AIRT_CHECK_CUDA(cudaEventSynchronize(ev[(c - lag) % 3]));
      if (hact[(c - lag) % 3] == 0) break;
    }
  }
  for (int q = 0; q < 3; ++q) cudaEventDestroy(ev[q]);
  if (gexec) cudaGraphExecDestroy(gexec);
  AIRT_CHECK_CUDA(cudaEventRecord(t1, s));
  AIRT_CHECK_CUDA(cudaMemcpyAsync(d_x, P.x64.p, P.n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  std::vector<int> hit(K), hrule(K);
  AIRT_CHECK_CUDA(cudaMemcpyAsync(hit.data(), B.iters.p, K * sizeof(int), cudaMemcpyDeviceToHost, s));
  AIRT_CHECK_CUDA(cudaMemcpyAsync(hrule.data(), B.rule.p, K * sizeof(int), cudaMemcpyDeviceToHost, s));
  AIRT_CHECK_CUDA(cudaStreamSynchronize(s));
  float ms = 0;
  cudaEventElapsedTime(&ms, t0, t1);
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  for (int k = 0; k < K; ++k) {
    if (finaliter) finaliter[k] = hit[k];
    if (stoprule) stoprule[k] = hrule[k];
  }
  if (gpu_ms) *gpu_ms = ms;
}

// x = D .* A'(M .* b) per instance: the first SIRT iterate from x0 = 0 with
// relaxpar 1 and no bounds, in one transpose pass (the residual of x0 = 0 is
// b itself, so the forward pass of a one-iteration SIRT call is skipped).
void batch_backproject(Batch &B, int method, const double *d_b, double *d_x, double *gpu_ms) {
  Problem &P = B.P;
  cudaStream_t s = P.stream;
  const int K = B.ninst;
  cudaEvent_t t0, t1;
  AIRT_CHECK_CUDA(cudaEventCreate(&t0));
  AIRT_CHECK_CUDA(cudaEventCreate(&t1));
  batch_tune(B);
  AIRT_CHECK_CUDA(cudaEventRecord(t0, s));
  batch_weights(B, method);
  P.x64.ensure(P.n);
  P.x32.ensure(P.n);
  P.mr32.ensure(P.m);
  B.stop.ensure(K);
  B.lam.ensure(K);
  const std::vector<double> ones(K, 1.0);
  B.lam.upload(ones.data(), K, s);
  AIRT_CHECK_CUDA(cudaMemsetAsync(B.stop.p, 0, K * sizeof(int), s));
  AIRT_CHECK_CUDA(cudaMemsetAsync(P.x64.p, 0, P.n * sizeof(double), s));
  build_tiles(B, B.stop.p);
  k_batch_mb<<<grid_for(P.m, 256), 256, 0, s>>>(P.m, P.M.p, d_b, P.mr32.p);
  AIRT_LAUNCH_CHECK();
  BUpd uo{P.D.p, B.lam.p, P.x64.p, P.x32.p, B.inst_col.p, B.stop.p, 0, 0, 0.0, 0.0, 0};
  bwd_classes(B, uo);
  AIRT_CHECK_CUDA(cudaEventRecord(t1, s));
  AIRT_CHECK_CUDA(cudaMemcpyAsync(d_x, P.x64.p, P.n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  AIRT_CHECK_CUDA(cudaStreamSynchronize(s));
  float ms = 0;
  cudaEventElapsedTime(&ms, t0, t1);
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  if (gpu_ms) *gpu_ms = ms;
}

// ---------------------------------------------------------------- Kaczmarz
namespace {
// Level schedule of every instance's kaczmarz order (rows with nonzero norm,
// ascending; art.m:188), one warp per instance: level(row) = 1 + max level
// of the earlier steps touching one of its pixels (last[] holds the latest
// level per pixel, -1 initially).  Rows with zero norm get level -1.
__global__ void k_inst_levels(int ninst, const int64_t *__restrict__ roff, const int64_t *__restrict__ rp,
                              const int *__restrict__ ci, const double *__restrict__ nrm, int *__restrict__ last,
                              int *__restrict__ level, int *__restrict__ nlev) {
  const int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (k >= ninst) return;
  int maxl = -1;
  for (int64_t r = roff[k]; r < roff[k + 1]; ++r) {
    if (!(nrm[r] > 0)) {
      if (lane == 0) level[r] = -1;
      continue;
    }
    int L = 0;
    for (int64_t e = rp[r] + lane; e < rp[r + 1]; e += 32) L = max(L, last[ci[e]] + 1);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) L = max(L, __shfl_xor_sync(0xffffffffu, L, o));
    __syncwarp();
    for (int64_t e = rp[r] + lane; e < rp[r + 1]; e += 32) last[ci[e]] = L;
    __syncwarp();
    if (lane == 0) level[r] = L;
    maxl = max(maxl, L);
  }
  if (lane == 0) nlev[k] = maxl + 1;
}

// Steps per level: lev_ptr[base_k + L + 1] counts instance k's rows of
// level L (base_k = roff[k] + k; lev_ptr starts at zero).
__global__ void k_level_hist(int64_t m, const int64_t *__restrict__ roff, const int *__restrict__ level,
                             const int *__restrict__ inst_row, int *__restrict__ lev_ptr) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < m; r += (int64_t)gridDim.x * blockDim.x) {
    const int L = level[r];
    if (L >= 0) {
      const int k = inst_row[r];
      atomicAdd(lev_ptr + roff[k] + k + L + 1, 1);
    }
  }
}

// Inclusive scan of each instance's level counts (one thread per instance)
// and a copy as fill cursors.
__global__ void k_level_scan(int ninst, const int64_t *__restrict__ roff, const int *__restrict__ nlev,
                             int *__restrict__ lev_ptr, int *__restrict__ cursor) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ninst) return;
  int *p = lev_ptr + roff[k] + k;
  int *c = cursor + roff[k] + k;
  int run = (int)roff[k];  // steps of instance k start at its first row
  p[0] = run;
  c[0] = run;
  for (int L = 0; L < nlev[k]; ++L) {
    run += p[L + 1];
    p[L + 1] = run;
    c[L + 1] = run;
  }
}

__global__ void k_level_fill(int64_t m, const int64_t *__restrict__ roff, const int *__restrict__ level,
                             const int *__restrict__ inst_row, int *__restrict__ cursor, int *__restrict__ steps) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < m; r += (int64_t)gridDim.x * blockDim.x) {
    const int L = level[r];
    if (L >= 0) {
      const int k = inst_row[r];
      steps[atomicAdd(cursor + roff[k] + k + L, 1)] = (int)r;
    }
  }
}

constexpr int kBatchKaczCache = 6;  // gathered x values a lane keeps for the update

// Kaczmarz sweeps of one instance per CTA over its level schedule: the steps
// of a level touch disjoint pixels and run one per warp (fixed lane order and
// shuffle tree); a block barrier separates levels, so every pixel sees the
// update sequence of the sequential sweep (art.m:248-285).
__global__ void __launch_bounds__(512)
    k_batch_kacz_levels(const int64_t *__restrict__ roff, const int *__restrict__ lev_ptr,
                        const int *__restrict__ nlev, const int *__restrict__ steps,
                        const int64_t *__restrict__ rp, const int *__restrict__ ci, const float *__restrict__ rv,
                        const double *__restrict__ b, const double *__restrict__ nrm, double lam, int lbk,
                        double lb, int ubk, double ub, int sweeps, double *__restrict__ x) {
  const int k = blockIdx.x;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const int *lp = lev_ptr + roff[k] + k;
  const int nl = nlev[k];
  for (int sw = 0; sw < sweeps; ++sw) {
    for (int L = 0; L < nl; ++L) {
      const int q1 = lp[L + 1];
      for (int q = lp[L] + warp; q < q1; q += nw) {
        const int row = steps[q];
        const int64_t s0 = rp[row], s1 = rp[row + 1];
        const int64_t e0 = s0 + lane;
        // the first kBatchKaczCache gathers per lane are issued together and
        // kept for the update (no other step of the level touches these
        // pixels); the FMAs keep the order of the plain strided loop
        double cx[kBatchKaczCache];
#pragma unroll
        for (int u = 0; u < kBatchKaczCache; ++u)
          cx[u] = e0 + 32 * u < s1 ? x[ci[e0 + 32 * u]] : 0.0;
        double acc = 0.0;
#pragma unroll
        for (int u = 0; u < kBatchKaczCache; ++u)
          if (e0 + 32 * u < s1) acc = fma((double)rv[e0 + 32 * u], cx[u], acc);
        for (int64_t e = e0 + 32 * kBatchKaczCache; e < s1; e += 32)
          acc = fma((double)rv[e], x[ci[e]], acc);
        acc = warp_sum(acc);
        const double c = __ddiv_rn(__dmul_rn(lam, __dsub_rn(b[row], acc)), nrm[row]);
#pragma unroll
        for (int u = 0; u < kBatchKaczCache; ++u)
          if (e0 + 32 * u < s1) {
            double v = __dadd_rn(cx[u], __dmul_rn(c, (double)rv[e0 + 32 * u]));
            if (lbk) v = fmax(v, lb);
            if (ubk) v = fmin(v, ub);
            x[ci[e0 + 32 * u]] = v;
          }
        for (int64_t e = e0 + 32 * kBatchKaczCache; e < s1; e += 32) {
          const int j = ci[e];
          double v = __dadd_rn(x[j], __dmul_rn(c, (double)rv[e]));
          if (lbk) v = fmax(v, lb);
          if (ubk) v = fmin(v, ub);
          x[j] = v;
        }
      }
      __syncthreads();
    }
  }
}

}  // namespace

void batch_kaczmarz(Batch &B, const double *d_b, int64_t sweeps, double lam, int lbk, double lb,
                    int ubk, double ub, double *d_x, double *gpu_ms) {
  Problem &P = B.P;
  cudaStream_t s = P.stream;
  AIRT_REQUIRE(sweeps >= 0 && sweeps < INT32_MAX, "sweeps out of range");
  cudaEvent_t t0, t1;
  AIRT_CHECK_CUDA(cudaEventCreate(&t0));
  AIRT_CHECK_CUDA(cudaEventCreate(&t1));
  P.w1.ensure(P.m > P.n ? P.m : P.n);
  row_sums_sq(P, P.w1.p);
  // x0 = 0 is feasible for lb <= 0 <= ub, so the whole-vector clamp after the
  // first row step (art.m:279-284) only matters on each row's support.
  AIRT_REQUIRE((lbk == 0 || lb <= 0) && (ubk == 0 || ub >= 0),
               "batched Kaczmarz starts from x0 = 0 and needs lbound <= 0 <= ubound");
  if (!B.kz_ready) {
    // level schedules, once per batch (the pattern and the row norms never change)
    const int K = B.ninst;
    DevBuf<int> last, level, cursor;
    last.ensure(P.n);
    level.ensure(P.m);
    cursor.ensure(P.m + K + 1);
    B.kz_lev_ptr.ensure(P.m + K + 1);
    B.kz_steps.ensure(P.m > 0 ? P.m : 1);
    B.kz_nlev.ensure(K);
    AIRT_CHECK_CUDA(cudaMemsetAsync(last.p, 0xff, P.n * sizeof(int), s));  // -1
    AIRT_CHECK_CUDA(cudaMemsetAsync(B.kz_lev_ptr.p, 0, (P.m + K + 1) * sizeof(int), s));
    k_inst_levels<<<(K + 3) / 4, 128, 0, s>>>(K, B.d_row_off.p, P.rp.p, P.ci.p, P.w1.p, last.p, level.p,
                                              B.kz_nlev.p);
    k_level_hist<<<grid_for(P.m, 256), 256, 0, s>>>(P.m, B.d_row_off.p, level.p, B.inst_row.p, B.kz_lev_ptr.p);
    k_level_scan<<<(K + 127) / 128, 128, 0, s>>>(K, B.d_row_off.p, B.kz_nlev.p, B.kz_lev_ptr.p, cursor.p);
    k_level_fill<<<grid_for(P.m, 256), 256, 0, s>>>(P.m, B.d_row_off.p, level.p, B.inst_row.p, cursor.p,
                                                    B.kz_steps.p);
    AIRT_LAUNCH_CHECK();
    AIRT_CHECK_CUDA(cudaStreamSynchronize(s));
    B.kz_ready = true;
  }
  AIRT_CHECK_CUDA(cudaEventRecord(t0, s));
  AIRT_CHECK_CUDA(cudaMemsetAsync(d_x, 0, P.n * sizeof(double), s));
  k_batch_kacz_levels<<<B.ninst, 512, 0, s>>>(B.d_row_off.p, B.kz_lev_ptr.p, B.kz_nlev.p, B.kz_steps.p, P.rp.p,
                                              P.ci.p, P.rv.p, d_b, P.w1.p, lam, lbk, lb, ubk, ub, (int)sweeps,
                                              d_x);
  AIRT_LAUNCH_CHECK();
  AIRT_CHECK_CUDA(cudaEventRecord(t1, s));
  AIRT_CHECK_CUDA(cudaEventSynchronize(t1));
  float ms = 0;
  cudaEventElapsedTime(&ms, t0, t1);
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  if (gpu_ms) *gpu_ms = ms;
}

}  // namespace airt
