// Device ray tracer of the paralleltomo / fanlineartomo / fancurvedtomo /
// seismictomo line model.
//
// One ray is one row of A.  The reference (testprobs/paralleltomo.m:207-263,
// testprobs/fanlineartomo.m:271-318, testprobs/seismictomo.m:194-249) computes
// the crossings with all x = const and y = const grid lines, sorts them by the
// line parameter t (stable, NaN last), keeps the points inside the square,
// drops a point whose successor is within 1e-10 in both coordinates, and turns
// consecutive points into (pixel, length) pairs.  Both crossing sequences are
// monotone in t, so the sort is replaced here by a two-way merge that takes the
// x-crossing first on equal t -- the same order the stable sort gives for every
// point that survives the box filter (non-finite t values never survive it).
// All FP64 arithmetic uses explicit round-to-nearest intrinsics, so no
// multiply-add is contracted and the points, lengths and pixel indices are
// bit-identical to the FP64 CPU restatement.
#pragma once

#include "common.cuh"

namespace airt {

struct Ray {
  double x0t, y0t, a, b;
};

// Ray parameters, paralleltomo.m:195-200 / fanlineartomo.m:230-257 /
// seismictomo.m:188-200.
__device__ __forceinline__ Ray ray_of(const RayGeom &g, int64_t r) {
  const int i = (int)(r / g.p);
  const int j = (int)(r - (int64_t)i * g.p);
  Ray q;
  if (g.kind == GEO_SEISMIC) {
    // from source i to receiver j (t = 1 at the receiver)
    q.x0t = g.src_x[i];
    q.y0t = g.src_y[i];
    q.a = __dsub_rn(g.rcv_x[j], q.x0t);
    q.b = __dsub_rn(g.rcv_y[j], q.y0t);
    return q;
  }
  const double c = g.cos_t[i], s = g.sin_t[i];
  if (g.kind == GEO_PARALLEL) {
    const double x0 = g.offsets[j];
    q.x0t = __dsub_rn(__dmul_rn(c, x0), __dmul_rn(s, 0.0));
    q.y0t = __dadd_rn(__dmul_rn(s, x0), __dmul_rn(c, 0.0));
    q.a = -s;
    q.b = c;
  } else {
    q.x0t = __dadd_rn(__dmul_rn(c, 0.0), __dmul_rn(-s, g.R));
    q.y0t = __dadd_rn(__dmul_rn(s, 0.0), __dmul_rn(c, g.R));
    const double ab1 = __ddiv_rn(-q.x0t, g.R);
    const double ab2 = __ddiv_rn(-q.y0t, g.R);
    const double cw = g.cos_w[j], sw = g.sin_w[j];
    q.a = __dadd_rn(__dmul_rn(cw, ab1), __dmul_rn(-sw, ab2));
    q.b = __dadd_rn(__dmul_rn(sw, ab1), __dmul_rn(cw, ab2));
  }
  return q;
}

// Index range [lo, hi] (within 0..N) of the grid lines u = i - h whose
// crossing with the ray can lie inside the square.  The crossing of line i
// has the other coordinate v(i) = v0 + (dv/du)(i - h - u0) (u0, v0: the ray
// origin; du, dv: its direction); lines whose exact v(i) is outside
// [-h - kBoxSlack, h + kBoxSlack] are left out.  Their computed points differ
// from the exact ones by far less than kBoxSlack (a few ulps of values of
// order N), so the box test below would reject every one of them: leaving
// them out changes no output, it only saves their divisions.  One index of
// margin on each side absorbs the rounding of the bounds themselves.
constexpr double kBoxSlack = 1e-6;

__device__ __forceinline__ void crossing_range(int N, double h, double u0, double v0, double du,
                                               double dv, int &lo, int &hi) {
  lo = 0;
  hi = N;
  if (dv == 0.0) {  // v(i) = v0 for every line
    if (fabs(v0) > h + kBoxSlack) hi = -1;
    return;
  }
  const double r = du / dv;
  const double i1 = h + u0 + r * (-h - kBoxSlack - v0);
  const double i2 = h + u0 + r * (h + kBoxSlack - v0);
  if (!(isfinite(i1) && isfinite(i2))) return;
  const double l = fmax(0.0, floor(fmin(i1, i2)) - 1.0);
  const double u = fmin((double)N, ceil(fmax(i1, i2)) + 1.0);
  if (l > u) {
    hi = -1;
    return;
  }
  lo = (int)l;
  hi = (int)u;
}

// Traces one ray and calls seg(col, len) for each segment in ray order
// (before duplicate merging).  col is the 0-based column-major pixel index.
template <class Seg>
__device__ __forceinline__ void trace_segments(int N, const Ray &q, bool exclude_top_right,
                                               Seg &&seg) {
  const double h = 0.5 * (double)N;
  if (exclude_top_right && ((q.b == 0.0 && fabs(__dsub_rn(q.y0t, h)) < 1e-15) ||
                            (q.a == 0.0 && fabs(__dsub_rn(q.x0t, h)) < 1e-15)))
    return;
  // x-crossing sequence in ascending t, restricted to lines whose crossing
  // can be inside the square
  int nx = 0, ix = 0, sx = 1;
  if (q.a != 0.0) {
    int lo, hi;
    crossing_range(N, h, q.x0t, q.y0t, q.a, q.b, lo, hi);
    nx = hi >= lo ? hi - lo + 1 : 0;
    if (q.a > 0.0) { ix = lo; sx = 1; }
    else { ix = hi; sx = -1; }
  }
  int ny = 0, iy = 0, sy = 1;
  if (q.b != 0.0) {
    int lo, hi;
    crossing_range(N, h, q.y0t, q.x0t, q.b, q.a, lo, hi);
    ny = hi >= lo ? hi - lo + 1 : 0;
    if (q.b > 0.0) { iy = lo; sy = 1; }
    else { iy = hi; sy = -1; }
  }
  int cx = 0, cy = 0;
  double tx = 0.0, ty = 0.0;
  if (nx) tx = __ddiv_rn(__dsub_rn((double)ix - h, q.x0t), q.a);
  if (ny) ty = __ddiv_rn(__dsub_rn((double)iy - h, q.y0t), q.b);

  bool have_pend = false, have_last = false;
  double px = 0, py = 0, lx = 0, ly = 0;
  while (cx < nx || cy < ny) {
    // The next point comes from the x family (x-crossing first on equal t)
    // or the y family.  The step is written with selected operands, so that
    // the lanes of a warp, whose rays sit at different crossings, run one
    // multiply-add and one division per step instead of both branches.
    const bool takex = cy >= ny || (cx < nx && tx <= ty);
    const double t = takex ? tx : ty;
    const double fixed = (double)(takex ? ix : iy) - h;
    const double other = __dadd_rn(__dmul_rn(takex ? q.b : q.a, t), takex ? q.y0t : q.x0t);
    const double xx = takex ? fixed : other;
    const double yy = takex ? other : fixed;
    if (takex) {
      ++cx;
      ix += sx;
    } else {
      ++cy;
      iy += sy;
    }
    // the family's next crossing parameter (unused once the family is spent)
    const double tn = __ddiv_rn(__dsub_rn((double)(takex ? ix : iy) - h, takex ? q.x0t : q.y0t),
                                takex ? q.a : q.b);
    if (takex) tx = tn;
    else ty = tn;
    if (!(xx >= -h && xx <= h && yy >= -h && yy <= h)) continue;
    if (have_pend) {
      const bool close = fabs(__dsub_rn(xx, px)) <= 1e-10 && fabs(__dsub_rn(yy, py)) <= 1e-10;
      if (!close) {
        if (have_last) {
          const double dx = __dsub_rn(px, lx), dy = __dsub_rn(py, ly);
          const double len = __dsqrt_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)));
          const double xm = __dadd_rn(__dmul_rn(0.5, __dadd_rn(lx, px)), h);
          const double ym = __dadd_rn(__dmul_rn(0.5, __dadd_rn(ly, py)), h);
          const int col = (int)floor(xm) * N + (N - 1 - (int)floor(ym));
          seg(col, len);
        }
        lx = px;
        ly = py;
        have_last = true;
      }
    }
    px = xx;
    py = yy;
    have_pend = true;
  }
  if (have_pend && have_last) {
    const double dx = __dsub_rn(px, lx), dy = __dsub_rn(py, ly);
    const double len = __dsqrt_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)));
    const double xm = __dadd_rn(__dmul_rn(0.5, __dadd_rn(lx, px)), h);
    const double ym = __dadd_rn(__dmul_rn(0.5, __dadd_rn(ly, py)), h);
    const int col = (int)floor(xm) * N + (N - 1 - (int)floor(ym));
    seg(col, len);
  }
}

// Segments with duplicate pixels of the same ray merged, as MATLAB's
// sparse() sums duplicate (row, col) pairs (paralleltomo.m:300).  A straight
// ray meets a pixel in one segment; a duplicate can only come from a sliver
// segment at a grid corner, so a window of the last few entries suffices.
// emit(col, value) is called once per distinct pixel, in ray order of first
// appearance, with the FP64 sum.
constexpr int kMergeWindow = 4;

// The window of the last kMergeWindow distinct pixels (oldest at index 0).
struct MergeWindow {
  int wc[kMergeWindow];
  double wv[kMergeWindow];
  int cnt = 0;
  template <class Emit>
  __device__ __forceinline__ void add(int col, double len, Emit &&emit) {
#pragma unroll
    for (int k = 0; k < kMergeWindow; ++k)
      if (k < cnt && wc[k] == col) {
        wv[k] = __dadd_rn(wv[k], len);
        return;
      }
    if (cnt == kMergeWindow) {
      emit(wc[0], wv[0]);
#pragma unroll
      for (int k = 0; k + 1 < kMergeWindow; ++k) {
        wc[k] = wc[k + 1];
        wv[k] = wv[k + 1];
      }
      cnt = kMergeWindow - 1;
    }
#pragma unroll
    for (int k = 0; k < kMergeWindow; ++k)
      if (k == cnt) {
        wc[k] = col;
        wv[k] = len;
      }
    ++cnt;
  }
  template <class Emit>
  __device__ __forceinline__ void flush(Emit &&emit) {
#pragma unroll
    for (int k = 0; k < kMergeWindow; ++k)
      if (k < cnt) emit(wc[k], wv[k]);
  }
};

template <class Emit>
__device__ __forceinline__ void trace_entries(int N, const Ray &q, bool exclude_top_right,
                                              Emit &&emit) {
  MergeWindow w;
  trace_segments(N, q, exclude_top_right, [&](int col, double len) { w.add(col, len, emit); });
  w.flush(emit);
}

// ---- one ray traced by two threads
// trace_segments_part(part = 0 or 1) emits the first or the second half of
// the segments trace_segments emits, so that two threads can share a long
// ray.  The split is at the middle crossing S of the family with more
// crossings (the primary family), provided S is clean: no crossing of the
// other family lies within kSplitGap of it in t.  Then S is a kept point
// (its successor is not within 1e-10), the segment ending at S is emitted by
// part 0 as its last one and the segment starting at S by part 1 as its
// first, every other point has the same neighbours as in the whole trace,
// and the two halves lie on either side of one grid line, so no pixel
// appears in both (the duplicate merge of trace_entries stays within a
// half).  Part 0 runs the merge from the ray's start and stops after S; part
// 1 starts from S as the pending point with the other family's position
// found from t(S) (an estimate, then exact comparisons of crossing
// parameters).  Rays too short to be worth splitting, or without a clean
// crossing near the middle, go to part 0 whole (part 1 emits nothing).
constexpr int kSplitMin = 48;        // crossings (both families) of a ray worth splitting
constexpr double kSplitGap = 1e-7;   // minimum |t| distance of S to the other family

__device__ __forceinline__ double cross_t(int i, double h, double o, double d) {
  return __ddiv_rn(__dsub_rn((double)i - h, o), d);
}

template <class Seg>
__device__ __forceinline__ void trace_segments_part(int N, const Ray &q, bool exclude_top_right, int part,
                                                    Seg &&seg) {
  const double h = 0.5 * (double)N;
  if (exclude_top_right && ((q.b == 0.0 && fabs(__dsub_rn(q.y0t, h)) < 1e-15) ||
                            (q.a == 0.0 && fabs(__dsub_rn(q.x0t, h)) < 1e-15)))
    return;
  int nx = 0, ix0 = 0, sx = 1;
  if (q.a != 0.0) {
    int lo, hi;
    crossing_range(N, h, q.x0t, q.y0t, q.a, q.b, lo, hi);
    nx = hi >= lo ? hi - lo + 1 : 0;
    if (q.a > 0.0) { ix0 = lo; sx = 1; }
    else { ix0 = hi; sx = -1; }
  }
  int ny = 0, iy0 = 0, sy = 1;
  if (q.b != 0.0) {
    int lo, hi;
    crossing_range(N, h, q.y0t, q.x0t, q.b, q.a, lo, hi);
    ny = hi >= lo ? hi - lo + 1 : 0;
    if (q.b > 0.0) { iy0 = lo; sy = 1; }
    else { iy0 = hi; sy = -1; }
  }
  // ---- the split: primary family P (more crossings), position mP of S,
  // position pQ of the first crossing of the other family after S
  bool split = false;
  const bool px_primary = nx >= ny;  // P = x family (ties: x first, as the merge)
  int mP = 0, pQ = 0;
  double tS = 0.0;
  if (nx + ny >= kSplitMin) {
    const int nP = px_primary ? nx : ny, nQ = px_primary ? ny : nx;
    const int iP0 = px_primary ? ix0 : iy0, sP = px_primary ? sx : sy;
    const int iQ0 = px_primary ? iy0 : ix0, sQ = px_primary ? sy : sx;
    const double oP = px_primary ? q.x0t : q.y0t, dP = px_primary ? q.a : q.b;
    const double oQ = px_primary ? q.y0t : q.x0t, dQ = px_primary ? q.b : q.a;
    for (int tryk = 0; tryk < 4 && !split; ++tryk) {
      const int m = nP / 2 + ((tryk & 1) ? -((tryk + 1) / 2) : (tryk / 2));
      if (m < 1 || m >= nP - 1) continue;
      const double t = cross_t(iP0 + m * sP, h, oP, dP);
      // Q position: crossings of Q before S in the merged order are those
      // with t_Q < t (P = x: x first on equal t) or t_Q <= t (P = y)
      int p = 0;
      if (nQ > 0) {
        const double est = __dmul_rn(__dsub_rn(__dadd_rn(__dadd_rn(h, oQ), __dmul_rn(dQ, t)), (double)iQ0),
                                     (double)sQ);
        p = (int)fmin(fmax(ceil(est), 0.0), (double)nQ);
        // exact adjustment (the sequence is increasing in t); bounded steps
        for (int it = 0; it < 4 && p > 0; ++it) {
          const double tb = cross_t(iQ0 + (p - 1) * sQ, h, oQ, dQ);
          if (px_primary ? tb < t : tb <= t) break;
          --p;
        }
        for (int it = 0; it < 4 && p < nQ; ++it) {
          const double ta = cross_t(iQ0 + p * sQ, h, oQ, dQ);
          if (px_primary ? ta >= t : ta > t) break;
          ++p;
        }
        // clean and certain: the Q neighbours of S are on the right sides of
        // t(S) and farther than kSplitGap from it
        const double tb = p > 0 ? cross_t(iQ0 + (p - 1) * sQ, h, oQ, dQ) : -INFINITY;
        const double ta = p < nQ ? cross_t(iQ0 + p * sQ, h, oQ, dQ) : INFINITY;
        if (!(tb < t - kSplitGap && ta > t + kSplitGap)) continue;
      }
      // S itself must lie inside the square (the box filter keeps it)
      const double fixed = (double)(iP0 + m * sP) - h;
      const double other = __dadd_rn(__dmul_rn(px_primary ? q.b : q.a, t), px_primary ? q.y0t : q.x0t);
      if (!(fixed > -h && fixed < h && other > -h && other < h)) continue;
      split = true;
      mP = m;
      pQ = p;
      tS = t;
    }
  }
  if (part == 1 && !split) return;
  // ---- loop state of this part
  int cx = 0, cy = 0, ix = ix0, iy = iy0;
  int endx = nx, endy = ny;  // positions at which the families stop
  bool have_pend = false, have_last = false;
  double px = 0, py = 0, lx = 0, ly = 0;
  if (split) {
    const int endP = mP + 1;  // part 0 takes S (position mP) last
    if (part == 0) {
      if (px_primary) { endx = endP; endy = pQ; }
      else { endy = endP; endx = pQ; }
    } else {
      if (px_primary) {
        cx = mP + 1;
        cy = pQ;
        px = (double)(ix0 + mP * sx) - h;
        py = __dadd_rn(__dmul_rn(q.b, tS), q.y0t);
      } else {
        cy = mP + 1;
        cx = pQ;
        py = (double)(iy0 + mP * sy) - h;
        px = __dadd_rn(__dmul_rn(q.a, tS), q.x0t);
      }
      ix = ix0 + cx * sx;
      iy = iy0 + cy * sy;
      have_pend = true;
    }
  }
  double tx = 0.0, ty = 0.0;
  if (cx < endx) tx = cross_t(ix, h, q.x0t, q.a);
  if (cy < endy) ty = cross_t(iy, h, q.y0t, q.b);
  while (cx < endx || cy < endy) {
    // the merge step of trace_segments, over this part's positions
    const bool takex = cy >= endy || (cx < endx && tx <= ty);
    const double t = takex ? tx : ty;
    const double fixed = (double)(takex ? ix : iy) - h;
    const double other = __dadd_rn(__dmul_rn(takex ? q.b : q.a, t), takex ? q.y0t : q.x0t);
    const double xx = takex ? fixed : other;
    const double yy = takex ? other : fixed;
    if (takex) {
      ++cx;
      ix += sx;
    } else {
      ++cy;
      iy += sy;
    }
    const double tn = __ddiv_rn(__dsub_rn((double)(takex ? ix : iy) - h, takex ? q.x0t : q.y0t),
                                takex ? q.a : q.b);
    if (takex) tx = tn;
    else ty = tn;
    if (!(xx >= -h && xx <= h && yy >= -h && yy <= h)) continue;
    if (have_pend) {
      const bool close = fabs(__dsub_rn(xx, px)) <= 1e-10 && fabs(__dsub_rn(yy, py)) <= 1e-10;
      if (!close) {
        if (have_last) {
          const double dx = __dsub_rn(px, lx), dy = __dsub_rn(py, ly);
          const double len = __dsqrt_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)));
          const double xm = __dadd_rn(__dmul_rn(0.5, __dadd_rn(lx, px)), h);
          const double ym = __dadd_rn(__dmul_rn(0.5, __dadd_rn(ly, py)), h);
          seg((int)floor(xm) * N + (N - 1 - (int)floor(ym)), len);
        }
        lx = px;
        ly = py;
        have_last = true;
      }
    }
    px = xx;
    py = yy;
    have_pend = true;
  }
  if (have_pend && have_last) {
    const double dx = __dsub_rn(px, lx), dy = __dsub_rn(py, ly);
    const double len = __dsqrt_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)));
    const double xm = __dadd_rn(__dmul_rn(0.5, __dadd_rn(lx, px)), h);
    const double ym = __dadd_rn(__dmul_rn(0.5, __dadd_rn(ly, py)), h);
    seg((int)floor(xm) * N + (N - 1 - (int)floor(ym)), len);
  }
}

// trace_entries over one part of a split ray (trace_segments_part): the
// merged entries of the whole ray are exactly the union of the two parts'.
template <class Emit>
__device__ __forceinline__ void trace_entries_part(int N, const Ray &q, bool exclude_top_right, int part,
                                                   Emit &&emit) {
  MergeWindow w;
  trace_segments_part(N, q, exclude_top_right, part, [&](int col, double len) { w.add(col, len, emit); });
  w.flush(emit);
}

// sphericaltomo (testprobs/sphericaltomo.m:203-224): sample k of a circle of
// radius rad about (xix, yiy) lands in the pixel (round(xx), round(yy)) of
// xx = (xix + rad*cos(k))/dx + ceil(N/2); returns its 0-based column-major
// index, or -1 outside the image.  round() rounds halves away from zero, as
// MATLAB's round does; the cosines and sines come from the host tables.
__device__ __forceinline__ int sphere_pixel(const RayGeom &g, double xix, double xiy, double rad,
                                            int64_t k) {
  const double xx =
      __dadd_rn(__ddiv_rn(__dadd_rn(xix, __dmul_rn(rad, g.cos_k[k])), g.dx), (double)g.center);
  const double yy =
      __dadd_rn(__ddiv_rn(__dadd_rn(xiy, __dmul_rn(rad, g.sin_k[k])), g.dx), (double)g.center);
  const double col = round(xx), row = round(yy);
  if (!(col > 0.0 && col <= (double)g.N && row > 0.0 && row <= (double)g.N)) return -1;
  return (g.N - (int)row) + ((int)col - 1) * g.N;
}

// The entries of row r for the linear operators (products and the SIRT
// residual): a straight ray's merged (pixel, length) pairs, or, for a circle,
// one (pixel, 2*pi*r/nPhi) pair per sample inside the image -- a pixel hit w
// times appears w times, which sums to the reference's w*2*pi*r/nPhi.
template <class Emit>
__device__ __forceinline__ void row_entries(const RayGeom &g, int64_t r, bool exclude_top_right,
                                            Emit &&emit) {
  if (g.kind == GEO_SPHERE) {
    const int i = (int)(r / g.p);
    const int n = (int)(r - (int64_t)i * g.p);
    const double xix = g.cos_t[i], xiy = g.sin_t[i], rad = g.radius[n], c = g.cscale[n];
    for (int64_t k = g.koff[n]; k < g.koff[n + 1]; ++k) {
      const int J = sphere_pixel(g, xix, xiy, rad, k);
      if (J >= 0) emit(J, c);
    }
    return;
  }
  trace_entries(g.N, ray_of(g, r), exclude_top_right, emit);
}

// row_entries for one of the two threads that share row r (part 0 or 1):
// straight rays are split by trace_entries_part; a circle goes to part 0.
template <class Emit>
__device__ __forceinline__ void row_entries_part(const RayGeom &g, int64_t r, bool exclude_top_right, int part,
                                                 Emit &&emit) {
  if (g.kind == GEO_SPHERE) {
    if (part == 0) row_entries(g, r, exclude_top_right, emit);
    return;
  }
  trace_entries_part(g.N, ray_of(g, r), exclude_top_right, part, emit);
}

}  // namespace airt
