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

template <class Emit>
__device__ __forceinline__ void trace_entries(int N, const Ray &q, bool exclude_top_right,
                                              Emit &&emit) {
  int wc[kMergeWindow];
  double wv[kMergeWindow];
  int cnt = 0;  // entries held in the window (oldest at index 0)
  trace_segments(N, q, exclude_top_right, [&](int col, double len) {
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
  });
#pragma unroll
  for (int k = 0; k < kMergeWindow; ++k)
    if (k < cnt) emit(wc[k], wv[k]);
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

}  // namespace airt
