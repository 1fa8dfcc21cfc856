// Learned warm start: a U-Net (levels x {conv3x3+ReLU, conv3x3+ReLU},
// 2x2 max-pool down, nearest 2x up + skip concatenation, 1x1 head) trained
// and evaluated with this project's own kernels.  No counterpart in the
// reference: its output only enters the solvers as x0 (sirt/sirt.m:5).
//
// Layout: activations NHWC BF16 ([pixel][channel], pixel = (b*H + h)*W + w),
// gradients FP32, weights FP32 masters [Cout][Kp] with a BF16 copy for the
// tensor cores (Kp = 9*Cin rounded up to 64, zero padded; K index
// (kh*3 + kw)*Cin + ci).  Every 3x3 convolution is a tcgen05 GEMM of
// umma.cuh whose A tiles are gathered straight from the NHWC activations
// (implicit GEMM, col(X) is never stored):
//   forward  Y[P][Co]  = relu(col(X)[P][Kp] * W[Co][Kp]^T + b)   (K/K-major)
//   dW^T     [Kp][Co] += col(X)^T * dYm   (both MN-major, split-K atomics
//                        written transposed straight into W's layout)
//   dX       [P][Ci]  += col(dYm)[P][Kq] * Wt[Ci][Kq]^T, the 3x3 convolution
//                        of dYm with the tap-flipped, transposed weights
//                        Wt[ci][(8-tap)*Co + co] = W[co][tap*Ci + ci].
// The first convolution (Cin = 1, not a multiple of 8 channels) keeps an
// explicit im2col.  The image (x(:), column-major N x N) maps to NHWC with
// h = column-major row.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <random>
#include <vector>

#include "common.cuh"
#include "umma.cuh"

namespace airt {

namespace {

constexpr int kT = 256;

// Grid-stride loop with 32-bit indices: every tensor of the network holds
// fewer than 2^30 elements (checked in unet_create), and 32-bit index
// decoding avoids the long 64-bit division sequences.
#define AIRT_FOR32(t, total) \
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < (total); t += gridDim.x * blockDim.x)

__device__ __forceinline__ void bf8_to_f(const uint4 &u, float (&f)[8]) {
  const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&u);
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const float2 t = __bfloat1622float2(h[i]);
    f[2 * i] = t.x;
    f[2 * i + 1] = t.y;
  }
}

__device__ __forceinline__ uint4 f_to_bf8(const float (&f)[8]) {
  uint4 u;
  __nv_bfloat162 *h = reinterpret_cast<__nv_bfloat162 *>(&u);
#pragma unroll
  for (int i = 0; i < 4; ++i) h[i] = __floats2bfloat162_rn(f[2 * i], f[2 * i + 1]);
  return u;
}

__device__ __forceinline__ void ld_f8(const float *p, float (&f)[8]) {
  const float4 a = reinterpret_cast<const float4 *>(p)[0], b = reinterpret_cast<const float4 *>(p)[1];
  f[0] = a.x, f[1] = a.y, f[2] = a.z, f[3] = a.w, f[4] = b.x, f[5] = b.y, f[6] = b.z, f[7] = b.w;
}

__device__ __forceinline__ void st_f8(float *p, const float (&f)[8]) {
  reinterpret_cast<float4 *>(p)[0] = make_float4(f[0], f[1], f[2], f[3]);
  reinterpret_cast<float4 *>(p)[1] = make_float4(f[4], f[5], f[6], f[7]);
}

// Per-channel sums over rows.  A 256-thread block walks its rows with
// thread t owning row offset t / C8 and channel group t % C8 (R = 256 / C8
// rows per pass, threads t >= R*C8 idle); the per-thread sums of 8 channels
// meet in shared memory and leave as one atomicAdd per channel.
__device__ __forceinline__ void colsum_flush(const float (&acc)[8], int C8, float *sh, float *out) {
  const int t = threadIdx.x, R = 256 / C8;
#pragma unroll
  for (int i = 0; i < 8; ++i) sh[i * 256 + t] = acc[i];
  __syncthreads();
  for (int c = t; c < C8 * 8; c += 256) {
    const int cg = c >> 3, i = c & 7;
    float a = 0.f;
    for (int r = 0; r < R; ++r) a += sh[i * 256 + r * C8 + cg];
    atomicAdd(out + c, a);
  }
}

__global__ void k_im2col(int B, int H, int W, int C, int Kp, const __nv_bfloat16 *__restrict__ X,
                         __nv_bfloat16 *__restrict__ col) {
  const int64_t total = (int64_t)B * H * W * Kp;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int kk = (int)(t % Kp);
    const int64_t p = t / Kp;
    __nv_bfloat16 v = __float2bfloat16(0.f);
    if (kk < 9 * C) {
      const int ci = kk % C, tap = kk / C;
      const int kh = tap / 3, kw = tap % 3;
      const int w = (int)(p % W), h = (int)((p / W) % H), b = (int)(p / ((int64_t)W * H));
      const int hh = h + kh - 1, ww = w + kw - 1;
      if (hh >= 0 && hh < H && ww >= 0 && ww < W) v = X[(((int64_t)b * H + hh) * W + ww) * C + ci];
    }
    col[t] = v;
  }
}

// Wt[ci][kq] = W[co][(8 - tap)*Ci + ci] for kq = tap*Co + co < 9*Co, else 0.
__global__ void k_flip_w(int Co, int Ci, int Kp, int Kq, const __nv_bfloat16 *__restrict__ w,
                         __nv_bfloat16 *__restrict__ wt) {
  const int64_t total = (int64_t)Ci * Kq;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int kq = (int)(t % Kq), ci = (int)(t / Kq);
    const int tap = kq / Co, co = kq - tap * Co;
    wt[t] = tap < 9 ? w[(int64_t)co * Kp + (8 - tap) * Ci + ci] : __float2bfloat16(0.f);
  }
}

__global__ void k_col2im(int B, int H, int W, int C, int Kp, const float *__restrict__ dcol,
                         float *__restrict__ dX) {
  const int64_t total = (int64_t)B * H * W * C;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int ci = (int)(t % C);
    const int64_t p = t / C;
    const int w = (int)(p % W), h = (int)((p / W) % H), b = (int)(p / ((int64_t)W * H));
    float acc = 0.f;
#pragma unroll
    for (int kh = 0; kh < 3; ++kh)
#pragma unroll
      for (int kw = 0; kw < 3; ++kw) {
        const int hs = h - kh + 1, ws = w - kw + 1;
        if (hs >= 0 && hs < H && ws >= 0 && ws < W)
          acc += dcol[(((int64_t)b * H + hs) * W + ws) * Kp + (kh * 3 + kw) * C + ci];
      }
    dX[t] += acc;
  }
}

// dYm = bf16(dY * (Y > 0)) and db += column sums (one block per 256 columns-slab)
// dYm = bf16(dY * (Y > 0)) and db[c] += sum over pixels of dYm[p][c], 8
// channels per thread (C a multiple of 8); each block owns a contiguous range
// of pixel rows.
__global__ void __launch_bounds__(256) k_relu_mask_colsum(int64_t P, int C, int64_t rows_per_block,
                                                          const float *__restrict__ dY,
                                                          const __nv_bfloat16 *__restrict__ Y,
                                                          __nv_bfloat16 *__restrict__ dYm,
                                                          float *__restrict__ db) {
  __shared__ float sh[8 * 256];
  const int C8 = C / 8, R = 256 / C8, t = threadIdx.x;
  const int64_t r0 = blockIdx.x * rows_per_block;
  const int64_t r1 = min(P, r0 + rows_per_block);
  float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  if (t < R * C8) {
    const int cg = t % C8;
    for (int64_t r = r0 + t / C8; r < r1; r += R) {
      const int64_t i = r * C + cg * 8;
      float d[8], y[8], m[8];
      ld_f8(dY + i, d);
      bf8_to_f(*reinterpret_cast<const uint4 *>(Y + i), y);
#pragma unroll
      for (int j = 0; j < 8; ++j) m[j] = y[j] > 0.f ? d[j] : 0.f;
      const uint4 u = f_to_bf8(m);
      *reinterpret_cast<uint4 *>(dYm + i) = u;
      bf8_to_f(u, m);
#pragma unroll
      for (int j = 0; j < 8; ++j) acc[j] += m[j];
    }
  }
  colsum_flush(acc, C8, sh, db);
}

// 2x2 max pool, 8 channels (16 bytes) per thread.
__global__ void k_pool(int B, int H, int W, int C, const __nv_bfloat16 *__restrict__ X,
                       __nv_bfloat16 *__restrict__ Y) {
  const int Ho = H / 2, Wo = W / 2, C8 = C / 8;
  AIRT_FOR32(t, B * Ho * Wo * C8) {
    const int cg = t % C8, q = t / C8;
    const int w = q % Wo, h = (q / Wo) % Ho, b = q / (Wo * Ho);
    float m[8], v[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) m[j] = -INFINITY;
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        bf8_to_f(*reinterpret_cast<const uint4 *>(X + (((int64_t)b * H + 2 * h + i) * W + 2 * w + k) * C + cg * 8), v);
#pragma unroll
        for (int j = 0; j < 8; ++j) m[j] = fmaxf(m[j], v[j]);
      }
    reinterpret_cast<uint4 *>(Y)[t] = f_to_bf8(m);
  }
}

// Gradient of the max pool: each window's gradient goes to its first maximal
// element (row-major window order); 8 channels per thread, every element of
// dX belongs to exactly one window.
__global__ void k_pool_back(int B, int H, int W, int C, const __nv_bfloat16 *__restrict__ X,
                            const float *__restrict__ dY, float *__restrict__ dX) {
  const int Ho = H / 2, Wo = W / 2, C8 = C / 8;
  AIRT_FOR32(t, B * Ho * Wo * C8) {
    const int cg = t % C8, q = t / C8;
    const int w = q % Wo, h = (q / Wo) % Ho, b = q / (Wo * Ho);
    int64_t off[4];
    float x[4][8], m[8], g[8];
    int arg[8];
#pragma unroll
    for (int pos = 0; pos < 4; ++pos) {
      off[pos] = (((int64_t)b * H + 2 * h + pos / 2) * W + 2 * w + pos % 2) * C + cg * 8;
      bf8_to_f(*reinterpret_cast<const uint4 *>(X + off[pos]), x[pos]);
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      m[j] = -INFINITY;
      arg[j] = 0;
    }
#pragma unroll
    for (int pos = 0; pos < 4; ++pos)
#pragma unroll
      for (int j = 0; j < 8; ++j)
        if (x[pos][j] > m[j]) {
          m[j] = x[pos][j];
          arg[j] = pos;
        }
    ld_f8(dY + (int64_t)q * C + cg * 8, g);
#pragma unroll
    for (int pos = 0; pos < 4; ++pos) {
      float d[8];
      ld_f8(dX + off[pos], d);
#pragma unroll
      for (int j = 0; j < 8; ++j) d[j] += arg[j] == pos ? g[j] : 0.f;
      st_f8(dX + off[pos], d);
    }
  }
}

// cat[..., 0:C1] = up2(prev) (prev at H/2 x W/2), cat[..., C1:C1+C2] = skip
// cat = [nearest-2x(prev) | skip] along channels, 8 channels (16 bytes) per
// thread; C1 and C2 are multiples of 8.  Block x is one output row (b, h),
// block y a run of that row's W * C8 16-byte groups, so a thread's indices
// take one division instead of a chain of them per group.
__global__ void k_up_concat(int H, int W, int C1, int C2, const __nv_bfloat16 *__restrict__ prev,
                            const __nv_bfloat16 *__restrict__ skip, __nv_bfloat16 *__restrict__ cat) {
  const int C8 = (C1 + C2) / 8, c18 = C1 / 8, c28 = C2 / 8;
  const int x = blockIdx.y * blockDim.x + threadIdx.x;
  if (x >= W * C8) return;
  const int r = (int)blockIdx.x, bi = r / H, h = r - bi * H;
  const int64_t row = r, b = bi;
  const int w = x / C8, c8 = x - w * C8;
  uint4 v;
  if (c8 < c18)
    v = reinterpret_cast<const uint4 *>(prev)[((b * (H / 2) + h / 2) * (W / 2) + w / 2) * c18 + c8];
  else
    v = reinterpret_cast<const uint4 *>(skip)[(row * W + w) * c28 + (c8 - c18)];
  reinterpret_cast<uint4 *>(cat)[row * W * C8 + x] = v;
}

// Backward of [nearest-2x(prev) | skip]: dskip += its channels of dcat,
// dprev += the sum of the four children; 4 channels (16 bytes) per thread.
__global__ void k_up_concat_back(int B, int H, int W, int C1, int C2, const float *__restrict__ dcat,
                                 float *__restrict__ dprev, float *__restrict__ dskip) {
  const int C = C1 + C2, C24 = C2 / 4, C14 = C1 / 4;
  AIRT_FOR32(t, B * H * W * C24) {
    const int c4 = t % C24, p = t / C24;
    const float4 g = *reinterpret_cast<const float4 *>(dcat + (int64_t)p * C + C1 + 4 * c4);
    float4 &d = reinterpret_cast<float4 *>(dskip)[t];
    float4 v = d;
    v.x += g.x, v.y += g.y, v.z += g.z, v.w += g.w;
    d = v;
  }
  const int Hh = H / 2, Wh = W / 2;
  AIRT_FOR32(t, B * Hh * Wh * C14) {
    const int c4 = t % C14, q = t / C14;
    const int w = q % Wh, h = (q / Wh) % Hh, b = q / (Wh * Hh);
    float4 a = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const float4 g = *reinterpret_cast<const float4 *>(
            dcat + (((int64_t)b * H + 2 * h + i) * W + 2 * w + j) * C + 4 * c4);
        a.x += g.x, a.y += g.y, a.z += g.z, a.w += g.w;
      }
    float4 &d = reinterpret_cast<float4 *>(dprev)[t];
    float4 v = d;
    v.x += a.x, v.y += a.y, v.z += a.z, v.w += a.w;
    d = v;
  }
}

// head: out[p] = b + sum_c w[c]*Y[p][c] (channels in order), one pixel per
// thread, 8 channels per 16-byte load.  With the channel count a template
// constant every 16-byte load of a pixel is issued before the first FMA and
// the weights sit in registers.
__global__ void k_head(int64_t P, int C, const __nv_bfloat16 *__restrict__ Y, const float *__restrict__ w,
                       const float *__restrict__ b, float *__restrict__ out) {
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < P;
       p += (int64_t)gridDim.x * blockDim.x) {
    float a = b[0];
    for (int cg = 0; cg < C / 8; ++cg) {
      float y[8];
      bf8_to_f(*reinterpret_cast<const uint4 *>(Y + p * C + cg * 8), y);
#pragma unroll
      for (int j = 0; j < 8; ++j) a += w[cg * 8 + j] * y[j];
    }
    out[p] = a;
  }
}

template <int C>
__global__ void __launch_bounds__(256) k_head_c(int64_t P, const __nv_bfloat16 *__restrict__ Y,
                                                const float *__restrict__ w, const float *__restrict__ b,
                                                float *__restrict__ out) {
  float wr[C];
#pragma unroll
  for (int c = 0; c < C; ++c) wr[c] = __ldg(w + c);
  const float b0 = __ldg(b);
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < P;
       p += (int64_t)gridDim.x * blockDim.x) {
    uint4 u[C / 8];
#pragma unroll
    for (int cg = 0; cg < C / 8; ++cg) u[cg] = __ldg(reinterpret_cast<const uint4 *>(Y + p * C) + cg);
    float a = b0;
#pragma unroll
    for (int cg = 0; cg < C / 8; ++cg) {
      float y[8];
      bf8_to_f(u[cg], y);
#pragma unroll
      for (int j = 0; j < 8; ++j) a += wr[cg * 8 + j] * y[j];
    }
    out[p] = a;
  }
}

// loss += mean((out - t)^2); dout = 2 (out - t) / P; dY = dout * w;
// gw[c] += sum_p dout[p] Y[p][c]; gb += sum_p dout[p].  Rows and channel
// groups as in k_relu_mask_colsum.
__global__ void __launch_bounds__(256) k_head_back(int64_t P, int C, int64_t rows_per_block,
                                                   const __nv_bfloat16 *__restrict__ Y,
                                                   const float *__restrict__ w, const float *__restrict__ out,
                                                   const float *__restrict__ tgt, float *__restrict__ dY,
                                                   float *__restrict__ gw, float *__restrict__ gb,
                                                   float *__restrict__ loss) {
  __shared__ float sh[8 * 256];
  const int C8 = C / 8, R = 256 / C8, t = threadIdx.x;
  const int64_t r0 = blockIdx.x * rows_per_block;
  const int64_t r1 = min(P, r0 + rows_per_block);
  float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  float lsum = 0.f, bsum = 0.f;
  if (t < R * C8) {
    const int cg = t % C8;
    float wc[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) wc[j] = w[cg * 8 + j];
    for (int64_t r = r0 + t / C8; r < r1; r += R) {
      const float d = out[r] - tgt[r];
      const float g = 2.f * d / (float)P;
      if (cg == 0) {
        lsum += d * d;
        bsum += g;
      }
      float y[8], o[8];
      bf8_to_f(*reinterpret_cast<const uint4 *>(Y + r * C + cg * 8), y);
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        o[j] = g * wc[j];
        acc[j] += g * y[j];
      }
      st_f8(dY + r * C + cg * 8, o);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
    bsum += __shfl_xor_sync(0xffffffffu, bsum, o);
  }
  if ((t & 31) == 0) {
    atomicAdd(loss, lsum / (float)P);
    atomicAdd(gb, bsum);
  }
  colsum_flush(acc, C8, sh, gw);
}

// First convolution (one input channel): y[p][co] = relu(b[co] +
// sum_tap w[co][tap] * x[p + tap]), FP32 sums of the BF16 products, 8
// output channels per thread.
__global__ void k_conv1_fwd(int64_t P, int H, int W, int Co, int Kp, const __nv_bfloat16 *__restrict__ x,
                            const __nv_bfloat16 *__restrict__ wt, const float *__restrict__ bias,
                            __nv_bfloat16 *__restrict__ y) {
  __shared__ float sw[64 * 9], sb[64];  // Co <= 64
  for (int i = threadIdx.x; i < Co * 9; i += blockDim.x)
    sw[i] = __bfloat162float(wt[(int64_t)(i / 9) * Kp + i % 9]);
  for (int i = threadIdx.x; i < Co; i += blockDim.x) sb[i] = bias[i];
  __syncthreads();
  const int C8 = Co / 8;
  AIRT_FOR32(t, (int)P * C8) {
    const int og = t % C8, p = t / C8;
    const int w = p % W, h = (p / W) % H;
    float xv[9];
#pragma unroll
    for (int tap = 0; tap < 9; ++tap) {
      const int dh = tap / 3 - 1, dw = tap % 3 - 1;
      const bool in = h + dh >= 0 && h + dh < H && w + dw >= 0 && w + dw < W;
      xv[tap] = in ? __bfloat162float(x[p + dh * W + dw]) : 0.f;
    }
    float o[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int co = og * 8 + j;
      float a = 0.f;
#pragma unroll
      for (int tap = 0; tap < 9; ++tap) a += sw[co * 9 + tap] * xv[tap];
      o[j] = fmaxf(a + sb[co], 0.f);
    }
    reinterpret_cast<uint4 *>(y)[t] = f_to_bf8(o);
  }
}

// The same convolution with CPT (a template constant, 16) output channels of
// one pixel per thread (CO / CPT threads per pixel, so that three blocks fit
// per SM): the nine neighbours are loaded once per thread, the weights are
// read from shared memory as [tap][co] float4 broadcasts, and the channels
// leave as 16-byte stores.  Per channel the sum runs over the taps in the
// same order as k_conv1_fwd.
template <int CO, int CPT>
__global__ void __launch_bounds__(256, 3) k_conv1_fwd_px(int P, int H, int W, int Kp,
                                                         const __nv_bfloat16 *__restrict__ x,
                                                         const __nv_bfloat16 *__restrict__ wt,
                                                         const float *__restrict__ bias,
                                                         __nv_bfloat16 *__restrict__ y) {
  static_assert(CO % CPT == 0 && CPT % 8 == 0, "channel split");
  constexpr int G = CO / CPT;
  __shared__ __align__(16) float sw[9 * CO];
  __shared__ __align__(16) float sb[CO];
  for (int i = threadIdx.x; i < CO * 9; i += blockDim.x) {
    const int tap = i / CO, co = i % CO;
    sw[i] = __bfloat162float(wt[(int64_t)co * Kp + tap]);
  }
  for (int i = threadIdx.x; i < CO; i += blockDim.x) sb[i] = bias[i];
  __syncthreads();
  const int HW = H * W;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < P * G; t += gridDim.x * blockDim.x) {
    const int p = t / G, c0 = (t - p * G) * CPT;
    const int q = p % HW, h = q / W, w = q - h * W;
    float xv[9];
#pragma unroll
    for (int tap = 0; tap < 9; ++tap) {
      const int dh = tap / 3 - 1, dw = tap % 3 - 1;
      const bool in = h + dh >= 0 && h + dh < H && w + dw >= 0 && w + dw < W;
      xv[tap] = in ? __bfloat162float(x[p + dh * W + dw]) : 0.f;
    }
    float a[CPT];
#pragma unroll
    for (int co = 0; co < CPT; ++co) a[co] = 0.f;
#pragma unroll
    for (int tap = 0; tap < 9; ++tap) {
      const float4 *w4 = reinterpret_cast<const float4 *>(sw + tap * CO + c0);
#pragma unroll
      for (int c4 = 0; c4 < CPT / 4; ++c4) {
        const float4 wv = w4[c4];
        a[4 * c4] += wv.x * xv[tap];
        a[4 * c4 + 1] += wv.y * xv[tap];
        a[4 * c4 + 2] += wv.z * xv[tap];
        a[4 * c4 + 3] += wv.w * xv[tap];
      }
    }
    uint4 *yo = reinterpret_cast<uint4 *>(y + (int64_t)p * CO + c0);
#pragma unroll
    for (int g8 = 0; g8 < CPT / 8; ++g8) {
      float o[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) o[j] = fmaxf(a[g8 * 8 + j] + sb[c0 + g8 * 8 + j], 0.f);
      yo[g8] = f_to_bf8(o);
    }
  }
}

// Weight gradient of the first convolution: gw[co][tap] += sum_p dYm[p][co]
// * x[p + tap].  Lane -> output channels lane and lane + 32 (Co <= 64), all
// nine taps in registers; the 8 warps of a block take every 8th pixel of the
// block's range, and the block's sums meet in shared memory before one
// atomicAdd per (co, tap).
__global__ void __launch_bounds__(256) k_conv1_wgrad(int64_t P, int H, int W, int Co, int Kp,
                                                     int64_t rows_per_block, const __nv_bfloat16 *__restrict__ x,
                                                     const __nv_bfloat16 *__restrict__ dYm,
                                                     float *__restrict__ gw) {
  __shared__ float sh[9 * 64];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int i = threadIdx.x; i < 9 * 64; i += blockDim.x) sh[i] = 0.f;
  __syncthreads();
  const int64_t r0 = blockIdx.x * rows_per_block;
  const int64_t r1 = min(P, r0 + rows_per_block);
  float a0[9], a1[9];
#pragma unroll
  for (int t = 0; t < 9; ++t) a0[t] = a1[t] = 0.f;
  int64_t p = r0 + warp;
  int w = (int)(p % W), h = (int)((p / W) % H);
  for (; p < r1; p += 8) {
    float xv[9];
#pragma unroll
    for (int tap = 0; tap < 9; ++tap) {
      const int dh = tap / 3 - 1, dw = tap % 3 - 1;
      const bool in = h + dh >= 0 && h + dh < H && w + dw >= 0 && w + dw < W;
      xv[tap] = in ? __bfloat162float(x[p + (int64_t)dh * W + dw]) : 0.f;
    }
    const float d0 = lane < Co ? __bfloat162float(dYm[p * Co + lane]) : 0.f;
    const float d1 = lane + 32 < Co ? __bfloat162float(dYm[p * Co + lane + 32]) : 0.f;
#pragma unroll
    for (int tap = 0; tap < 9; ++tap) {
      a0[tap] += d0 * xv[tap];
      a1[tap] += d1 * xv[tap];
    }
    w += 8;
    while (w >= W) {
      w -= W;
      if (++h == H) h = 0;
    }
  }
#pragma unroll
  for (int tap = 0; tap < 9; ++tap) {
    if (lane < Co) atomicAdd(&sh[tap * 64 + lane], a0[tap]);
    if (lane + 32 < Co) atomicAdd(&sh[tap * 64 + lane + 32], a1[tap]);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 9 * Co; i += blockDim.x) {
    const int tap = i / Co, co = i - tap * Co;
    atomicAdd(gw + (int64_t)co * Kp + tap, sh[tap * 64 + co]);
  }
}

__global__ void k_to_bf16(int64_t n, const float *__restrict__ a, __nv_bfloat16 *__restrict__ b) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    b[i] = __float2bfloat16(a[i]);
}

__global__ void k_adam(int64_t n, float *__restrict__ w, const float *__restrict__ g, float *__restrict__ m1,
                       float *__restrict__ m2, float lr, float b1, float b2, float eps, float c1, float c2) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float a = b1 * m1[i] + (1.f - b1) * gi;
    const float v = b2 * m2[i] + (1.f - b2) * gi * gi;
    m1[i] = a;
    m2[i] = v;
    w[i] -= lr * (a / c1) / (sqrtf(v / c2) + eps);
  }
}

inline unsigned gsz(int64_t n) { return grid_for(n, kT, 8); }

}  // namespace

struct Tensor {
  int C = 0, H = 0, W = 0;
  DevBuf<__nv_bfloat16> y;  // [B*H*W][C]
  DevBuf<float> g;          // gradient
};

struct Conv {
  int cin, cout, kp, H, W;
  Tensor *in, *out;
  DevBuf<float> w, gw, mw, vw, b, gb, mb, vb;
  DevBuf<__nv_bfloat16> w16, wt16;  // wt16: tap-flipped transpose for dX
};

struct UNet {
  int H, W, base, levels, maxB;
  cudaStream_t s = nullptr;
  std::vector<Tensor *> tensors;
  Tensor *xin;
  std::vector<Tensor *> ea, eb, pool, cat, da, db;
  std::vector<Conv> convs;  // forward order
  DevBuf<float> hw, hgw, hmw, hvw, hb, hgb, hmb, hvb;  // head (1x1, base -> 1)
  DevBuf<float> out, loss;
  DevBuf<__nv_bfloat16> col, dym;
  DevBuf<float> dcol;
  DevBuf<float> tgt;  // training target in NHWC order, maxB*H*W
  DevBuf<int> err;
  int64_t adam_t = 0;
  Tensor *T(int C, int H, int W) {
    Tensor *t = new Tensor();
    t->C = C;
    t->H = H;
    t->W = W;
    tensors.push_back(t);
    return t;
  }
  ~UNet() {
    for (Tensor *t : tensors) delete t;
  }
};

namespace {

int kp_of(int cin) { return ((9 * cin + 63) / 64) * 64; }

void conv_alloc(UNet &U, Conv &c, std::mt19937_64 &rng) {
  c.kp = kp_of(c.cin);
  const size_t nw = (size_t)c.cout * c.kp;
  std::vector<float> hw(nw, 0.f), hb(c.cout, 0.f);
  std::normal_distribution<float> nd(0.f, std::sqrt(2.f / (9.f * c.cin)));
  for (int o = 0; o < c.cout; ++o)
    for (int k = 0; k < 9 * c.cin; ++k) hw[(size_t)o * c.kp + k] = nd(rng);
  c.w.upload(hw.data(), nw, U.s);
  c.b.upload(hb.data(), c.cout, U.s);
  for (DevBuf<float> *d : {&c.gw, &c.mw, &c.vw}) {
    d->ensure(nw);
    AIRT_CHECK_CUDA(cudaMemsetAsync(d->p, 0, nw * 4, U.s));
  }
  for (DevBuf<float> *d : {&c.gb, &c.mb, &c.vb}) {
    d->ensure(c.cout);
    AIRT_CHECK_CUDA(cudaMemsetAsync(d->p, 0, c.cout * 4, U.s));
  }
  c.w16.ensure(nw);
  k_to_bf16<<<gsz(nw), kT, 0, U.s>>>(nw, c.w.p, c.w16.p);
  if (c.cin % 8 == 0 && c.cout % 8 == 0) c.wt16.ensure((size_t)c.cin * kp_of(c.cout));
}

void ensure_act(UNet &U, Tensor *t, int B) {
  const size_t n = (size_t)B * t->H * t->W * t->C;
  t->y.ensure(n);
  t->g.ensure(n);
}

int bn_for(int n) { return n >= 256 ? 256 : n >= 128 ? 128 : n >= 64 ? 64 : 32; }

// Blocks of contiguous pixel rows for the row-reduction kernels: about 8
// per SM, at least 64 rows each.
void row_blocks(int64_t P, int64_t &blocks, int64_t &rpb) {
  blocks = std::min<int64_t>(1184, std::max<int64_t>(1, P / 64));
  rpb = (P + blocks - 1) / blocks;
  blocks = (P + rpb - 1) / rpb;
}

void conv_forward(UNet &U, Conv &c, int B) {
  const int64_t P = (int64_t)B * c.H * c.W;
  if (c.cin == 1 && c.cout % 8 == 0) {  // first convolution: direct kernel
    if (c.cout == 32)
      k_conv1_fwd_px<32, 16><<<gsz(2 * P), kT, 0, U.s>>>((int)P, c.H, c.W, c.kp, c.in->y.p, c.w16.p, c.b.p,
                                                          c.out->y.p);
    else if (c.cout == 16)
      k_conv1_fwd_px<16, 16><<<gsz(P), kT, 0, U.s>>>((int)P, c.H, c.W, c.kp, c.in->y.p, c.w16.p, c.b.p,
                                                      c.out->y.p);
    else
      k_conv1_fwd<<<gsz(P * c.cout / 8), kT, 0, U.s>>>(P, c.H, c.W, c.cout, c.kp, c.in->y.p, c.w16.p, c.b.p,
                                                       c.out->y.p);
    AIRT_LAUNCH_CHECK();
    return;
  }
  if (c.cin % 8 == 0 && c.cout % 8 == 0) {  // implicit GEMM: taps gathered from the NHWC input
    GemmArgs g{};
    g.M = (int)P;
    g.N = c.cout;
    g.K = c.kp;
    g.B = c.w16.p;
    g.ldb = c.kp;
    g.D = c.out->y.p;
    g.ldd = c.cout;
    g.bias = c.b.p;
    g.err = U.err.p;
    g.convX = c.in->y.p;
    g.conv_H = c.H;
    g.conv_W = c.W;
    g.conv_C = c.cin;
    conv3x3_bf16(g, bn_for(c.cout), EPI_BIAS_RELU_BF16, U.s);
    return;
  }
  AIRT_REQUIRE(U.col.n >= (size_t)(P * c.kp), "im2col buffer too small");
  k_im2col<<<gsz(P * c.kp), kT, 0, U.s>>>(B, c.H, c.W, c.cin, c.kp, c.in->y.p, U.col.p);
  AIRT_LAUNCH_CHECK();
  GemmArgs g{};
  g.M = (int)P;
  g.N = c.cout;
  g.K = c.kp;
  g.A = U.col.p;
  g.lda = c.kp;
  g.B = c.w16.p;
  g.ldb = c.kp;
  g.D = c.out->y.p;
  g.ldd = c.cout;
  g.bias = c.b.p;
  g.ksplit = 0;
  g.err = U.err.p;
  gemm_bf16(g, bn_for(c.cout), false, false, EPI_BIAS_RELU_BF16, U.s);
}

void conv_backward(UNet &U, Conv &c, int B, bool need_dx) {
  const int64_t P = (int64_t)B * c.H * c.W;
  const int64_t ksplit = std::max<int64_t>(64, ((P / 64 + 63) / 64) * 64);  // ~64 K-splits
  {
    int64_t blocks, rpb;
    row_blocks(P, blocks, rpb);
    k_relu_mask_colsum<<<(unsigned)blocks, 256, 0, U.s>>>(P, c.cout, rpb, c.out->g.p, c.out->y.p, U.dym.p,
                                                         c.gb.p);
    AIRT_LAUNCH_CHECK();
  }
  if (c.cin == 1) {  // first convolution: direct weight gradient, no dX
    AIRT_REQUIRE(!need_dx && c.cout <= 64, "first convolution: unsupported configuration");
    int64_t blocks, rpb;
    row_blocks(P, blocks, rpb);
    k_conv1_wgrad<<<(unsigned)blocks, 256, 0, U.s>>>(P, c.H, c.W, c.cout, c.kp, rpb, c.in->y.p, U.dym.p,
                                                     c.gw.p);
    AIRT_LAUNCH_CHECK();
    return;
  }
  if (c.cin % 8 == 0 && c.cout % 8 == 0) {
    GemmArgs gw{};
    gw.M = c.kp;
    gw.N = c.cout;
    gw.K = (int)P;
    gw.B = U.dym.p;
    gw.ldb = c.cout;
    gw.D = c.gw.p;
    gw.ldd = c.kp;
    gw.ksplit = (int)ksplit;
    gw.err = U.err.p;
    gw.convX = c.in->y.p;
    gw.conv_H = c.H;
    gw.conv_W = c.W;
    gw.conv_C = c.cin;
    conv3x3_wgrad_bf16(gw, bn_for(c.cout), U.s);
    if (!need_dx) return;
    const int kq = kp_of(c.cout);
    k_flip_w<<<gsz((int64_t)c.cin * kq), kT, 0, U.s>>>(c.cout, c.cin, c.kp, kq, c.w16.p, c.wt16.p);
    AIRT_LAUNCH_CHECK();
    GemmArgs gd{};
    gd.M = (int)P;
    gd.N = c.cin;
    gd.K = kq;
    gd.B = c.wt16.p;
    gd.ldb = kq;
    gd.D = c.in->g.p;
    gd.ldd = c.cin;
    gd.err = U.err.p;
    gd.convX = U.dym.p;
    gd.conv_H = c.H;
    gd.conv_W = c.W;
    gd.conv_C = c.cout;
    conv3x3_bf16(gd, bn_for(c.cin), EPI_ADD_F32, U.s);
    return;
  }
  AIRT_REQUIRE(U.col.n >= (size_t)(P * c.kp) && (!need_dx || U.dcol.n >= (size_t)(P * c.kp)),
               "im2col buffer too small");
  k_im2col<<<gsz(P * c.kp), kT, 0, U.s>>>(B, c.H, c.W, c.cin, c.kp, c.in->y.p, U.col.p);
  AIRT_LAUNCH_CHECK();
  // dW^T[Kp][Co] += col^T * dYm, stored transposed into gw[Co][Kp]
  GemmArgs gw{};
  gw.M = c.kp;
  gw.N = c.cout;
  gw.K = (int)P;
  gw.A = U.col.p;
  gw.lda = c.kp;
  gw.B = U.dym.p;
  gw.ldb = c.cout;
  gw.D = c.gw.p;
  gw.ldd = c.kp;
  gw.ksplit = (int)ksplit;
  gw.err = U.err.p;
  gemm_bf16(gw, bn_for(c.cout), true, true, EPI_ATOMIC_F32_T, U.s);
  if (!need_dx) return;
  // dcol[P][Kp] = dYm[P][Co] * W[Co][Kp]
  GemmArgs gd{};
  gd.M = (int)P;
  gd.N = c.kp;
  gd.K = c.cout;
  gd.A = U.dym.p;
  gd.lda = c.cout;
  gd.B = c.w16.p;
  gd.ldb = c.kp;
  gd.D = U.dcol.p;
  gd.ldd = c.kp;
  gd.ksplit = 0;
  gd.err = U.err.p;
  gemm_bf16(gd, bn_for(c.kp), false, true, EPI_STORE_F32, U.s);
  k_col2im<<<gsz(P * c.cin), kT, 0, U.s>>>(B, c.H, c.W, c.cin, c.kp, U.dcol.p, c.in->g.p);
  AIRT_LAUNCH_CHECK();
}

}  // namespace

UNet *unet_create(int H, int W, int base, int levels, int maxB, uint64_t seed) {
  AIRT_REQUIRE(levels >= 2 && levels <= 6, "levels must be 2..6");
  AIRT_REQUIRE(base % 8 == 0 && base >= 8, "base width must be a multiple of 8");
  AIRT_REQUIRE(H % (1 << (levels - 1)) == 0 && W % (1 << (levels - 1)) == 0,
               "image size must be divisible by 2^(levels-1)");
  AIRT_REQUIRE(maxB >= 1, "batch must be positive");
  AIRT_REQUIRE(base <= 64, "head supports at most 64 channels");
  UNet *U = new UNet();
  try {
    U->H = H;
    U->W = W;
    U->base = base;
    U->levels = levels;
    U->maxB = maxB;
    AIRT_CHECK_CUDA(cudaStreamCreateWithFlags(&U->s, cudaStreamNonBlocking));
    std::mt19937_64 rng(seed);
    U->xin = U->T(1, H, W);
    U->ea.resize(levels);
    U->eb.resize(levels);
    U->pool.assign(levels, nullptr);
    U->cat.resize(levels - 1);
    U->da.resize(levels - 1);
    U->db.resize(levels - 1);
    for (int l = 0; l < levels; ++l) {
      const int h = H >> l, w = W >> l, c = base << l;
      if (l > 0) U->pool[l] = U->T(base << (l - 1), h, w);
      U->ea[l] = U->T(c, h, w);
      U->eb[l] = U->T(c, h, w);
    }
    for (int l = levels - 2; l >= 0; --l) {
      const int h = H >> l, w = W >> l, c = base << l;
      U->cat[l] = U->T((base << (l + 1)) + c, h, w);
      U->da[l] = U->T(c, h, w);
      U->db[l] = U->T(c, h, w);
    }
    auto add = [&](Tensor *in, Tensor *out) {
      Conv c;
      c.cin = in->C;
      c.cout = out->C;
      c.H = out->H;
      c.W = out->W;
      c.in = in;
      c.out = out;
      U->convs.push_back(std::move(c));
    };
    U->convs.reserve(4 * levels);
    for (int l = 0; l < levels; ++l) {
      add(l == 0 ? U->xin : U->pool[l], U->ea[l]);
      add(U->ea[l], U->eb[l]);
    }
    for (int l = levels - 2; l >= 0; --l) {
      add(U->cat[l], U->da[l]);
      add(U->da[l], U->db[l]);
    }
    for (Conv &c : U->convs) conv_alloc(*U, c, rng);
    std::normal_distribution<float> nd(0.f, std::sqrt(1.f / base));
    std::vector<float> hw(base);
    for (float &v : hw) v = nd(rng);
    float zero = 0.f;
    U->hw.upload(hw.data(), base, U->s);
    U->hb.upload(&zero, 1, U->s);
    for (DevBuf<float> *d : {&U->hgw, &U->hmw, &U->hvw}) {
      d->ensure(base);
      AIRT_CHECK_CUDA(cudaMemsetAsync(d->p, 0, base * 4, U->s));
    }
    for (DevBuf<float> *d : {&U->hgb, &U->hmb, &U->hvb}) {
      d->ensure(1);
      AIRT_CHECK_CUDA(cudaMemsetAsync(d->p, 0, 4, U->s));
    }
    for (Tensor *t : U->tensors) {
      AIRT_REQUIRE((int64_t)maxB * t->H * t->W * t->C < ((int64_t)1 << 30),
                   "max_batch too large: every activation tensor must hold fewer than 2^30 values");
      ensure_act(*U, t, maxB);
    }
    // col / dcol only for convolutions without the implicit path (Cin = 1);
    // the first convolution never needs dX.
    size_t colmax = 1, dcolmax = 1;
    int64_t dymax = 0;
    for (size_t i = 0; i < U->convs.size(); ++i) {
      const Conv &c = U->convs[i];
      const size_t ncol = (size_t)maxB * c.H * c.W * c.kp;
      if (c.cin != 1 && (c.cin % 8 != 0 || c.cout % 8 != 0)) {
        colmax = std::max(colmax, ncol);
        if (i > 0) dcolmax = std::max(dcolmax, ncol);
      }
      dymax = std::max<int64_t>(dymax, (int64_t)maxB * c.H * c.W * c.cout);
    }
    U->col.ensure(colmax);
    U->dcol.ensure(dcolmax);
    U->tgt.ensure((size_t)maxB * H * W);
    U->dym.ensure(dymax);
    U->out.ensure((size_t)maxB * H * W);
    U->loss.ensure(1);
    U->err.ensure(1);
    AIRT_CHECK_CUDA(cudaMemsetAsync(U->err.p, 0, sizeof(int), U->s));
    AIRT_CHECK_CUDA(cudaStreamSynchronize(U->s));
  } catch (...) {
    if (U->s) cudaStreamSynchronize(U->s);
    cudaStream_t s = U->s;
    delete U;
    if (s) cudaStreamDestroy(s);
    throw;
  }
  return U;
}

void unet_destroy(UNet *U) {
  if (!U) return;
  cudaStream_t s = U->s;
  if (s) cudaStreamSynchronize(s);
  delete U;
  if (s) cudaStreamDestroy(s);
}

cudaStream_t unet_stream(UNet &U) { return U.s; }

// in: [B][H*W] FP32 images in the x(:) (column-major) order of the solvers;
// with NHWC pixel (b, h, w) = in[b][w*H + h] ... the map is a transpose, so
// images are copied with h = row index of the column-major image.
namespace {
template <typename TI>
__global__ void k_img_in(int B, int H, int W, const TI *__restrict__ in, __nv_bfloat16 *__restrict__ x) {
  AIRT_FOR32(t, B * H * W) {
    const int w = t % W, h = (t / W) % H, b = t / (W * H);
    x[t] = __float2bfloat16((float)in[(int64_t)b * H * W + (int64_t)w * H + h]);
  }
}
template <typename TO>
__global__ void k_img_out(int B, int H, int W, const float *__restrict__ o, TO *__restrict__ out) {
  AIRT_FOR32(t, B * H * W) {
    const int w = t % W, h = (t / W) % H, b = t / (W * H);
    out[(int64_t)b * H * W + (int64_t)w * H + h] = (TO)o[t];
  }
}
__global__ void k_img_tgt(int B, int H, int W, const float *__restrict__ in, float *__restrict__ o) {
  AIRT_FOR32(t, B * H * W) {
    const int w = t % W, h = (t / W) % H, b = t / (W * H);
    o[t] = in[(int64_t)b * H * W + (int64_t)w * H + h];
  }
}
}  // namespace

void unet_forward_body(UNet &U, int B);

template <typename TI>
void unet_forward_t(UNet &U, const TI *d_in, int B) {
  AIRT_REQUIRE(B >= 1 && B <= U.maxB, "batch larger than the network was created for");
  const int64_t P0 = (int64_t)B * U.H * U.W;
  k_img_in<TI><<<gsz(P0), kT, 0, U.s>>>(B, U.H, U.W, d_in, U.xin->y.p);
  unet_forward_body(U, B);
}

void unet_forward(UNet &U, const float *d_in, int B) { unet_forward_t<float>(U, d_in, B); }

void unet_forward_body(UNet &U, int B) {
  const int64_t P0 = (int64_t)B * U.H * U.W;
  int ci = 0;
  for (int l = 0; l < U.levels; ++l) {
    if (l > 0) {
      Tensor *src = U.eb[l - 1];
      k_pool<<<gsz((int64_t)B * U.pool[l]->H * U.pool[l]->W * src->C / 8), kT, 0, U.s>>>(
          B, src->H, src->W, src->C, src->y.p, U.pool[l]->y.p);
    }
    conv_forward(U, U.convs[ci++], B);
    conv_forward(U, U.convs[ci++], B);
  }
  for (int l = U.levels - 2; l >= 0; --l) {
    Tensor *prev = (l == U.levels - 2) ? U.eb[U.levels - 1] : U.db[l + 1];
    Tensor *cat = U.cat[l];
    const dim3 ug((unsigned)((int64_t)B * cat->H), (unsigned)((cat->W * (cat->C / 8) + kT - 1) / kT));
    k_up_concat<<<ug, kT, 0, U.s>>>(cat->H, cat->W, prev->C, U.eb[l]->C, prev->y.p, U.eb[l]->y.p,
                                    cat->y.p);
    conv_forward(U, U.convs[ci++], B);
    conv_forward(U, U.convs[ci++], B);
  }
  if (U.base == 32) k_head_c<32><<<gsz(P0), kT, 0, U.s>>>(P0, U.db[0]->y.p, U.hw.p, U.hb.p, U.out.p);
  else if (U.base == 16) k_head_c<16><<<gsz(P0), kT, 0, U.s>>>(P0, U.db[0]->y.p, U.hw.p, U.hb.p, U.out.p);
  else k_head<<<gsz(P0), kT, 0, U.s>>>(P0, U.base, U.db[0]->y.p, U.hw.p, U.hb.p, U.out.p);
  AIRT_LAUNCH_CHECK();
}

template <typename TO>
void unet_output(UNet &U, TO *d_out, int B) {
  k_img_out<TO><<<gsz((int64_t)B * U.H * U.W), kT, 0, U.s>>>(B, U.H, U.W, U.out.p, d_out);
  AIRT_LAUNCH_CHECK();
}

// Forward + backward; gradients land in the g* buffers (zeroed here).
// Returns the MSE loss of the batch.
float unet_gradients(UNet &U, const float *d_in, const float *d_tgt, int B) {
  unet_forward(U, d_in, B);
  const int64_t P0 = (int64_t)B * U.H * U.W;
  for (Conv &c : U.convs) {
    AIRT_CHECK_CUDA(cudaMemsetAsync(c.gw.p, 0, (size_t)c.cout * c.kp * 4, U.s));
    AIRT_CHECK_CUDA(cudaMemsetAsync(c.gb.p, 0, (size_t)c.cout * 4, U.s));
  }
  AIRT_CHECK_CUDA(cudaMemsetAsync(U.hgw.p, 0, U.base * 4, U.s));
  AIRT_CHECK_CUDA(cudaMemsetAsync(U.hgb.p, 0, 4, U.s));
  AIRT_CHECK_CUDA(cudaMemsetAsync(U.loss.p, 0, 4, U.s));
  for (Tensor *t : U.tensors)
    AIRT_CHECK_CUDA(cudaMemsetAsync(t->g.p, 0, (size_t)B * t->H * t->W * t->C * 4, U.s));
  float *tgt = U.tgt.p;
  k_img_tgt<<<gsz(P0), kT, 0, U.s>>>(B, U.H, U.W, d_tgt, tgt);
  {
    int64_t blocks, rpb;
    row_blocks(P0, blocks, rpb);
    k_head_back<<<(unsigned)blocks, 256, 0, U.s>>>(P0, U.base, rpb, U.db[0]->y.p, U.hw.p, U.out.p, tgt,
                                                   U.db[0]->g.p, U.hgw.p, U.hgb.p, U.loss.p);
  }
  AIRT_LAUNCH_CHECK();
  int ci = (int)U.convs.size() - 1;
  // decoder, in reverse of the forward order (levels 0 .. L-2)
  for (int l = 0; l <= U.levels - 2; ++l) {
    conv_backward(U, U.convs[ci--], B, true);  // da[l] -> db[l]
    conv_backward(U, U.convs[ci--], B, true);  // cat[l] -> da[l]
    Tensor *prev = (l == U.levels - 2) ? U.eb[U.levels - 1] : U.db[l + 1];
    Tensor *cat = U.cat[l];
    k_up_concat_back<<<gsz((int64_t)B * cat->H * cat->W * cat->C / 4), kT, 0, U.s>>>(
        B, cat->H, cat->W, prev->C, U.eb[l]->C, cat->g.p, prev->g.p, U.eb[l]->g.p);
    AIRT_LAUNCH_CHECK();
  }
  // encoder, levels L-1 .. 0; eb[l] has its skip and pool gradients by now
  for (int l = U.levels - 1; l >= 0; --l) {
    conv_backward(U, U.convs[ci--], B, true);    // ea[l] -> eb[l]
    conv_backward(U, U.convs[ci--], B, l > 0);   // in -> ea[l]
    if (l > 0) {
      Tensor *src = U.eb[l - 1];
      k_pool_back<<<gsz((int64_t)B * U.pool[l]->H * U.pool[l]->W * src->C / 8), kT, 0, U.s>>>(
          B, src->H, src->W, src->C, src->y.p, U.pool[l]->g.p, src->g.p);
      AIRT_LAUNCH_CHECK();
    }
  }
  float h = 0.f;
  AIRT_CHECK_CUDA(cudaMemcpyAsync(&h, U.loss.p, 4, cudaMemcpyDeviceToHost, U.s));
  AIRT_CHECK_CUDA(cudaStreamSynchronize(U.s));
  int herr = 0;
  AIRT_CHECK_CUDA(cudaMemcpy(&herr, U.err.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (herr) {
    set_error("a bounded tensor-core wait gave up");
    throw Status{AIRT_ERR_TIMEOUT};
  }
  return h;
}

void unet_adam(UNet &U, float lr) {
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  ++U.adam_t;
  const float c1 = 1.f - std::pow(b1, (float)U.adam_t), c2 = 1.f - std::pow(b2, (float)U.adam_t);
  for (Conv &c : U.convs) {
    const int64_t nw = (int64_t)c.cout * c.kp;
    k_adam<<<gsz(nw), kT, 0, U.s>>>(nw, c.w.p, c.gw.p, c.mw.p, c.vw.p, lr, b1, b2, eps, c1, c2);
    k_adam<<<gsz(c.cout), kT, 0, U.s>>>(c.cout, c.b.p, c.gb.p, c.mb.p, c.vb.p, lr, b1, b2, eps, c1, c2);
    k_to_bf16<<<gsz(nw), kT, 0, U.s>>>(nw, c.w.p, c.w16.p);
  }
  k_adam<<<1, kT, 0, U.s>>>(U.base, U.hw.p, U.hgw.p, U.hmw.p, U.hvw.p, lr, b1, b2, eps, c1, c2);
  k_adam<<<1, kT, 0, U.s>>>(1, U.hb.p, U.hgb.p, U.hmb.p, U.hvb.p, lr, b1, b2, eps, c1, c2);
  AIRT_LAUNCH_CHECK();
}

// Flattened parameters: per convolution (forward order) W[cout][9*cin]
// (K index (kh*3+kw)*cin + ci) then b[cout]; then the head w[base], b.
int64_t unet_num_params(const UNet &U) {
  int64_t n = 0;
  for (const Conv &c : U.convs) n += (int64_t)c.cout * 9 * c.cin + c.cout;
  return n + U.base + 1;
}

void unet_params(UNet &U, float *host, bool grads, bool set) {
  int64_t off = 0;
  auto xfer = [&](DevBuf<float> &d, size_t n, size_t dst_stride, size_t src_stride, size_t rows) {
    // rows x n block between host (packed, stride n) and device (stride src_stride)
    std::vector<float> tmp(rows * src_stride);
    if (!set) {
      AIRT_CHECK_CUDA(cudaMemcpyAsync(tmp.data(), d.p, tmp.size() * 4, cudaMemcpyDeviceToHost, U.s));
      AIRT_CHECK_CUDA(cudaStreamSynchronize(U.s));
      for (size_t r = 0; r < rows; ++r)
        for (size_t k = 0; k < n; ++k) host[off + r * dst_stride + k] = tmp[r * src_stride + k];
    } else {
      std::fill(tmp.begin(), tmp.end(), 0.f);
      for (size_t r = 0; r < rows; ++r)
        for (size_t k = 0; k < n; ++k) tmp[r * src_stride + k] = host[off + r * dst_stride + k];
      AIRT_CHECK_CUDA(cudaMemcpyAsync(d.p, tmp.data(), tmp.size() * 4, cudaMemcpyHostToDevice, U.s));
      AIRT_CHECK_CUDA(cudaStreamSynchronize(U.s));
    }
    off += rows * n;
  };
  for (Conv &c : U.convs) {
    xfer(grads ? c.gw : c.w, 9 * c.cin, 9 * c.cin, c.kp, c.cout);
    xfer(grads ? c.gb : c.b, c.cout, c.cout, c.cout, 1);
    if (set && !grads) {
      const int64_t nw = (int64_t)c.cout * c.kp;
      k_to_bf16<<<gsz(nw), kT, 0, U.s>>>(nw, c.w.p, c.w16.p);
    }
  }
  xfer(grads ? U.hgw : U.hw, U.base, U.base, U.base, 1);
  xfer(grads ? U.hgb : U.hb, 1, 1, 1, 1);
  AIRT_CHECK_CUDA(cudaStreamSynchronize(U.s));
}

}  // namespace airt

using namespace airt;

#define UNET_API_BEGIN try {
#define UNET_API_END                 \
  }                                  \
  catch (const airt::Status &st) {   \
    return st.code;                  \
  }                                  \
  catch (...) {                      \
    set_error("unexpected internal error"); \
    return AIRT_ERR_CUDA;            \
  }                                  \
  return AIRT_OK;

extern "C" {

int airt_unet_create(int H, int W, int base, int levels, int max_batch, uint64_t seed, airt_unet **out) {
  UNET_API_BEGIN
  AIRT_REQUIRE(out, "null pointer argument");
  *out = reinterpret_cast<airt_unet *>(unet_create(H, W, base, levels, max_batch, seed));
  UNET_API_END
}

int airt_unet_destroy(airt_unet *h) {
  UNET_API_BEGIN
  unet_destroy(reinterpret_cast<UNet *>(h));
  UNET_API_END
}

int airt_unet_stream(const airt_unet *h, void **cuda_stream) {
  UNET_API_BEGIN
  AIRT_REQUIRE(h && cuda_stream, "null pointer argument");
  *cuda_stream = (void *)reinterpret_cast<const UNet *>(h)->s;
  UNET_API_END
}

int airt_unet_num_params(const airt_unet *h, int64_t *n) {
  UNET_API_BEGIN
  AIRT_REQUIRE(h && n, "null pointer argument");
  *n = unet_num_params(*reinterpret_cast<const UNet *>(h));
  UNET_API_END
}

int airt_unet_get_params(airt_unet *h, float *host) {
  UNET_API_BEGIN
  AIRT_REQUIRE(h && host, "null pointer argument");
  unet_params(*reinterpret_cast<UNet *>(h), host, false, false);
  UNET_API_END
}

int airt_unet_set_params(airt_unet *h, const float *host) {
  UNET_API_BEGIN
  AIRT_REQUIRE(h && host, "null pointer argument");
  unet_params(*reinterpret_cast<UNet *>(h), const_cast<float *>(host), false, true);
  UNET_API_END
}

int airt_unet_get_grads(airt_unet *h, float *host) {
  UNET_API_BEGIN
  AIRT_REQUIRE(h && host, "null pointer argument");
  unet_params(*reinterpret_cast<UNet *>(h), host, true, false);
  UNET_API_END
}

int airt_unet_forward(airt_unet *h, const float *d_in, float *d_out, int B) {
  UNET_API_BEGIN
  AIRT_REQUIRE(h && d_in && d_out, "null pointer argument");
  UNet &U = *reinterpret_cast<UNet *>(h);
  unet_forward(U, d_in, B);
  unet_output(U, d_out, B);
  UNET_API_END
}

int airt_unet_forward_f64(airt_unet *h, const double *d_in, double *d_out, int B, void *cuda_stream) {
  UNET_API_BEGIN
  AIRT_REQUIRE(h && d_in && d_out, "null pointer argument");
  UNet &U = *reinterpret_cast<UNet *>(h);
  // order the network after work already queued on the caller's stream
  cudaEvent_t ev = nullptr;
  if (cuda_stream) {
    AIRT_CHECK_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    AIRT_CHECK_CUDA(cudaEventRecord(ev, static_cast<cudaStream_t>(cuda_stream)));
    AIRT_CHECK_CUDA(cudaStreamWaitEvent(U.s, ev, 0));
  }
  for (int b0 = 0; b0 < B; b0 += U.maxB) {
    const int nb = std::min(U.maxB, B - b0);
    const int64_t off = (int64_t)b0 * U.H * U.W;
    unet_forward_t<double>(U, d_in + off, nb);
    unet_output<double>(U, d_out + off, nb);
  }
  if (cuda_stream) {
    AIRT_CHECK_CUDA(cudaEventRecord(ev, U.s));
    AIRT_CHECK_CUDA(cudaStreamWaitEvent(static_cast<cudaStream_t>(cuda_stream), ev, 0));
    cudaEventDestroy(ev);
  }
  UNET_API_END
}

int airt_unet_gradients(airt_unet *h, const float *d_in, const float *d_tgt, int B, float *loss) {
  UNET_API_BEGIN
  AIRT_REQUIRE(h && d_in && d_tgt, "null pointer argument");
  const float l = unet_gradients(*reinterpret_cast<UNet *>(h), d_in, d_tgt, B);
  if (loss) *loss = l;
  UNET_API_END
}

int airt_unet_train_step(airt_unet *h, const float *d_in, const float *d_tgt, int B, float lr,
                         float *loss) {
  UNET_API_BEGIN
  AIRT_REQUIRE(h && d_in && d_tgt && lr > 0, "invalid argument");
  UNet &U = *reinterpret_cast<UNet *>(h);
  const float l = unet_gradients(U, d_in, d_tgt, B);
  unet_adam(U, lr);
  if (loss) *loss = l;
  UNET_API_END
}

}  // extern "C"
