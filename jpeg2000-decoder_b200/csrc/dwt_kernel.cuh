/*
 * dwt_kernel.cuh — inverse 5/3 and 9/7 DWT levels and the inverse MCT / DC-shift / pack
 * stage for sm_100a.
 *
 * One CTA reconstructs a 64x64 output tile of one resolution level of one
 * tile-component: it stages the 72x72 interleaved input window (the four quadrants of the
 * Mallat layout plus a 4-sample whole-sample-symmetric halo) in shared memory with
 * coalesced asynchronous copies, lifts each window row and then each output column in
 * registers (one thread streams one line), and writes
 * the 64x64 result with coalesced stores.  Every level is one read and one write of the
 * level's samples; all tile-components of a batch at a given level share one launch.
 *
 * Arithmetic follows the reference exactly so that results are bit-identical:
 *   9/7: each lifting update is D = S - c * (L + R) with three separately rounded float
 *        operations (bmi_cpu_dwt_decoder.cpp:2374-2385, vdwt_analyst_line :4975-4993),
 *        constants of bmi_cpu_dwt.h:31-41; the reconstructed LL entering a finer level is
 *        multiplied by K_lo*K_lo (:1599, :1626); band gains are folded in by Tier-1.
 *   5/3: x[2n] -= (x[2n-1] + x[2n+1] + 2) >> 2, x[2n+1] += (x[2n] + x[2n+2]) >> 1 with
 *        symmetric ends (:2609-2659, :3311-3534); with J2K_FLAG_REF_COMPAT the last
 *        column rows are rebuilt the way VDWT_R53_LINES does (:3364-3398).
 * A whole-sample symmetric input extension is preserved by every lifting step, so
 * mirroring the input once and lifting across the halo gives the same values as the
 * reference's per-step mirroring at the region edges.
 */
#pragma once
#include <cstdint>
#include <type_traits>

namespace j2k_dev {

constexpr int DWT_T = 64;          // output tile edge
constexpr int DWT_H = 4;           // halo
constexpr int DWT_N = DWT_T + 2 * DWT_H;  // 72
constexpr int DWT_PITCH = DWT_N + 1;      // odd pitch: conflict-free column access

struct DwtLevel {
  uint64_t base;     // element offset of the tile-component region (same in every buffer)
  int32_t stride;    // tile-component width
  int32_t rw, rh;    // size of the resolution being rebuilt
  int32_t lw, lh;    // size of its low-pass part (resolution r-1)
  int8_t ll_src;     // buffer holding the LL quadrant: 0 coefficients, 1 B, 2 C
  int8_t out_dst;    // buffer receiving the level: 1 B, 2 C
  int8_t ll_gain;    // 9/7: scale the LL quadrant by K_lo^2 (reconstructed LL)
  int8_t refcompat;  // 5/3: reference column-end arithmetic
  int32_t tiles_x;
};

struct DwtTask {
  uint32_t level;  // index into the DwtLevel array
  uint16_t tx, ty;
};

// Output stage: one tile of one image, up to four components.
struct OutGroup {
  uint64_t comp_off[4];  // element offsets of the final component regions
  int8_t comp_buf[4];    // buffer ids (0 coefficients, 1 B, 2 C), -1 = absent
  int32_t stride[4];
  int32_t x0, y0, w, h;  // tile rectangle in the output image
  uint64_t out_off;      // byte offset of the image in the output buffer
  int32_t pitch_px;      // output width in pixels
  int16_t fmt, bitdepth;
  int8_t rev, mct, ncomp, checkout;  // checkout: reference mCheckOutComponent, -1 = all
  int32_t tiles_x;
  // sub-sampled components (SIZ XRsiz / YRsiz > 1): pixel (x0 + xx, y0 + yy) shows sample
  // (floor((ax + xx) / sx[c]) - cx[c], floor((ay + yy) / sy[c]) - cy[c]) of component c's
  // tile-component (clamped to its cw x ch samples), ax / ay being the tile's absolute
  // pixel origin and cx / cy the tile-component's absolute origin on the component's grid
  int32_t ax, ay;
  int32_t cx[4], cy[4], cw[4], ch[4];
  uint8_t sx[4], sy[4];
  int8_t sampled;
};
struct OutTask {
  uint32_t group;
  uint16_t tx, ty;
};

__device__ __forceinline__ int mirror(int p, int n) {
  if (n == 1) return 0;
  const int period = 2 * (n - 1);
  p %= period;
  if (p < 0) p += period;
  return p >= n ? period - p : p;
}

__device__ __forceinline__ float lift97(float s, float c, float l, float r) {
  return __fsub_rn(s, __fmul_rn(c, __fadd_rn(l, r)));
}

template <bool REV>
struct DwtTypes;
template <>
struct DwtTypes<true> {
  typedef int32_t T;
};
template <>
struct DwtTypes<false> {
  typedef float T;
};

constexpr int DWT_THREADS = 128;    // threads per CTA of the level kernels
constexpr int FUSED_THREADS = 256;  // threads per CTA of the fused last-level + output kernel

// Lifting of one window line (72 samples, element stride `st`), streamed by one thread
// through registers: iteration m reads the pair (x[2m], x[2m+1]) and retires the samples
// whose every lifting step is complete, in place behind the read position.  The values are
// those of the step-by-step scheme that updates evens 2..70 and odds 1..69 in each step
// (x[0] and x[71] keep their input values), which the 4-sample halo makes exact for the 64
// centre positions; positions above 67 are not all written.
template <bool REV>
__device__ __forceinline__ void lift_line(typename DwtTypes<REV>::T *p, int st) {
  constexpr int NP = DWT_N / 2;  // 36 pairs
  if constexpr (REV) {
    // x[2n] -= (x[2n-1] + x[2n+1] + 2) >> 2; x[2n+1] += (x[2n] + x[2n+2]) >> 1
    int xo_prev = p[st], e_prev = p[0];  // pair 0: x[0] is not updated
#pragma unroll 5
    for (int m = 1; m < NP; ++m) {
      const int xe = p[2 * m * st], xo = p[(2 * m + 1) * st];
      const int e = xe - ((xo_prev + xo + 2) >> 2);
      const int o = xo_prev + ((e_prev + e) >> 1);  // position 2m-1
      p[2 * m * st] = e;
      p[(2 * m - 1) * st] = o;
      xo_prev = xo;
      e_prev = e;
    }
  } else {
    // steps c0 (evens), c1 (odds), c2 (evens), c3 (odds): x -= c * (left + right), each
    // operation rounded separately
    const float c0 = 0.44350685204397f, c1 = 0.88291107553093f, c2 = -0.05298011857296f, c3 = -1.58613434205992f;
    const float x0 = p[0], x1 = p[st];
    const float x2 = p[2 * st], x3 = p[3 * st];
    // m = 1
    float e0_prev = lift97(x2, c0, x1, x3);     // e0 at 2
    float o1_prev = lift97(x1, c1, x0, e0_prev);  // o1 at 1 (e0 at 0 = x0)
    float e2_prev = x0;                            // e2 at 0 = x0
    float xo_prev = x3;
    p[0] = x0;
#pragma unroll 5
    for (int m = 2; m < NP; ++m) {
      const float xe = p[2 * m * st], xo = p[(2 * m + 1) * st];
      const float e0 = lift97(xe, c0, xo_prev, xo);           // position 2m
      const float o1 = lift97(xo_prev, c1, e0_prev, e0);      // position 2m-1
      const float e2 = lift97(e0_prev, c2, o1_prev, o1);      // position 2m-2
      const float o3 = lift97(o1_prev, c3, e2_prev, e2);      // position 2m-3
      p[(2 * m - 2) * st] = e2;
      p[(2 * m - 3) * st] = o3;
      xo_prev = xo;
      e0_prev = e0;
      o1_prev = o1;
      e2_prev = e2;
    }
  }
}

template <bool REV>
__device__ __forceinline__ typename DwtTypes<REV>::T *dwt_buf(int id, void *a, void *b, void *c) {
  typedef typename DwtTypes<REV>::T T;
  return (T *)(id == 0 ? a : (id == 1 ? b : c));
}

// Shared memory of one CTA: the staged window, the reference-compat column-end inputs and
// the source row / column of every window line (mirrored, low or high part)
template <bool REV>
struct DwtSmem {
  typename DwtTypes<REV>::T tile[DWT_N * DWT_PITCH];
  typename DwtTypes<REV>::T keep[2][DWT_T];
  int32_t srow[DWT_N], scol[DWT_N];
};

// Inputs of one window: the level's Mallat quadrants (`quad`) and the LL quadrant
// (`llsrc`, another buffer for every level but the first)
template <bool REV>
struct WinSrc {
  const typename DwtTypes<REV>::T *quad;
  int stride_q;
  const typename DwtTypes<REV>::T *llsrc;
  int stride_ll;
};

// Rebuild the 64x64 output tile at (ox, oy) of one level for `nw` windows of the same
// geometry (the components of one tile at their last level, or one tile-component): the
// results are left in the centre of each window, S[w].tile[(y + 4) * DWT_PITCH + x + 4].
template <bool REV>
__device__ __forceinline__ void dwt_windows(DwtSmem<REV> *S, int nw, const WinSrc<REV> *src, int rw, int rh, int lw,
                                            int lh, bool ll_gain, float gain, bool refcompat, int ox, int oy) {
  typedef typename DwtTypes<REV>::T T;
  // source line of every window row / column: window index i <-> position o - 4 + i, whose
  // mirror keeps its parity, so even window lines come from the low part and odd ones
  // from the high part (the same for every window)
  for (int i = threadIdx.x; i < 2 * DWT_N; i += blockDim.x) {
    const bool col = i >= DWT_N;
    const int w = col ? i - DWT_N : i;
    const int n = col ? rw : rh, lo = col ? lw : lh;
    // the window may reach far past a level smaller than the tile: full periodic mirror
    const int x = mirror((col ? ox : oy) - DWT_H + w, n);
    const int sl = (x & 1) ? lo + (x >> 1) : (x >> 1);
    if (col) S[0].scol[w] = sl;
    else S[0].srow[w] = sl;
  }
  __syncthreads();
  // stage quadrant by quadrant with asynchronous 4-byte copies (cp.async): every thread
  // issues all of its loads before waiting, so a CTA has all its windows in flight;
  // consecutive threads read consecutive source columns
  constexpr int QN = DWT_N / 2;  // 36 window lines of each parity
  // a warp copies one quadrant row at a time; each lane holds the source columns of
  // quadrant columns j = lane and (lanes 0..3) j = lane + 32, for both parities
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const bool two = lane < QN - 32;
  const int sc_e0 = S[0].scol[2 * lane], sc_o0 = S[0].scol[2 * lane + 1];
  const int sc_e1 = two ? S[0].scol[2 * (lane + 32)] : 0, sc_o1 = two ? S[0].scol[2 * (lane + 32) + 1] : 0;
  for (int w = 0; w < nw; ++w) {
    const uint32_t tile_s = (uint32_t)__cvta_generic_to_shared(S[w].tile);
#pragma unroll
    for (int qd = 0; qd < 4; ++qd) {  // quadrant LL, HL, LH, HH
      const T *qbase = qd == 0 ? src[w].llsrc : src[w].quad;
      const int qstride = qd == 0 ? src[w].stride_ll : src[w].stride_q;
      const int odd = qd & 1;
      const T *lo0 = qbase + (odd ? sc_o0 : sc_e0), *lo1 = qbase + (odd ? sc_o1 : sc_e1);
      const uint32_t d0 = tile_s + 4u * (odd + 2 * lane), d1 = d0 + 4u * 64;
#pragma unroll 2
      for (int r = warp; r < QN; r += nwarps) {
        const int iy = 2 * r + (qd >> 1);
        const size_t row = (size_t)S[0].srow[iy] * qstride;
        const uint32_t drow = 4u * iy * DWT_PITCH;
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d0 + drow), "l"(lo0 + row));
        if (two) asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d1 + drow), "l"(lo1 + row));
      }
    }
  }
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  __syncthreads();
  if (!REV && ll_gain) {
    // the reconstructed LL entering a finer 9/7 level is scaled by K_lo^2
    for (int e = threadIdx.x; e < nw * QN * QN; e += blockDim.x) {
      const int w = e / (QN * QN), q = e - w * QN * QN, r = q / QN, j = q - r * QN;
      T *v = S[w].tile + 2 * r * DWT_PITCH + 2 * j;
      *v = (T)__fmul_rn((float)*v, gain);
    }
    __syncthreads();
  }
  if (rw > 1) {
    for (int l = threadIdx.x; l < nw * DWT_N; l += blockDim.x) {
      const int w = l / DWT_N, r = l - w * DWT_N;
      lift_line<REV>(S[w].tile + r * DWT_PITCH, 1);
    }
    __syncthreads();
  }
  // reference-compat: keep the horizontally transformed inputs the column end reads
  const int n = rh;
  const bool fix = REV && refcompat && n >= 3 && (oy <= n - 1) && (n - 2 < oy + DWT_T);
  int rowA = -1, rowB = -1;
  if (fix) {
    if (!(n & 1)) {
      rowA = n - 3;  // H[m-2]
    } else {
      const int m = (n + 1) / 2;
      rowA = n - 3;                 // L[m-2]
      rowB = (m >= 3) ? n - 4 : 1;  // H[m-3] (H[0] when m == 2)
    }
    for (int e = threadIdx.x; e < nw * DWT_T; e += blockDim.x) {
      const int w = e / DWT_T, c = e - w * DWT_T;
      S[w].keep[0][c] = S[w].tile[(rowA - oy + DWT_H) * DWT_PITCH + DWT_H + c];
      if (rowB >= 0) S[w].keep[1][c] = S[w].tile[(rowB - oy + DWT_H) * DWT_PITCH + DWT_H + c];
    }
    __syncthreads();
  }
  if (rh > 1) {
    for (int l = threadIdx.x; l < nw * DWT_T; l += blockDim.x) {
      const int w = l / DWT_T, c = l - w * DWT_T;
      lift_line<REV>(S[w].tile + DWT_H + c, DWT_PITCH);
    }
    __syncthreads();
  }
  if constexpr (REV) {
    if (fix) {
      for (int e = threadIdx.x; e < nw * DWT_T; e += blockDim.x) {
        const int w = e / DWT_T, c = e - w * DWT_T;
        T *col = S[w].tile + DWT_H + c;
        const int r1 = n - 1 - oy + DWT_H, r2 = n - 2 - oy + DWT_H, r3 = n - 3 - oy + DWT_H;
        if (!(n & 1)) {
          col[r1 * DWT_PITCH] = S[w].keep[0][c] + col[r2 * DWT_PITCH];
        } else {
          const T hx = S[w].keep[1][c];
          const T x1 = S[w].keep[0][c] - ((hx + 1) >> 1);
          col[r1 * DWT_PITCH] = x1;
          col[r2 * DWT_PITCH] = hx + ((x1 + col[r3 * DWT_PITCH]) >> 1);
        }
      }
      __syncthreads();
    }
  }
}

// One 64x64 output tile of one level of one tile-component, stored to `out`.
template <bool REV>
__device__ __forceinline__ void dwt_tile(DwtSmem<REV> &S, const typename DwtTypes<REV>::T *quad, int stride_q,
                                         const typename DwtTypes<REV>::T *llsrc, int stride_ll,
                                         typename DwtTypes<REV>::T *out, int stride_out, int rw, int rh, int lw,
                                         int lh, bool ll_gain, float gain, bool refcompat, int ox, int oy) {
  const WinSrc<REV> src{quad, stride_q, llsrc, stride_ll};
  dwt_windows<REV>(&S, 1, &src, rw, rh, lw, lh, ll_gain, gain, refcompat, ox, oy);
  const int ow = min(DWT_T, rw - ox), oh = min(DWT_T, rh - oy);
  for (int i = threadIdx.x; i < DWT_T * DWT_T; i += blockDim.x) {
    const int yy = i / DWT_T, xx = i % DWT_T;
    if (yy < oh && xx < ow)
      out[(size_t)(oy + yy) * stride_out + ox + xx] = S.tile[(yy + DWT_H) * DWT_PITCH + xx + DWT_H];
  }
  __syncthreads();
}

template <bool REV>
__global__ void __launch_bounds__(DWT_THREADS) dwt_level_kernel(const DwtLevel *__restrict__ levels,
                                                        const DwtTask *__restrict__ tasks, int ntasks, void *bufA,
                                                        void *bufB, void *bufC, float ll_gain_value) {
  typedef typename DwtTypes<REV>::T T;
  __shared__ DwtSmem<REV> S;
  for (int task = blockIdx.x; task < ntasks; task += gridDim.x) {
    const DwtTask tk = tasks[task];
    const DwtLevel L = levels[tk.level];
    const T *A = dwt_buf<REV>(0, bufA, bufB, bufC) + L.base;
    const T *LLsrc = dwt_buf<REV>(L.ll_src, bufA, bufB, bufC) + L.base;
    T *out = dwt_buf<REV>(L.out_dst, bufA, bufB, bufC) + L.base;
    dwt_tile<REV>(S, A, L.stride, LLsrc, L.stride, out, L.stride, L.rw, L.rh, L.lw, L.lh, L.ll_gain != 0,
                  ll_gain_value, L.refcompat != 0, tk.tx * DWT_T, tk.ty * DWT_T);
  }
}

// ------------------------------------------------------------------ output stage -------
__device__ __forceinline__ int clampi(int v, int hi) { return v < 0 ? 0 : (v > hi ? hi : v); }
__device__ __forceinline__ int lift_depth(int v, int in, int out) { return in >= out ? v >> (in - out) : v << (out - in); }

// bytes per pixel and container depth of a reference OutputFormat
__device__ __host__ __forceinline__ int fmt_bytes(int fmt) {
  switch (fmt) {
    case 0: return 4;
    case 1: return 6;
    case 2: return 3;
    case 3: return 4;
    case 4: return 8;
    case 5: return 6;
    case 6: return 3;
    case 8: return 8;
    default: return 0;
  }
}

__device__ __forceinline__ void put_slot(uint8_t *px, int pxb, int slot, int v) {
  // reference pixel structs store the highest component index first (codec_base.h:51-143)
  if (pxb == 3) px[2 - slot] = (uint8_t)v;
  else if (pxb == 4) px[3 - slot] = (uint8_t)v;
  else if (pxb == 6) ((uint16_t *)px)[2 - slot] = (uint16_t)v;
  else ((uint16_t *)px)[3 - slot] = (uint16_t)v;
}

// Last level of every component of one tile with the output stage fused into its store:
// the components' windows stay in shared memory and the packed pixels are the only write.
struct FusedGroup {
  OutGroup G;
  uint64_t base[3];  // element offset of each component's region (same in every buffer)
  int8_t ll_src[3];  // buffer of each component's LL quadrant: 0 coefficients, 1 B, 2 C
  int8_t ll_gain, refcompat;
  int32_t stride, rw, rh, lw, lh;
};

// Inverse RCT (5/3, int) or ICT (9/7, float) + DC level shift + clamp of one pixel: R, G, B
// (RRct_53 :3936-4130, RICT_97_FLOAT :3570-3643 of bmi_cpu_dwt_decoder.cpp)
template <typename T>
__device__ __forceinline__ void mct_pixel(T y, T u, T w, int dc, int maxv, int *rgb) {
  if constexpr (std::is_integral<T>::value) {
    const int g = (int)y - (((int)u + (int)w) >> 2) + dc;
    rgb[0] = clampi((int)w + g, maxv);
    rgb[1] = clampi(g, maxv);
    rgb[2] = clampi((int)u + g, maxv);
  } else {
    const float sh = (float)dc, fm = (float)maxv;
    float t = __fadd_rn(__fadd_rn(y, __fmul_rn(1.402f, w)), sh);
    rgb[0] = (int)(t < 0.f ? 0.f : (t > fm ? fm : t));
    t = __fadd_rn(__fadd_rn(__fadd_rn(y, __fmul_rn(-0.34413f, u)), __fmul_rn(-0.71414f, w)), sh);
    rgb[1] = (int)(t < 0.f ? 0.f : (t > fm ? fm : t));
    t = __fadd_rn(__fadd_rn(y, __fmul_rn(1.772f, u)), sh);
    rgb[2] = (int)(t < 0.f ? 0.f : (t > fm ? fm : t));
  }
}

// Inverse RCT / ICT + DC level shift + clamp + LIFT + pack of one pixel (bmi_cpu_dwt_decoder.cpp
// RICT_97_FLOAT :3570-3643, RRct_53 :3936-4130, MergeComponents :4283-4598).  `v[c]` is
// component c's reconstructed sample (int32 for 5/3, float for 9/7), `have[c]` whether the
// component is present.
template <typename T>
__device__ __forceinline__ void emit_pixel(const OutGroup &G, uint8_t *out, int yy, int xx, const T *v,
                                           const bool *have) {
  const int pxb = fmt_bytes(G.fmt);
  const int B = G.bitdepth;
  const int outdepth = (pxb == 3 || pxb == 4) ? 8 : 16;
  const int maxv = (1 << B) - 1, dc = 1 << (B - 1);
  const bool rgb = (G.fmt == 0 || G.fmt == 1 || G.fmt == 2 || G.fmt == 8);
  const bool do_mct = rgb && G.mct && G.ncomp >= 3 && have[1] && have[2];
  const int slot0 = (pxb == 4 || pxb == 8) ? 1 : 0;
  uint8_t *px = out + G.out_off + ((size_t)(G.y0 + yy) * G.pitch_px + (G.x0 + xx)) * pxb;
  uint8_t tmp[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  if (do_mct) {
    int c3[3];
    mct_pixel<T>(v[0], v[1], v[2], dc, maxv, c3);
    if (G.checkout >= 0 && G.checkout < 3) {
      // one component replicated into R, G and B (RICT_97_FLOAT / RRct_53 case 0..2)
      const int vv = lift_depth(c3[G.checkout], B, outdepth);
      for (int k = 0; k < 3; ++k) put_slot(tmp, pxb, k + slot0, vv);
    } else {
      for (int k = 0; k < 3; ++k) put_slot(tmp, pxb, k + slot0, lift_depth(c3[k], B, outdepth));
    }
  } else if (G.checkout >= 0 && have[G.checkout]) {
    // MergeComponents with a checked-out component: value in R = G = B, and in the
    // alpha slot only for the 4-component formats (bmi_cpu_dwt_decoder.cpp:4300-4308)
    const int vv = lift_depth(clampi((int)v[G.checkout] + dc, maxv), B, outdepth);
    if (pxb == 3 || pxb == 6) {
      for (int k = 0; k < 3; ++k) put_slot(tmp, pxb, k, vv);
    } else {
      for (int k = 1; k < 4; ++k) put_slot(tmp, pxb, k, vv);
      if (G.fmt == 3 || G.fmt == 4) put_slot(tmp, pxb, 0, vv);
    }
  } else {
    for (int c = 0; c < G.ncomp && c < 4; ++c) {
      if (!have[c]) continue;
      if ((pxb == 3 || pxb == 6) && c > 2) continue;
      put_slot(tmp, pxb, c, lift_depth(clampi((int)v[c] + dc, maxv), B, outdepth));
    }
  }
  for (int k = 0; k < pxb; ++k) px[k] = tmp[k];
}

#ifndef J2K_DWT_LEVELS_ONLY
// Output stage for tiles whose last level was not fused: reads the reconstructed
// components from the level buffers.
__global__ void __launch_bounds__(256) output_kernel(const OutGroup *__restrict__ groups,
                                                     const OutTask *__restrict__ tasks, int ntasks, const void *bufA,
                                                     const void *bufB, const void *bufC, uint8_t *out) {
  for (int task = blockIdx.x; task < ntasks; task += gridDim.x) {
    const OutTask tk = tasks[task];
    const OutGroup G = groups[tk.group];
    const void *cb[4];
    bool have[4];
    for (int c = 0; c < 4; ++c) {
      const void *bb = G.comp_buf[c] == 0 ? bufA : (G.comp_buf[c] == 1 ? bufB : bufC);
      cb[c] = G.comp_buf[c] < 0 ? nullptr : (const void *)((const uint8_t *)bb + G.comp_off[c] * 4);
      have[c] = cb[c] != nullptr;
    }
    const int ox = tk.tx * 64, oy = tk.ty * 64;
    for (int i = threadIdx.x; i < 64 * 64; i += blockDim.x) {
      const int yy = oy + i / 64, xx = ox + i % 64;
      if (yy >= G.h || xx >= G.w) continue;
      size_t at[4];
      for (int c = 0; c < 4; ++c) {
        at[c] = (size_t)yy * G.stride[c] + xx;
        if (G.sampled && have[c]) {  // replicate a sub-sampled component's nearest-left sample
          const int i = min(max((G.ax + xx) / G.sx[c] - G.cx[c], 0), G.cw[c] - 1);
          const int j = min(max((G.ay + yy) / G.sy[c] - G.cy[c], 0), G.ch[c] - 1);
          at[c] = (size_t)j * G.stride[c] + i;
        }
      }
      if (G.rev) {
        int32_t v[4] = {0, 0, 0, 0};
        for (int c = 0; c < 4; ++c)
          if (have[c]) v[c] = ((const int32_t *)cb[c])[at[c]];
        emit_pixel<int32_t>(G, out, yy, xx, v, have);
      } else {
        float v[4] = {0.f, 0.f, 0.f, 0.f};
        for (int c = 0; c < 4; ++c)
          if (have[c]) v[c] = ((const float *)cb[c])[at[c]];
        emit_pixel<float>(G, out, yy, xx, v, have);
      }
    }
  }
}

// Last DWT level of up to three components of one tile fused with the output stage (the
// inverse MCT reads the components' windows in shared memory): one CTA per 64x64 tile.
// Dynamic shared memory: `nwin` DwtSmem windows.
template <bool REV>
__global__ void __launch_bounds__(FUSED_THREADS) last_level_output_kernel(const FusedGroup *__restrict__ groups,
                                                                        const OutTask *__restrict__ tasks, int ntasks,
                                                                        void *bufA, void *bufB, void *bufC,
                                                                        float ll_gain_value, uint8_t *out) {
  typedef typename DwtTypes<REV>::T T;
  extern __shared__ __align__(16) uint8_t dsm[];
  DwtSmem<REV> *S = reinterpret_cast<DwtSmem<REV> *>(dsm);
  for (int task = blockIdx.x; task < ntasks; task += gridDim.x) {
    const OutTask tk = tasks[task];
    const FusedGroup &F = groups[tk.group];
    const OutGroup G = F.G;
    const int nc = min(3, (int)G.ncomp);
    WinSrc<REV> src[3];
    bool have[4] = {false, false, false, false};
    for (int c = 0; c < nc; ++c) {
      const T *A = dwt_buf<REV>(0, bufA, bufB, bufC) + F.base[c];
      src[c] = {A, F.stride, dwt_buf<REV>(F.ll_src[c], bufA, bufB, bufC) + F.base[c], F.stride};
      have[c] = true;
    }
    const int ox = tk.tx * DWT_T, oy = tk.ty * DWT_T;
    dwt_windows<REV>(S, nc, src, F.rw, F.rh, F.lw, F.lh, F.ll_gain != 0, ll_gain_value, F.refcompat != 0, ox, oy);
    const int ow = min(DWT_T, F.rw - ox), oh = min(DWT_T, F.rh - oy);
    if (G.fmt == 2 && G.bitdepth == 8 && G.mct && nc == 3) {
      // 24-bit RGB after the inverse MCT (the common path): sixteen pixels per thread (48
      // bytes, bytes B, G, R per pixel) go out as three 16-byte stores when the run is
      // 16-byte aligned and whole, else as 32-bit words or bytes
      constexpr int RUN = 16;
      for (int i = threadIdx.x; i < DWT_T * (DWT_T / RUN); i += blockDim.x) {
        const int yy = i / (DWT_T / RUN), xx = (i % (DWT_T / RUN)) * RUN;
        if (yy >= oh || xx >= ow) continue;
        uint8_t *px = out + G.out_off + ((size_t)(G.y0 + oy + yy) * G.pitch_px + (G.x0 + ox + xx)) * 3;
        uint32_t words[12];
#pragma unroll
        for (int j = 0; j < 12; ++j) words[j] = 0;
        const int npx = min(RUN, ow - xx);
#pragma unroll
        for (int k = 0; k < RUN; ++k) {
          const int o = (yy + DWT_H) * DWT_PITCH + xx + k + DWT_H;
          int rgb[3];
          mct_pixel<T>(S[0].tile[o], S[1].tile[o], S[2].tile[o], 128, 255, rgb);
#pragma unroll
          for (int j = 0; j < 3; ++j) {
            const int b = k * 3 + j;  // byte j of pixel k: B, G, R
            words[b >> 2] |= (uint32_t)rgb[2 - j] << (8 * (b & 3));
          }
        }
        if (npx == RUN && !((uintptr_t)px & 15)) {
          uint4 *v = reinterpret_cast<uint4 *>(px);
          v[0] = make_uint4(words[0], words[1], words[2], words[3]);
          v[1] = make_uint4(words[4], words[5], words[6], words[7]);
          v[2] = make_uint4(words[8], words[9], words[10], words[11]);
        } else if (npx == RUN && !((uintptr_t)px & 3)) {
#pragma unroll
          for (int j = 0; j < 12; ++j) reinterpret_cast<uint32_t *>(px)[j] = words[j];
        } else {
          // a partial or unaligned run (picture edge, odd widths): pixel by pixel, recomputed
          // so that `words` stays in registers
          for (int k = 0; k < npx; ++k) {
            const int o = (yy + DWT_H) * DWT_PITCH + xx + k + DWT_H;
            int rgb[3];
            mct_pixel<T>(S[0].tile[o], S[1].tile[o], S[2].tile[o], 128, 255, rgb);
            px[3 * k] = (uint8_t)rgb[2];
            px[3 * k + 1] = (uint8_t)rgb[1];
            px[3 * k + 2] = (uint8_t)rgb[0];
          }
        }
      }
    } else {
      for (int i = threadIdx.x; i < DWT_T * DWT_T; i += blockDim.x) {
        const int yy = i / DWT_T, xx = i % DWT_T;
        if (yy >= oh || xx >= ow) continue;
        T v[4] = {0, 0, 0, 0};
        for (int c = 0; c < nc; ++c) v[c] = S[c].tile[(yy + DWT_H) * DWT_PITCH + xx + DWT_H];
        emit_pixel<T>(G, out, oy + yy, ox + xx, v, have);
      }
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------------ coarse levels -------
// The coarsest levels of a tile-component are tiny (a 512x512 tile-component with five
// levels synthesises 32x32 and 64x64 before its first 128x128 level), so one launch per
// level leaves the GPU idle between short grids.  Here one CTA synthesises every level up to
// resolution `rc` of one tile-component in shared memory: the top-left res_w[rc] x res_h[rc]
// block of the tile-component's Mallat region already holds LL and every band up to that
// resolution, so it is staged once, each level is rebuilt in place (rows into a second
// buffer, columns back), and resolution rc is written once to the level buffer the level
// kernels would have left it in.  Arithmetic is the per-level kernels' (and the oracle's):
// whole-sample symmetric lifting over the full line, the same rounded float operations,
// K_lo^2 on a reconstructed 9/7 LL, the reference's 5/3 column end on request.
constexpr int COARSE_MAX = 64;  // largest resolution edge synthesised here
struct CoarseTask {
  uint64_t base;      // element offset of the tile-component region
  int32_t stride;     // tile-component width
  int8_t rc;          // resolutions 1..rc are synthesised here
  int8_t out_dst;     // buffer receiving resolution rc: 1 B, 2 C
  int8_t refcompat;   // 5/3: reference column-end arithmetic
  int8_t pad;
  int16_t res_w[8], res_h[8];  // resolutions 0..rc (rc <= 7: 64 << 7 exceeds any level kept here)
};

// In-place inverse lifting of one interleaved line of n samples (element stride st), the
// oracle's line97 / line53: x[-1] = x[1], x[n] = x[n - 2]
template <bool REV>
__device__ __forceinline__ void lift_full_line(typename DwtTypes<REV>::T *x, int n, int st) {
  if (n < 2) return;
  auto at = [&](int i) -> typename DwtTypes<REV>::T & {
    const int j = i < 0 ? -i : (i >= n ? 2 * (n - 1) - i : i);
    return x[j * st];
  };
  if constexpr (REV) {
    for (int i = 0; i < n; i += 2) at(i) = at(i) - ((at(i - 1) + at(i + 1) + 2) >> 2);
    for (int i = 1; i < n; i += 2) at(i) = at(i) + ((at(i - 1) + at(i + 1)) >> 1);
  } else {
    for (int i = 0; i < n; i += 2) at(i) = lift97(at(i), 0.44350685204397f, at(i - 1), at(i + 1));
    for (int i = 1; i < n; i += 2) at(i) = lift97(at(i), 0.88291107553093f, at(i - 1), at(i + 1));
    for (int i = 0; i < n; i += 2) at(i) = lift97(at(i), -0.05298011857296f, at(i - 1), at(i + 1));
    for (int i = 1; i < n; i += 2) at(i) = lift97(at(i), -1.58613434205992f, at(i - 1), at(i + 1));
  }
}

template <bool REV>
__global__ void __launch_bounds__(128) dwt_coarse_kernel(const CoarseTask *__restrict__ tasks, int ntasks, void *bufA,
                                                          void *bufB, void *bufC, float ll_gain_value) {
  typedef typename DwtTypes<REV>::T T;
  constexpr int P = COARSE_MAX + 1;  // odd pitch
  __shared__ T X[COARSE_MAX * P], Y[COARSE_MAX * P];
  for (int task = blockIdx.x; task < ntasks; task += gridDim.x) {
    const CoarseTask tk = tasks[task];
    const T *A = dwt_buf<REV>(0, bufA, bufB, bufC) + tk.base;
    T *out = dwt_buf<REV>(tk.out_dst, bufA, bufB, bufC) + tk.base;
    const int W = tk.res_w[tk.rc], H = tk.res_h[tk.rc];
    for (int i = threadIdx.x; i < W * H; i += blockDim.x) {
      const int y = i / W, x = i - y * W;
      X[y * P + x] = A[(size_t)y * tk.stride + x];
    }
    __syncthreads();
    for (int r = 1; r <= tk.rc; ++r) {
      const int rw = tk.res_w[r], rh = tk.res_h[r], lw = tk.res_w[r - 1], lh = tk.res_h[r - 1];
      if (!REV && r > 1) {  // the reconstructed LL entering a finer 9/7 level
        for (int i = threadIdx.x; i < lw * lh; i += blockDim.x) {
          const int y = i / lw, x = i - y * lw;
          X[y * P + x] = (T)__fmul_rn((float)X[y * P + x], ll_gain_value);
        }
        __syncthreads();
      }
      // rows: interleave low / high parts into Y, lift
      for (int y = threadIdx.x; y < rh; y += blockDim.x) {
        T *row = Y + y * P;
        for (int i = 0; i < rw; ++i) row[i] = X[y * P + ((i & 1) ? lw + (i >> 1) : (i >> 1))];
        lift_full_line<REV>(row, rw, 1);
      }
      __syncthreads();
      // columns: interleave low / high rows back into X, lift (5/3: the reference's column
      // end on request, from the column's de-interleaved inputs as in the level kernels)
      for (int x = threadIdx.x; x < rw; x += blockDim.x) {
        T *col = X + x;
        for (int i = 0; i < rh; ++i) col[i * P] = Y[((i & 1) ? lh + (i >> 1) : (i >> 1)) * P + x];
        if constexpr (REV) {
          const int n = rh;
          const bool fix = tk.refcompat && n >= 3;
          T a = 0, b = 0;
          if (fix) {
            if (!(n & 1)) {
              a = Y[(lh + n / 2 - 2) * P + x];  // H[m - 2]
            } else {
              const int m = (n + 1) / 2;
              b = Y[(lh + (m >= 3 ? m - 3 : 0)) * P + x];  // H[m - 3] (H[0] when m == 2)
              a = Y[(m - 2) * P + x];                       // L[m - 2]
            }
          }
          lift_full_line<REV>(col, rh, P);
          if (fix) {
            if (!(n & 1)) {
              col[(n - 1) * P] = a + col[(n - 2) * P];
            } else {
              const T x1 = a - ((b + 1) >> 1);
              col[(n - 1) * P] = x1;
              col[(n - 2) * P] = b + ((x1 + col[(n - 3) * P]) >> 1);
            }
          }
        } else {
          lift_full_line<REV>(col, rh, P);
        }
      }
      __syncthreads();
    }
    for (int i = threadIdx.x; i < W * H; i += blockDim.x) {
      const int y = i / W, x = i - y * W;
      out[(size_t)y * tk.stride + x] = X[y * P + x];
    }
    __syncthreads();
  }
}
#endif  // J2K_DWT_LEVELS_ONLY

}  // namespace j2k_dev

namespace j2k_dev {

// One level of one tile-component with every buffer given explicitly (no descriptor
// tables in device memory): the CTA index selects the 64x64 output tile.  Used by the
// entry point that runs on a static scratch array (noalloc.cu).
template <bool REV>
__global__ void __launch_bounds__(DWT_THREADS) dwt_level_explicit_kernel(
    const typename DwtTypes<REV>::T *__restrict__ quad, int stride_q, const typename DwtTypes<REV>::T *llsrc,
    int stride_ll, typename DwtTypes<REV>::T *out, int stride_out, int rw, int rh, int lw, int lh, int ll_gain,
    float ll_gain_value, int refcompat) {
  __shared__ DwtSmem<REV> S;
  const int tiles_x = (rw + DWT_T - 1) / DWT_T;
  dwt_tile<REV>(S, quad, stride_q, llsrc, stride_ll, out, stride_out, rw, rh, lw, lh, ll_gain != 0, ll_gain_value,
                refcompat != 0, (blockIdx.x % tiles_x) * DWT_T, (blockIdx.x / tiles_x) * DWT_T);
}

}  // namespace j2k_dev
