// Shared device pieces of the LK tracker (lk.cu) and its adjoint (lk_adjoint.cu): window sizes,
// the bilinear tap geometry of a 9x9 patch, sampling from shared-memory windows and window staging.
// The taps are those lk_track_kernel fetches from its linear-filtered textures (lk_tracker.cu:69-379,
// texture setup cuda_helper.h:402-431).
#pragma once

#include <cuda_runtime.h>

#include "fe_common.cuh"

namespace fe {
namespace lk {

constexpr int kPW = 12, kPS = 13;  // previous-frame window 12x12, row stride 13
constexpr int kCW = 16, kCS = 17;  // current-frame window 16x16, row stride 17
// The tracker's windows start at a 16-byte aligned column (the origin rounded down to a multiple of
// 4 texels) and are staged as 16-byte row chunks: 12 rows of 4 chunks (16 texels) for the previous
// frame, 16 rows of 5 chunks (20 texels) for the current frame, which covers the 12- and 16-texel
// windows from any origin.
constexpr int kPA = 4, kPAS = 16;  // previous-frame chunks per row, row stride
constexpr int kCA = 5, kCAS = 20;  // current-frame chunks per row, row stride
constexpr int kNE = 3;             // taps per lane: ceil(81 / 32)
constexpr unsigned kFull = 0xffffffffu;

struct Tap {
  int off;  // window offset of the top-left texel
  float w00, w10, w01, w11;
};

// Texture-unit weights for quantised fractions A, B (in 1/256).
__device__ __forceinline__ void tex_weights(int A, int B, Tap& t) {
  const int p00 = (256 - A) * (256 - B), p10 = A * (256 - B), p01 = (256 - A) * B, p11 = A * B;
  t.w00 = (float)((p00 + 128) >> 8) * (1.f / 256.f);
  t.w10 = (float)((p10 + 127) >> 8) * (1.f / 256.f);
  t.w01 = (float)((p01 + 127) >> 8) * (1.f / 256.f);
  t.w11 = (float)((p11 + 128) >> 8) * (1.f / 256.f);
}

// Sampling state of one 9x9 patch whose first sample is at texture coordinate (xmin, ymin).
// Texel i covers [i, i+1): a sample at p has taps floor(p - 0.5) and +1 with fraction
// (p - 0.5) - floor(p - 0.5); the sample coordinates are xmin + i, ymin + j rounded to FP32 as the
// reference computes them.  Lanes 0-8 hold column i's values, lanes 16-24 row j's.
struct TapSet {
  Tap u;         // the weights (and offset of tap (0,0)) shared by all taps when `uniform`
  bool uniform;
  int base, q;   // this lane's column/row: texel index and quantised fraction
  float fr;      // this lane's column/row fraction
};

// Texture-unit weight rule (8-bit fractions) in both texture modes.
constexpr bool quantised(int sampling) { return sampling != FE_SAMPLE_EXACT; }

// PER_LANE = false: in the common case the per-lane column/row values (only the non-uniform taps
// read them) are left at zero.
template <int SAMPLING, bool PER_LANE = true>
__device__ __forceinline__ TapSet make_taps(float xmin, float ymin, int bx, int by, int stride, int lane) {
  TapSet s;
  const bool is_col = lane < 9, is_row = lane >= 16 && lane < 25;
  // Common case, decided warp-uniformly without shuffles: when xmin and xmin + 8 share an FP32
  // exponent (no binade boundary inside the patch; xmin >= 0 here), every xmin + i is exact, and
  // so are the - 0.5 and the fraction; the columns then have consecutive texels and one fraction,
  // and the same holds for the rows.  The per-lane values below are those the general path
  // computes, which would find the taps uniform too.
  if ((((__float_as_uint(xmin) ^ __float_as_uint(__fadd_rn(xmin, 8.f))) |
        (__float_as_uint(ymin) ^ __float_as_uint(__fadd_rn(ymin, 8.f)))) >> 23) == 0) {
    const float pbx = __fsub_rn(xmin, 0.5f), pby = __fsub_rn(ymin, 0.5f);
    const float flx = floorf(pbx), fly = floorf(pby);
    const float frx = __fsub_rn(pbx, flx), fry = __fsub_rn(pby, fly);
    const int b0x = (int)flx, b0y = (int)fly;
    const int q0x = quantised(SAMPLING) ? (int)floorf(__fmaf_rn(frx, 256.f, 0.5f)) : 0;
    const int q0y = quantised(SAMPLING) ? (int)floorf(__fmaf_rn(fry, 256.f, 0.5f)) : 0;
    s.uniform = true;
    if (PER_LANE) {
      s.base = is_col ? b0x + lane : (is_row ? b0y + (lane - 16) : b0y);
      s.fr = is_col ? frx : fry;
      s.q = is_col ? q0x : q0y;
    } else {
      s.base = s.q = 0;
      s.fr = 0.f;
    }
    if (quantised(SAMPLING)) {
      tex_weights(q0x, q0y, s.u);
    } else {
      s.u.w00 = frx;
      s.u.w10 = fry;
      s.u.w01 = s.u.w11 = 0.f;
    }
    s.u.off = (b0y - by) * stride + (b0x - bx);
    return s;
  }
  const float p = is_col ? __fadd_rn(xmin, (float)lane) : __fadd_rn(ymin, (float)(is_row ? lane - 16 : 0));
  const float pb = __fsub_rn(p, 0.5f);
  const float fl = floorf(pb);
  s.fr = __fsub_rn(pb, fl);
  s.base = (int)fl;
  s.q = quantised(SAMPLING) ? (int)floorf(__fmaf_rn(s.fr, 256.f, 0.5f)) : 0;
  const int base0x = __shfl_sync(kFull, s.base, 0), base0y = __shfl_sync(kFull, s.base, 16);
  const int q0x = __shfl_sync(kFull, s.q, 0), q0y = __shfl_sync(kFull, s.q, 16);
  const float fr0x = __shfl_sync(kFull, s.fr, 0), fr0y = __shfl_sync(kFull, s.fr, 16);
  bool ok = true;
  if (is_col) ok = s.base == base0x + lane && (quantised(SAMPLING) ? s.q == q0x : s.fr == fr0x);
  if (is_row) ok = s.base == base0y + (lane - 16) && (quantised(SAMPLING) ? s.q == q0y : s.fr == fr0y);
  s.uniform = __all_sync(kFull, ok);
  if (quantised(SAMPLING)) {
    tex_weights(q0x, q0y, s.u);
  } else {
    s.u.w00 = fr0x;
    s.u.w10 = fr0y;
    s.u.w01 = s.u.w11 = 0.f;
  }
  s.u.off = (base0y - by) * stride + (base0x - bx);
  return s;
}

// Tap (ix, iy) of a patch.  All lanes must call it together (the non-uniform case shuffles).
template <int SAMPLING>
__device__ __forceinline__ Tap tap_of(const TapSet& s, int ix, int iy, int bx, int by, int stride) {
  if (s.uniform) {
    Tap t = s.u;
    t.off += iy * stride + ix;
    return t;
  }
  // a column or row rounded differently: this tap takes its own column's and row's values
  Tap t;
  const int bxe = __shfl_sync(kFull, s.base, ix), bye = __shfl_sync(kFull, s.base, 16 + iy);
  t.off = (bye - by) * stride + (bxe - bx);
  if (quantised(SAMPLING)) {
    tex_weights(__shfl_sync(kFull, s.q, ix), __shfl_sync(kFull, s.q, 16 + iy), t);
  } else {
    t.w00 = __shfl_sync(kFull, s.fr, ix);
    t.w10 = __shfl_sync(kFull, s.fr, 16 + iy);
    t.w01 = t.w11 = 0.f;
  }
  return t;
}

template <int SAMPLING>
__device__ __forceinline__ float sample(const float* win, int stride, const Tap& t) {
  const float t00 = win[t.off], t10 = win[t.off + 1];
  const float t01 = win[t.off + stride], t11 = win[t.off + stride + 1];
  if (SAMPLING == FE_SAMPLE_TEXTURE_WIDE) {
    // w * t is exact in FP64 (9 + 24 significant bits): the sum is rounded to FP32 once
    double v = __dmul_rn((double)t.w00, (double)t00);
    v = __fma_rn((double)t.w10, (double)t10, v);
    v = __fma_rn((double)t.w01, (double)t01, v);
    return __double2float_rn(__fma_rn((double)t.w11, (double)t11, v));
  }
  if (SAMPLING == FE_SAMPLE_TEXTURE) {
    float v = __fmul_rn(t.w00, t00);
    v = __fmaf_rn(t.w10, t10, v);
    v = __fmaf_rn(t.w01, t01, v);
    return __fmaf_rn(t.w11, t11, v);
  }
  const float top = __fmaf_rn(t.w00, __fsub_rn(t10, t00), t00);
  const float bot = __fmaf_rn(t.w00, __fsub_rn(t11, t01), t01);
  return __fmaf_rn(t.w10, __fsub_rn(bot, top), top);
}

// Stage the n x n texels starting at (bx, by), clamped to the image (the texture's clamp mode), as
// asynchronous copies; the caller waits (cp_async_wait_all) and then __syncwarp()s.
template <int N, int S>
__device__ __forceinline__ void stage(float* win, const float* img, int pitch, int w, int h, int bx, int by,
                                      int lane) {
#pragma unroll
  for (int i = lane; i < N * N; i += 32) {
    const int r = i / N, c = i - r * N;
    const int y = min(max(by + r, 0), h - 1), x = min(max(bx + c, 0), w - 1);
    cp_async4(win + r * S + c, img + (size_t)y * pitch + x);
  }
}

// Rows [by, by + ROWS) x columns [ax, ax + 4 CHUNKS) (ax a multiple of 4) of NP planes that share
// one pitch, clamped to the image as the texture's clamp mode: 16-byte asynchronous copies when the
// block lies inside the image (its rows start 16-byte aligned: 16-byte aligned planes and pitches),
// else one texel at a time, each lane owning a column (its clamped x computed once) and a share of
// the rows.  The caller waits (cp_async_wait_all) and then __syncwarp()s.
template <int ROWS, int CHUNKS, int S, int NP>
__device__ __forceinline__ void stage_planes(float* const (&win)[NP], const float* const (&img)[NP], int pitch, int w,
                                             int h, int ax, int by, int lane) {
  if (ax >= 0 && by >= 0 && ax + 4 * CHUNKS <= w && by + ROWS <= h) {
#pragma unroll
    for (int i = lane; i < ROWS * CHUNKS; i += 32) {
      const int r = i / CHUNKS, k = i - r * CHUNKS;
      const size_t go = (size_t)(by + r) * pitch + ax + 4 * k;
#pragma unroll
      for (int q = 0; q < NP; ++q) cp_async16(win[q] + r * S + 4 * k, img[q] + go);
    }
  } else {
    constexpr int C = 4 * CHUNKS, LPC = 32 / C;  // columns, lanes per column
    static_assert(LPC >= 1, "a warp covers a row");
    if (lane < C * LPC) {
      const int c = lane % C;
      const int x = min(max(ax + c, 0), w - 1);
#pragma unroll 4
      for (int r = lane / C; r < ROWS; r += LPC) {
        const size_t go = (size_t)min(max(by + r, 0), h - 1) * pitch + x;
#pragma unroll
        for (int q = 0; q < NP; ++q) cp_async4(win[q] + r * S + c, img[q] + go);
      }
    }
  }
}

template <int ROWS, int CHUNKS, int S>
__device__ __forceinline__ void stage_aligned(float* win, const float* img, int pitch, int w, int h, int ax, int by,
                                              int lane) {
  float* const wv[1] = {win};
  const float* const iv[1] = {img};
  stage_planes<ROWS, CHUNKS, S, 1>(wv, iv, pitch, w, h, ax, by, lane);
}

// Windows of one warp: sized for both the adjoint's layout (kPS / kCS strides) and the tracker's
// aligned one (kPAS / kCAS); 16-byte aligned for the chunked copies.
struct alignas(16) WarpSmem {
  float img[kPW * kPAS];
  float gx[kPW * kPAS];
  float gy[kPW * kPAS];
  float cur[kCW * kCAS];
};
static_assert(kPW * kPAS >= kPW * kPS && kCW * kCAS >= kCW * kCS, "window arrays hold both layouts");
static_assert(kPW * kPAS % 4 == 0 && kCW * kCAS % 4 == 0, "16-byte aligned window arrays");
static_assert(4 * kPA >= kPW + 3 && 4 * kCA >= kCW + 3, "aligned windows cover the windows from any origin");

// Value and spatial derivative of the bilinear interpolant at tap t (exact weights: t.w00 = fx,
// t.w10 = fy).  The value is computed exactly as sample<FE_SAMPLE_EXACT>.
__device__ __forceinline__ void sample_vg(const float* win, int stride, const Tap& t, float& v, float& dx, float& dy) {
  const float t00 = win[t.off], t10 = win[t.off + 1];
  const float t01 = win[t.off + stride], t11 = win[t.off + stride + 1];
  const float ax = __fsub_rn(t10, t00), bx = __fsub_rn(t11, t01);
  const float top = __fmaf_rn(t.w00, ax, t00);
  const float bot = __fmaf_rn(t.w00, bx, t01);
  v = __fmaf_rn(t.w10, __fsub_rn(bot, top), top);
  dx = __fmaf_rn(t.w10, __fsub_rn(bx, ax), ax);
  dy = __fsub_rn(bot, top);
}

// What the unrolled differentiable tracker did on each level, for its adjoint (global memory, one
// per track, written by lane 0): template position, the sampled iterates then the end position,
// each step's update v and brightness offset delta = mean P2 - mean P1, the number of steps, flags
// 1 = template built, 2 = level accepted.
constexpr int kMaxRecIt = 16;
struct LkRecord {
  float2 s[kMaxLevels];
  float2 it[kMaxLevels][kMaxRecIt + 1];
  float2 v[kMaxLevels][kMaxRecIt];
  float delta[kMaxLevels][kMaxRecIt];
  int K[kMaxLevels];
  int flags[kMaxLevels];
};

}  // namespace lk
}  // namespace fe
