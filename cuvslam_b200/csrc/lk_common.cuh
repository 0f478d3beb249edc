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

template <int SAMPLING>
__device__ __forceinline__ TapSet make_taps(float xmin, float ymin, int bx, int by, int stride, int lane) {
  TapSet s;
  const bool is_col = lane < 9, is_row = lane >= 16 && lane < 25;
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

struct WarpSmem {
  float img[kPW * kPS];
  float gx[kPW * kPS];
  float gy[kPW * kPS];
  float cur[kCW * kCS];
};

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
