// Pyramidal Lucas-Kanade, one warp per track.
//
// Per level (coarse to fine) a warp stages the integer-pixel window under its 9x9 patch in shared
// memory (12x12 texels per image: the 10x10 the bilinear taps touch plus a one-texel margin), computes
// the 81 bilinear taps from shared memory (3 per lane, lane-major like the reference), and reduces
// with xor-butterfly shuffles; every Gauss-Newton iteration re-stages the current frame's window at
// the new position.  A CTA holds 8 independent warps; tracks of all cameras form one flattened list.
//
// The algorithm and evaluation order are lk_track_kernel / lk_track_horizontal_kernel
// (lk_tracker.cu:69-379, 381-665): window weights gauss9(i)*gauss9(j), mean-subtracted gradients,
// H = sum w g g^T plus 1/32 per lane, mean-compensated residual, at most 11 iterations per level,
// stop when |v|^2 < 0.12^2 (|v| < 0.12 horizontally), level search-radius gate, 5x5 NCC gate, and
// coordinates scaled by 2 about (0.5, 0.5) between levels.  Texture sampling is restated in
// software: FE_SAMPLE_TEXTURE uses cudaFilterModeLinear's 8-bit-fraction weight rule (round-half-up
// fractions; corner products rounded half up, cross products half down), FE_SAMPLE_EXACT exact
// weights.  Divisions are IEEE (the reference's __fdividef differs by <= 2 ulp).
#include <cuda_runtime.h>

#include "fe_common.cuh"
#include "fe_internal.h"

namespace fe {

namespace {

constexpr int kWarps = 8;
constexpr int kWin = 12;               // staged window edge (texels)
constexpr int kWinStride = kWin + 1;   // padded row
constexpr int kWinSize = kWin * kWinStride;
constexpr int kNE = 3;                 // taps per lane: ceil(81 / 32)

struct Tap {
  int off;          // window offset of the top-left texel
  float w00, w10, w01, w11;
};

// Texel base and bilinear weights of a tap at texture coordinate (px, py), relative to the window
// origin (bx, by).  Texel i covers [i, i+1): taps floor(p - 0.5) and +1.
template <int SAMPLING>
__device__ __forceinline__ Tap make_tap(float px, float py, int bx, int by) {
  const float xb = __fsub_rn(px, 0.5f), yb = __fsub_rn(py, 0.5f);
  const float fx = floorf(xb), fy = floorf(yb);
  const float a = __fsub_rn(xb, fx), b = __fsub_rn(yb, fy);
  Tap t;
  t.off = ((int)fy - by) * kWinStride + ((int)fx - bx);
  if (SAMPLING == FE_SAMPLE_TEXTURE) {
    const int A = (int)floorf(__fmaf_rn(a, 256.f, 0.5f)), B = (int)floorf(__fmaf_rn(b, 256.f, 0.5f));
    const int p00 = (256 - A) * (256 - B), p10 = A * (256 - B), p01 = (256 - A) * B, p11 = A * B;
    t.w00 = (float)((p00 + 128) >> 8) * (1.f / 256.f);
    t.w10 = (float)((p10 + 127) >> 8) * (1.f / 256.f);
    t.w01 = (float)((p01 + 127) >> 8) * (1.f / 256.f);
    t.w11 = (float)((p11 + 128) >> 8) * (1.f / 256.f);
  } else {
    t.w00 = a;  // exact mode keeps the fractions; see sample()
    t.w10 = b;
    t.w01 = 0.f;
    t.w11 = 0.f;
  }
  return t;
}

template <int SAMPLING>
__device__ __forceinline__ float sample(const float* win, const Tap& t) {
  const float t00 = win[t.off], t10 = win[t.off + 1];
  const float t01 = win[t.off + kWinStride], t11 = win[t.off + kWinStride + 1];
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

// Stage the kWin x kWin texels starting at (bx, by), clamped to the image.
__device__ __forceinline__ void stage(float* win, const float* img, int pitch, int w, int h, int bx, int by,
                                      int lane) {
  for (int i = lane; i < kWin * kWin; i += 32) {
    const int r = i / kWin, c = i - r * kWin;
    const int y = min(max(by + r, 0), h - 1), x = min(max(bx + c, 0), w - 1);
    win[r * kWinStride + c] = __ldg(img + (size_t)y * pitch + x);
  }
}

template <int SAMPLING, bool HORIZ>
__global__ void __launch_bounds__(kWarps * 32) lk_kernel(const __grid_constant__ LkLaunch p) {
  __shared__ float swin[kWarps][3][kWinSize];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int g = blockIdx.x * kWarps + wid;
  if (g >= p.total) return;  // warp-uniform
  const LkCam* cams = p.cams ? p.cams : &p.single;
  int lo = 0, hi = p.ncams - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (cams[mid].begin <= g) lo = mid; else hi = mid - 1;
  }
  const LkCam& cam = cams[lo];
  fe_track_data& td = cam.tracks[g - cam.begin];
  float* w_img = swin[wid][0];
  float* w_gx = swin[wid][1];
  float* w_gy = swin[wid][2];

  const float radius = td.search_radius_px;
  const float ncc_thr = td.ncc_threshold;
  if (radius < 0.f) {
    if (lane == 0) td.track_status = 0;
    return;
  }
  __syncwarp();
  if (lane < 4) td.info[lane] = (lane == 0 || lane == 3) ? 1.f / 9.f : 0.f;

  const int levels = cam.prev.levels;
  const int top = levels - 1;
  const float tx = td.track[0], ty = td.track[1];
  const float cx0 = __fadd_rn(tx, td.offset[0]), cy0 = __fadd_rn(ty, td.offset[1]);
  const float W0 = (float)cam.prev.lv[0].w, H0 = (float)cam.prev.lv[0].h;
  const float CW0 = (float)cam.cur.lv[0].w, CH0 = (float)cam.cur.lv[0].h;
  if (!(tx >= 0.f && tx < W0 && ty >= 0.f && ty < H0) || !(cx0 >= 0.f && cx0 < CW0 && cy0 >= 0.f && cy0 < CH0)) {
    if (lane == 0) td.track_status = 0;
    return;
  }
  const float scale = 1.f / (float)(1 << top);
  float sx = __fmaf_rn(__fsub_rn(tx, 0.5f), scale, 0.5f), sy = __fmaf_rn(__fsub_rn(ty, 0.5f), scale, 0.5f);
  float cx = __fmaf_rn(__fsub_rn(cx0, 0.5f), scale, 0.5f), cy = __fmaf_rn(__fsub_rn(cy0, 0.5f), scale, 0.5f);

  // this lane's taps: flat f = lane + 32 e
  float ixf[kNE], iyf[kNE], wt[kNE];
  bool valid[kNE], nccm[kNE];
#pragma unroll
  for (int e = 0; e < kNE; ++e) {
    const int f = lane + 32 * e;
    const int iy = f / 9, ix = f - iy * 9;
    valid[e] = f < 81;
    nccm[e] = valid[e] && ix >= 2 && ix < 7 && iy >= 2 && iy < 7;
    ixf[e] = (float)ix;
    iyf[e] = (float)iy;
    wt[e] = valid[e] ? gauss9(iy) * gauss9(ix) : 0.f;
  }
  const float rcp81 = 1.f / 81.f, rcp25 = 1.f / 25.f;
  const float thr2 = 0.12f * 0.12f;
  bool conv = false;

  for (int i = 0; i < levels; ++i) {
    const int level = top - i;
    const Level& PL = cam.prev.lv[level];
    const Level& CL = cam.cur.lv[level];
    const int W = CL.w, H = CL.h;
    float xmin = __fadd_rn(sx, -4.f), ymin = __fadd_rn(sy, -4.f);
    // the patch box must lie inside the level (written so that a NaN position also fails)
    bool good = xmin >= 0.f && __fadd_rn(sx, 5.f) < (float)W && ymin >= 0.f && __fadd_rn(sy, 5.f) < (float)H;
    if (good) {
      // previous-frame patch: image and gradients
      int bx = (int)floorf(__fsub_rn(xmin, 0.5f)) - 1, by = (int)floorf(__fsub_rn(ymin, 0.5f)) - 1;
      __syncwarp();
      stage(w_img, PL.img, PL.pitch, PL.w, PL.h, bx, by, lane);
      stage(w_gx, PL.gx, PL.pitch, PL.w, PL.h, bx, by, lane);
      if (!HORIZ) stage(w_gy, PL.gy, PL.pitch, PL.w, PL.h, bx, by, lane);
      __syncwarp();
      float gxp[kNE], gyp[kNE], p1[kNE];
      float sgx = 0.f, sgy = 0.f, sp = 0.f;
#pragma unroll
      for (int e = 0; e < kNE; ++e) {
        gxp[e] = gyp[e] = p1[e] = 0.f;
        if (valid[e]) {
          const Tap t = make_tap<SAMPLING>(__fadd_rn(xmin, ixf[e]), __fadd_rn(ymin, iyf[e]), bx, by);
          gxp[e] = sample<SAMPLING>(w_gx, t);
          if (!HORIZ) gyp[e] = sample<SAMPLING>(w_gy, t);
          p1[e] = sample<SAMPLING>(w_img, t);
          sgx = __fadd_rn(sgx, gxp[e]);
          if (!HORIZ) sgy = __fadd_rn(sgy, gyp[e]);
          sp = __fadd_rn(sp, p1[e]);
        }
      }
      sgx = warp_sum(sgx);
      if (!HORIZ) sgy = warp_sum(sgy);
      sp = warp_sum(sp);
      float lxx = 1.f / 32.f, lxy = 0.f, lyy = 1.f / 32.f;
#pragma unroll
      for (int e = 0; e < kNE; ++e) {
        if (valid[e]) {
          const float a = __fmaf_rn(-sgx, rcp81, gxp[e]);
          gxp[e] = a;
          if (HORIZ) {
            lxx = __fmaf_rn(__fmul_rn(wt[e], a), a, lxx);
          } else {
            const float bq = __fmaf_rn(-sgy, rcp81, gyp[e]);
            gyp[e] = bq;
            lxx = __fmaf_rn(__fmul_rn(a, a), wt[e], lxx);
            lxy = __fmaf_rn(__fmul_rn(a, bq), wt[e], lxy);
            lyy = __fmaf_rn(__fmul_rn(bq, bq), wt[e], lyy);
          }
        }
      }
      const float gxx = warp_sum(lxx);
      const float gxy = HORIZ ? 0.f : warp_sum(lxy);
      const float gyy = HORIZ ? 0.f : warp_sum(lyy);
      float det_rcp;
      if (HORIZ) {
        if (gxx < 1.1920928955078125e-07f) {
          if (lane == 0) td.track_status = 0;
          return;
        }
        det_rcp = __fdiv_rn(1.f, gxx);
      } else {
        const float det = __fmaf_rn(gxx, gyy, -__fmul_rn(gxy, gxy));
        if (det < 1.1920928955078125e-07f) {
          if (lane == 0) td.track_status = 0;
          return;
        }
        det_rcp = __fdiv_rn(1.f, det);
      }
      const float savex = cx, savey = cy;
      float p2[kNE];
#pragma unroll
      for (int e = 0; e < kNE; ++e) p2[e] = 0.f;
      for (int it = 0; it < 11; ++it) {
        xmin = __fadd_rn(cx, -4.f);
        ymin = __fadd_rn(cy, -4.f);
        if (!(xmin >= 0.f && __fadd_rn(cx, 5.f) < (float)W && ymin >= 0.f && __fadd_rn(cy, 5.f) < (float)H)) good = false;
        if (!good) break;
        bx = (int)floorf(__fsub_rn(xmin, 0.5f)) - 1;
        by = (int)floorf(__fsub_rn(ymin, 0.5f)) - 1;
        __syncwarp();
        stage(w_img, CL.img, CL.pitch, CL.w, CL.h, bx, by, lane);
        __syncwarp();
        float sc = 0.f;
#pragma unroll
        for (int e = 0; e < kNE; ++e) {
          if (valid[e]) {
            const Tap t = make_tap<SAMPLING>(__fadd_rn(xmin, ixf[e]), __fadd_rn(ymin, iyf[e]), bx, by);
            p2[e] = sample<SAMPLING>(w_img, t);
            sc = __fadd_rn(sc, p2[e]);
          }
        }
        sc = warp_sum(sc);
        const float delta = __fmul_rn(__fsub_rn(sc, sp), rcp81);
        float ex = 0.f, ey = 0.f;
#pragma unroll
        for (int e = 0; e < kNE; ++e) {
          if (valid[e]) {
            const float diff = __fsub_rn(__fsub_rn(p2[e], p1[e]), delta);
            const float wd = __fmul_rn(wt[e], diff);
            ex = __fmaf_rn(wd, gxp[e], ex);
            if (!HORIZ) ey = __fmaf_rn(wd, gyp[e], ey);
          }
        }
        ex = warp_sum(ex);
        float vx, vy;
        if (HORIZ) {
          vx = __fmul_rn(ex, det_rcp);
          vy = 0.f;
          conv = fabsf(vx) < 0.12f;
        } else {
          ey = warp_sum(ey);
          vx = __fmul_rn(__fmaf_rn(gyy, ex, -__fmul_rn(gxy, ey)), det_rcp);
          vy = __fmul_rn(__fmaf_rn(gxx, ey, -__fmul_rn(gxy, ex)), det_rcp);
          conv = __fmaf_rn(vx, vx, __fmul_rn(vy, vy)) < thr2;
        }
        if (conv) break;
        cx = __fadd_rn(cx, vx);
        cy = __fadd_rn(cy, vy);
      }
      if (conv) {
        const float r = __fdiv_rn(radius, (float)(1 << level));
        const float dx = __fsub_rn(cx, savex), dy = __fsub_rn(cy, savey);
        if (__fmaf_rn(dx, dx, __fmul_rn(dy, dy)) > __fmul_rn(r, r)) conv = false;
      }
      if (conv) {
        float s1 = 0.f, s2 = 0.f, s11 = 0.f, s22 = 0.f, s12 = 0.f;
#pragma unroll
        for (int e = 0; e < kNE; ++e) {
          if (nccm[e]) {
            s1 = __fadd_rn(s1, p1[e]);
            s2 = __fadd_rn(s2, p2[e]);
            s11 = __fmaf_rn(p1[e], p1[e], s11);
            s22 = __fmaf_rn(p2[e], p2[e], s22);
            s12 = __fmaf_rn(p2[e], p1[e], s12);
          }
        }
        s1 = warp_sum(s1);
        s2 = warp_sum(s2);
        s11 = warp_sum(s11);
        s22 = warp_sum(s22);
        s12 = warp_sum(s12);
        const float a1 = __fmul_rn(s1, rcp25), a2 = __fmul_rn(s2, rcp25);
        const float d1 = __fmaf_rn(s11, rcp25, -__fmul_rn(a1, a1));
        const float d2 = __fmaf_rn(s22, rcp25, -__fmul_rn(a2, a2));
        const float d12 = __fmaf_rn(s12, rcp25, -__fmul_rn(a1, a2));
        const float d1d2 = __fmul_rn(d1, d2);
        const float ncc = d1d2 < 1.1920928955078125e-07f ? 0.f : __fmul_rn(d12, __frsqrt_rn(d1d2));
        conv = ncc > ncc_thr;
      }
      if (!conv && level > 0) {
        cx = savex;
        cy = savey;
      }
      conv = (level == 0) && conv;
    }
    if (i != levels - 1) {
      sx = __fmaf_rn(sx, 2.f, -0.5f);
      sy = __fmaf_rn(sy, 2.f, -0.5f);
      cx = __fmaf_rn(cx, 2.f, -0.5f);
      cy = __fmaf_rn(cy, 2.f, -0.5f);
    }
  }
  __syncwarp();
  if (lane == 0) {
    if (conv) {
      td.track[0] = cx;
      td.track[1] = cy;
    }
    td.track_status = conv ? 1 : 0;
  }
}

}  // namespace

cudaError_t launch_lk(const LkLaunch& p, cudaStream_t s) {
  if (p.total <= 0) return cudaSuccess;
  const int blocks = (p.total + kWarps - 1) / kWarps;
  if (p.sampling == FE_SAMPLE_EXACT) {
    if (p.horizontal) lk_kernel<FE_SAMPLE_EXACT, true><<<blocks, kWarps * 32, 0, s>>>(p);
    else lk_kernel<FE_SAMPLE_EXACT, false><<<blocks, kWarps * 32, 0, s>>>(p);
  } else {
    if (p.horizontal) lk_kernel<FE_SAMPLE_TEXTURE, true><<<blocks, kWarps * 32, 0, s>>>(p);
    else lk_kernel<FE_SAMPLE_TEXTURE, false><<<blocks, kWarps * 32, 0, s>>>(p);
  }
  return cudaGetLastError();
}

}  // namespace fe
