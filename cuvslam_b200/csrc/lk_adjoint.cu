// Adjoint of the differentiable LK tracker: one warp per track computes the track's gradient
// contributions to the pyramids' planes as small window records; a tile-segmented reduction sums
// the records of every 32x32 tile of every plane in track order; the pyramid adjoint then applies
// the transposed gradient filters and the transposed 5x5 decimation from the top level down to the
// level-0 images.  Everything is deterministic: no floating-point atomics.  No counterpart in the
// reference, which has no backward; the forward it differentiates follows lk_track_kernel's rule
// (lk_tracker.cu:69-379).
//
// Forward model (lk_track.cuh, exact bilinear sampling): per level l a template at s_l
// (P1, Gx, Gy on the 9x9 taps; a = Gx - mean, b = Gy - mean; H = I + sum w g g^T) and steps
// c += v, v = H^-1 e(c), e = sum w r g, r = P2(c) - P1 - (mean P2 - mean P1).
//
// Implicit mode (implicit-function theorem at the converged level-0 displacement c*, where
// e(c*) = 0): J = de/dc = sum w g (dP2/dc - mean dP2/dc)^T, J^T lambda = dL/dc*, and
// dL/dtheta = -lambda^T de/dtheta, i.e. per tap
//   dL/dP2 = u - mean u, dL/dP1 = -(u - mean u), u = -w (lambda . g),
//   dL/dGx = ab - mean ab, ab = -w r lambda_x  (Gy likewise).
// Unrolled mode: the forward's record of every step (iterate, update v, brightness offset; written by
// lk_track.cuh) is differentiated step by step backwards, patches re-sampled from the pyramids
// rather than stored:
//   mu = H^-1 cbar, Hbar -= mu v^T, dL/dP2 = u - mean u with u = w (mu . g), cbar += sum dL/dP2 dP2/dc,
//   dL/dP1 -= dL/dP2, abar += w r mu_x, bbar += w r mu_y; after the level
//   abar += w (2 Hbar_xx a + (Hbar_xy + Hbar_yx) b), bbar likewise, dL/dGx = abar - mean abar.
// Template positions receive sum dL/dP1 dP1/ds + dL/dGx dGx/ds + dL/dGy dGy/ds; positions map
// between levels as s_l = 2 s_{l+1} - 1/2.
#include <cuda_runtime.h>

#include <climits>

#include "fe_common.cuh"
#include "fe_internal.h"
#include "lk_common.cuh"
#include "lk_track.cuh"

namespace fe {

namespace {

using namespace lk;

constexpr int kAdjWarps = 4;
constexpr int kRP = 12;  // previous-image record edge (the template's 12x12 window)
constexpr int kTile = 32;
constexpr int kGatherThreads = 256;
constexpr int kGatherWarps = kGatherThreads / 32;
constexpr int kWarpList = 32;  // most records per tile that one warp sums (gather_warp_kernel)
constexpr int kLongThreads = 1024;  // gather_long_kernel: one CTA per SM, 32 warps per long tile
constexpr int kLongWarps = kLongThreads / 32;

struct AdjSmem {
  WarpSmem win;               // staging windows, as the forward
  float acc[32 * 32];         // current-image record
  float prec[3][kRP * kRP];   // previous-image records
  float coef[3][81];          // tap coefficients (serial scatter)
  int cb[9], rb[9];           // column / row texel index (serial scatter)
  float cf[9], rf[9];         // column / row fraction
};

// Adds the transposed bilinear taps of NP coefficient sets (tap f = lane + 32 e) into shared-memory
// records dst[p] (row stride rs, origin (rx0, ry0) in level texels).  Texel indices are clamped to
// the W x H level as the forward's staged windows clamp them.  When all taps share their fractions
// and none clamps, four conflict-free passes (one per bilinear corner) add the taps; otherwise lane 0
// adds every tap in order.  Both are deterministic.
template <int NP>
__device__ void scatter_taps(float* const (&dst)[NP], int rs, int rx0, int ry0, const TapSet& ts,
                             const float (&c)[NP][kNE], const bool (&valid)[kNE], const int (&ix)[kNE],
                             const int (&iy)[kNE], int W, int H, AdjSmem& sm, int lane) {
  const int b0x = __shfl_sync(kFull, ts.base, 0), b0y = __shfl_sync(kFull, ts.base, 16);
  __syncwarp();
  if (ts.uniform && b0x >= 0 && b0y >= 0 && b0x + 9 <= W - 1 && b0y + 9 <= H - 1) {
    const float fx = ts.u.w00, fy = ts.u.w10;
    const float gx = __fsub_rn(1.f, fx), gy = __fsub_rn(1.f, fy);
    const float wc[4] = {__fmul_rn(gx, gy), __fmul_rn(fx, gy), __fmul_rn(gx, fy), __fmul_rn(fx, fy)};
#pragma unroll
    for (int corner = 0; corner < 4; ++corner) {
      const int cx = corner & 1, cy = corner >> 1;
#pragma unroll
      for (int e = 0; e < kNE; ++e) {
        if (valid[e]) {
          const int o = (b0y + iy[e] + cy - ry0) * rs + (b0x + ix[e] + cx - rx0);
#pragma unroll
          for (int q = 0; q < NP; ++q) dst[q][o] = __fmaf_rn(wc[corner], c[q][e], dst[q][o]);
        }
      }
      __syncwarp();
    }
    return;
  }
#pragma unroll
  for (int e = 0; e < kNE; ++e)
    if (valid[e])
#pragma unroll
      for (int q = 0; q < NP; ++q) sm.coef[q][lane + 32 * e] = c[q][e];
  if (lane < 9) {
    sm.cb[lane] = ts.base;
    sm.cf[lane] = ts.fr;
  }
  if (lane >= 16 && lane < 25) {
    sm.rb[lane - 16] = ts.base;
    sm.rf[lane - 16] = ts.fr;
  }
  __syncwarp();
  if (lane == 0) {
    for (int f = 0; f < 81; ++f) {
      const int i = f % 9, j = f / 9;
      const float fx = sm.cf[i], fy = sm.rf[j];
      const float gx = __fsub_rn(1.f, fx), gy = __fsub_rn(1.f, fy);
      const int x0 = min(max(sm.cb[i], 0), W - 1) - rx0, x1 = min(max(sm.cb[i] + 1, 0), W - 1) - rx0;
      const int y0 = min(max(sm.rb[j], 0), H - 1) - ry0, y1 = min(max(sm.rb[j] + 1, 0), H - 1) - ry0;
#pragma unroll
      for (int q = 0; q < NP; ++q) {
        const float v = sm.coef[q][f];
        dst[q][y0 * rs + x0] = __fmaf_rn(__fmul_rn(gx, gy), v, dst[q][y0 * rs + x0]);
        dst[q][y0 * rs + x1] = __fmaf_rn(__fmul_rn(fx, gy), v, dst[q][y0 * rs + x1]);
        dst[q][y1 * rs + x0] = __fmaf_rn(__fmul_rn(gx, fy), v, dst[q][y1 * rs + x0]);
        dst[q][y1 * rs + x1] = __fmaf_rn(__fmul_rn(fx, fy), v, dst[q][y1 * rs + x1]);
      }
    }
  }
  __syncwarp();
}

__device__ __forceinline__ void zero_smem(float* p, int n, int lane) {
  for (int i = lane; i < n; i += 32) p[i] = 0.f;
  __syncwarp();
}

// Copies a w x h shared-memory record (row stride rs) to its global slot (row stride gs).
__device__ __forceinline__ void store_record(float* dst, int gs, const float* src, int rs, int w, int h, int lane) {
  for (int i = lane; i < w * h; i += 32) {
    const int r = i / w, c = i - r * w;
    dst[r * gs + c] = src[r * rs + c];
  }
}

// The template of one level: the previous-frame windows staged at the patch under s, the taps'
// samples, the mean-subtracted gradients and (unrolled) H, all as lk_track.cuh computes them.
struct Templ {
  float p1[kNE], a[kNE], b[kNE];
  float sp, gxx, gxy, gyy, det_rcp;
  int bx, by;  // the patch's 12x12 texel window
  int ax;      // its staged window's first column (bx rounded down to a multiple of 4)
  float sx, sy;  // the template position (its tap set is recomputed where needed, not kept live)
};

// The current-image window for a patch at c, staged from the 16-byte aligned column at or below
// the patch's first texel minus 2 when the window (wbx, wby) does not cover the patch's 12x12 texels
// (the tracker's rule, lk_track.cuh); the caller waits.  Returns whether it staged.
__device__ __forceinline__ bool stage_cur(const Level& CL, float cx, float cy, int& wbx, int& wby, AdjSmem& sm,
                                          int lane) {
  const float xmin = __fadd_rn(cx, -4.f), ymin = __fadd_rn(cy, -4.f);
  const int nbx = (int)floorf(__fsub_rn(xmin, 0.5f)) - 1, nby = (int)floorf(__fsub_rn(ymin, 0.5f)) - 1;
  if (nbx < wbx || nbx + kPW > wbx + 4 * kCA || nby < wby || nby + kPW > wby + kCW) {
    wbx = (nbx - 2) & ~3;
    wby = nby - 2;
    stage_aligned<kCW, kCA, kCAS>(sm.win.cur, CL.img, CL.pitch, CL.w, CL.h, wbx, wby, lane);
    return true;
  }
  return false;
}

// CL (may be null): the current image, whose window for the first patch at c (wbx, wby updated) is
// staged together with the template's so that one wait covers both.
__device__ void make_template(const Level& PL, float sx, float sy, const bool (&valid)[kNE], const int (&ix)[kNE],
                              const int (&iy)[kNE], const float (&wt)[kNE], AdjSmem& sm, int lane, Templ& T,
                              const Level* CL = nullptr, float2 c = make_float2(0.f, 0.f), int* wbx = nullptr,
                              int* wby = nullptr) {
  const float rcp81 = 1.f / 81.f;
  const float xmin = __fadd_rn(sx, -4.f), ymin = __fadd_rn(sy, -4.f);
  T.bx = (int)floorf(__fsub_rn(xmin, 0.5f)) - 1;
  T.by = (int)floorf(__fsub_rn(ymin, 0.5f)) - 1;
  T.ax = T.bx & ~3;
  __syncwarp();
  {
    float* const wv[3] = {sm.win.img, sm.win.gx, sm.win.gy};
    const float* const iv[3] = {PL.img, PL.gx, PL.gy};
    stage_planes<kPW, kPA, kPAS, 3>(wv, iv, PL.pitch, PL.w, PL.h, T.ax, T.by, lane);
  }
  if (CL) stage_cur(*CL, c.x, c.y, *wbx, *wby, sm, lane);
  cp_async_wait_all();
  __syncwarp();
  T.sx = sx;
  T.sy = sy;
  const TapSet ts = make_taps<FE_SAMPLE_EXACT>(xmin, ymin, T.ax, T.by, kPAS, lane);
  float gxp[kNE], gyp[kNE];
  float sgx = 0.f, sgy = 0.f, sp = 0.f;
#pragma unroll
  for (int e = 0; e < kNE; ++e) {
    gxp[e] = gyp[e] = T.p1[e] = 0.f;
    const Tap t = tap_of<FE_SAMPLE_EXACT>(ts, ix[e], iy[e], T.ax, T.by, kPAS);
    if (valid[e]) {
      gxp[e] = sample<FE_SAMPLE_EXACT>(sm.win.gx, kPAS, t);
      gyp[e] = sample<FE_SAMPLE_EXACT>(sm.win.gy, kPAS, t);
      T.p1[e] = sample<FE_SAMPLE_EXACT>(sm.win.img, kPAS, t);
      sgx = __fadd_rn(sgx, gxp[e]);
      sgy = __fadd_rn(sgy, gyp[e]);
      sp = __fadd_rn(sp, T.p1[e]);
    }
  }
  warp_sum3(sgx, sgy, sp, lane);
  T.sp = sp;
  float lxx = 1.f / 32.f, lxy = 0.f, lyy = 1.f / 32.f;
#pragma unroll
  for (int e = 0; e < kNE; ++e) {
    T.a[e] = T.b[e] = 0.f;
    if (valid[e]) {
      T.a[e] = __fmaf_rn(-sgx, rcp81, gxp[e]);
      T.b[e] = __fmaf_rn(-sgy, rcp81, gyp[e]);
      lxx = __fmaf_rn(__fmul_rn(T.a[e], T.a[e]), wt[e], lxx);
      lxy = __fmaf_rn(__fmul_rn(T.a[e], T.b[e]), wt[e], lxy);
      lyy = __fmaf_rn(__fmul_rn(T.b[e], T.b[e]), wt[e], lyy);
    }
  }
  warp_sum3(lxx, lxy, lyy, lane);
  T.gxx = lxx;
  T.gxy = lxy;
  T.gyy = lyy;
  T.det_rcp = __fdiv_rn(1.f, __fmaf_rn(T.gxx, T.gyy, -__fmul_rn(T.gxy, T.gxy)));
}

// Writes the three previous-image records of (level, track) from the template adjoint and returns
// dL/ds (the template position) through (dsx, dsy).  The staged windows of make_template are read.
__device__ void finish_template(const AdjLaunch& p, int g, int level, int W, int H, const Templ& T,
                                const float (&p1b)[kNE], const float (&gxb)[kNE], const float (&gyb)[kNE],
                                const bool (&valid)[kNE], const int (&ix)[kNE], const int (&iy)[kNE], AdjSmem& sm,
                                int lane, float& dsx, float& dsy) {
  // dL/ds from the staged windows
  const TapSet ts = make_taps<FE_SAMPLE_EXACT>(__fadd_rn(T.sx, -4.f), __fadd_rn(T.sy, -4.f), T.ax, T.by, kPAS, lane);
  float sx = 0.f, sy = 0.f;
#pragma unroll
  for (int e = 0; e < kNE; ++e) {
    const Tap t = tap_of<FE_SAMPLE_EXACT>(ts, ix[e], iy[e], T.ax, T.by, kPAS);
    if (valid[e]) {
      float v, dx, dy;
      sample_vg(sm.win.img, kPAS, t, v, dx, dy);
      sx = __fmaf_rn(p1b[e], dx, sx);
      sy = __fmaf_rn(p1b[e], dy, sy);
      sample_vg(sm.win.gx, kPAS, t, v, dx, dy);
      sx = __fmaf_rn(gxb[e], dx, sx);
      sy = __fmaf_rn(gxb[e], dy, sy);
      sample_vg(sm.win.gy, kPAS, t, v, dx, dy);
      sx = __fmaf_rn(gyb[e], dx, sx);
      sy = __fmaf_rn(gyb[e], dy, sy);
    }
  }
  warp_sum2(sx, sy, lane);
  dsx = sx;
  dsy = sy;
  // records
  const int rx0 = max(T.bx, 0), ry0 = max(T.by, 0);
  zero_smem(&sm.prec[0][0], 3 * kRP * kRP, lane);
  float* const dst[3] = {sm.prec[0], sm.prec[1], sm.prec[2]};
  const float c[3][kNE] = {{p1b[0], p1b[1], p1b[2]}, {gxb[0], gxb[1], gxb[2]}, {gyb[0], gyb[1], gyb[2]}};
  scatter_taps<3>(dst, kRP, rx0, ry0, ts, c, valid, ix, iy, W, H, sm, lane);
  const int rw = min(kRP, W - rx0), rh = min(kRP, H - ry0);
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const size_t slot = ((size_t)q * p.L + level) * p.total + g;
    store_record(p.data_prev + slot * (kRP * kRP), kRP, sm.prec[q], kRP, rw, rh, lane);
    if (lane == 0) p.hdr[slot] = make_int4(rx0, ry0, rw, rh);
  }
}

__device__ __forceinline__ void empty_level(const AdjLaunch& p, int g, int level, int lane) {
  if (lane < 4) p.hdr[((size_t)lane * p.L + level) * p.total + g] = make_int4(0, 0, 0, 0);
}

__device__ __forceinline__ void finish_track(const AdjCam& cam, int i, float gtx, float gty, float gox, float goy,
                                             int lane) {
  if (lane == 0) {
    if (cam.grad_track) reinterpret_cast<float2*>(cam.grad_track)[i] = make_float2(gtx, gty);
    if (cam.grad_offset) reinterpret_cast<float2*>(cam.grad_offset)[i] = make_float2(gox, goy);
  }
}

// The current-image window for a patch at c (staged and waited for when it does not cover the
// patch) and the patch's tap set.
__device__ __forceinline__ TapSet cur_taps(const Level& CL, float cx, float cy, int& wbx, int& wby, AdjSmem& sm,
                                           int lane) {
  __syncwarp();
  if (stage_cur(CL, cx, cy, wbx, wby, sm, lane)) {
    cp_async_wait_all();
    __syncwarp();
  }
  return make_taps<FE_SAMPLE_EXACT>(__fadd_rn(cx, -4.f), __fadd_rn(cy, -4.f), wbx, wby, kCAS, lane);
}

__device__ __forceinline__ int patch_base(float c) {
  return (int)floorf(__fsub_rn(__fadd_rn(c, -4.f), 0.5f));
}

template <int MODE>
__device__ void adjoint_one(const AdjLaunch& p, const AdjCam& cam, int g, AdjSmem& sm, int lane) {
  const int i = g - cam.lk.begin;
  const fe_track_data& tin = cam.lk.tracks_in[i];
  const float2 gout = reinterpret_cast<const float2*>(cam.grad_xy)[i];
  const int levels = cam.lk.prev.levels, top = levels - 1;
  const float rcp81 = 1.f / 81.f;

  int ix[kNE], iy[kNE];
  float wt[kNE];
  bool valid[kNE];
#pragma unroll
  for (int e = 0; e < kNE; ++e) {
    const int f = lane + 32 * e;
    valid[e] = f < 81;
    iy[e] = valid[e] ? f / 9 : 0;
    ix[e] = valid[e] ? f - (f / 9) * 9 : 0;
    wt[e] = valid[e] ? gauss9(iy[e]) * gauss9(ix[e]) : 0.f;
  }
  auto drop = [&](float value) {
    for (int l = 0; l < p.L; ++l) empty_level(p, g, l, lane);
    finish_track(cam, i, value, value, value, value, lane);
  };
  const bool gfinite = isfinite(gout.x) && isfinite(gout.y);

  if (MODE == kLkImplicit) {
    const fe_track_data& tout = cam.tracks_out[i];
    if (!tout.track_status || !gfinite) return drop(0.f);
    // level-0 template position, through the forward's chain of level scalings
    const float scale = 1.f / (float)(1 << top);
    float sx = __fmaf_rn(__fsub_rn(tin.track[0], 0.5f), scale, 0.5f);
    float sy = __fmaf_rn(__fsub_rn(tin.track[1], 0.5f), scale, 0.5f);
    for (int l = top; l > 0; --l) {
      sx = __fmaf_rn(sx, 2.f, -0.5f);
      sy = __fmaf_rn(sy, 2.f, -0.5f);
    }
    const float cx = tout.track[0], cy = tout.track[1];
    const Level& PL = cam.lk.prev.lv[0];
    const Level& CL = cam.lk.cur.lv[0];
    const int W = CL.w, H = CL.h;
    Templ T;
    int wbx = INT_MIN / 2, wby = INT_MIN / 2;
    make_template(PL, sx, sy, valid, ix, iy, wt, sm, lane, T, &CL, make_float2(cx, cy), &wbx, &wby);
    const TapSet tc = cur_taps(CL, cx, cy, wbx, wby, sm, lane);
    float p2[kNE], dx[kNE], dy[kNE];
    float sc = 0.f, sdx = 0.f, sdy = 0.f;
#pragma unroll
    for (int e = 0; e < kNE; ++e) {
      p2[e] = dx[e] = dy[e] = 0.f;
      const Tap t = tap_of<FE_SAMPLE_EXACT>(tc, ix[e], iy[e], wbx, wby, kCAS);
      if (valid[e]) {
        sample_vg(sm.win.cur, kCAS, t, p2[e], dx[e], dy[e]);
        sc = __fadd_rn(sc, p2[e]);
        sdx = __fadd_rn(sdx, dx[e]);
        sdy = __fadd_rn(sdy, dy[e]);
      }
    }
    warp_sum3(sc, sdx, sdy, lane);
    const float mdx = __fmul_rn(sdx, rcp81), mdy = __fmul_rn(sdy, rcp81);
    const float delta = __fmul_rn(__fsub_rn(sc, T.sp), rcp81);
    float r[kNE], j00 = 0.f, j01 = 0.f, j10 = 0.f, j11 = 0.f;
#pragma unroll
    for (int e = 0; e < kNE; ++e) {
      r[e] = 0.f;
      if (valid[e]) {
        r[e] = __fsub_rn(__fsub_rn(p2[e], T.p1[e]), delta);
        const float wa = __fmul_rn(wt[e], T.a[e]), wb = __fmul_rn(wt[e], T.b[e]);
        const float ddx = __fsub_rn(dx[e], mdx), ddy = __fsub_rn(dy[e], mdy);
        j00 = __fmaf_rn(wa, ddx, j00);
        j01 = __fmaf_rn(wa, ddy, j01);
        j10 = __fmaf_rn(wb, ddx, j10);
        j11 = __fmaf_rn(wb, ddy, j11);
      }
    }
    warp_sum2(j00, j01, lane);
    warp_sum2(j10, j11, lane);
    const float detj = __fmaf_rn(j00, j11, -__fmul_rn(j01, j10));
    if (!(fabsf(detj) > 0.f) || !isfinite(detj)) return drop(0.f);
    // J^T lambda = dL/dc*
    const float lx = __fdiv_rn(__fmaf_rn(j11, gout.x, -__fmul_rn(j10, gout.y)), detj);
    const float ly = __fdiv_rn(__fmaf_rn(j00, gout.y, -__fmul_rn(j01, gout.x)), detj);
    float u[kNE], ab[kNE], bb[kNE];
    float su = 0.f, sa = 0.f, sb = 0.f;
#pragma unroll
    for (int e = 0; e < kNE; ++e) {
      u[e] = ab[e] = bb[e] = 0.f;
      if (valid[e]) {
        u[e] = -__fmul_rn(wt[e], __fmaf_rn(lx, T.a[e], __fmul_rn(ly, T.b[e])));
        const float wr = __fmul_rn(wt[e], r[e]);
        ab[e] = -__fmul_rn(wr, lx);
        bb[e] = -__fmul_rn(wr, ly);
        su = __fadd_rn(su, u[e]);
        sa = __fadd_rn(sa, ab[e]);
        sb = __fadd_rn(sb, bb[e]);
      }
    }
    warp_sum3(su, sa, sb, lane);
    const float mu = __fmul_rn(su, rcp81);
    const float ma = __fmul_rn(sa, rcp81), mb = __fmul_rn(sb, rcp81);
    float p2b[kNE], p1b[kNE], gxb[kNE], gyb[kNE];
#pragma unroll
    for (int e = 0; e < kNE; ++e) {
      p2b[e] = valid[e] ? __fsub_rn(u[e], mu) : 0.f;
      p1b[e] = -p2b[e];
      gxb[e] = valid[e] ? __fsub_rn(ab[e], ma) : 0.f;
      gyb[e] = valid[e] ? __fsub_rn(bb[e], mb) : 0.f;
    }
    // current-image record at c*
    {
      const int rx0 = max(patch_base(cx) - 1, 0), ry0 = max(patch_base(cy) - 1, 0);
      const int rs = p.cur_s;
      zero_smem(sm.acc, rs * rs, lane);
      float* const dst[1] = {sm.acc};
      const float c1[1][kNE] = {{p2b[0], p2b[1], p2b[2]}};
      scatter_taps<1>(dst, rs, rx0, ry0, tc, c1, valid, ix, iy, W, H, sm, lane);
      const int rw = min(rs, W - rx0), rh = min(rs, H - ry0);
      const size_t slot = (size_t)g;  // level 0
      store_record(p.data_cur + slot * (rs * rs), rs, sm.acc, rs, rw, rh, lane);
      if (lane == 0) p.hdr[(size_t)3 * p.L * p.total + slot] = make_int4(rx0, ry0, rw, rh);
    }
    float dsx, dsy;
    finish_template(p, g, 0, W, H, T, p1b, gxb, gyb, valid, ix, iy, sm, lane, dsx, dsy);
    for (int l = 1; l < p.L; ++l) empty_level(p, g, l, lane);
    finish_track(cam, i, dsx, dsy, 0.f, 0.f, lane);
    return;
  }

  // ---- unrolled: the forward's record of every level (p.recs, global memory; uniform loads)
  const LkRecord& R = p.recs[g];
  if (R.flags[0] != 3 || !gfinite) return drop(0.f);  // level 0 accepted <=> the track is tracked
  // current-image record boxes of the accepted levels must fit cur_s x cur_s: taps of a patch reach
  // texels [base, base + 10]; the record starts one texel left of the smallest base
  for (int level = 0; level <= top; ++level) {
    if (R.flags[level] != 3) continue;
    const int K = R.K[level];
    int lox = INT_MAX, hix = INT_MIN, loy = INT_MAX, hiy = INT_MIN;
    for (int t = 0; t < K; ++t) {
      const float2 c = R.it[level][t];
      lox = min(lox, patch_base(c.x));
      hix = max(hix, patch_base(c.x));
      loy = min(loy, patch_base(c.y));
      hiy = max(hiy, patch_base(c.y));
    }
    if (hix - lox + 12 > p.cur_s || hiy - loy + 12 > p.cur_s) {
      if (lane == 0) atomicAdd(p.overflow, 1);
      return drop(__int_as_float(0x7fc00000));  // NaN: no gradient for this track
    }
  }
  float cbx = gout.x, cby = gout.y;  // dL/d(end position of the level)
  float gtx = 0.f, gty = 0.f;
  for (int level = 0; level <= top; ++level) {
    if (R.flags[level] == 3) {
      const Level& PL = cam.lk.prev.lv[level];
      const Level& CL = cam.lk.cur.lv[level];
      const int W = CL.w, H = CL.h;
      const float2 s = R.s[level];
      Templ T;
      const int K = R.K[level];
      int wbx = INT_MIN / 2, wby = INT_MIN / 2;  // current-image window (the first step replayed, t = K - 1)
      make_template(PL, s.x, s.y, valid, ix, iy, wt, sm, lane, T, K > 0 ? &CL : nullptr,
                    K > 0 ? R.it[level][K - 1] : make_float2(0.f, 0.f), &wbx, &wby);
      int lox = INT_MAX, loy = INT_MAX, hix = INT_MIN, hiy = INT_MIN;
      for (int t = 0; t < K; ++t) {
        const int bx = patch_base(R.it[level][t].x), by = patch_base(R.it[level][t].y);
        lox = min(lox, bx);
        loy = min(loy, by);
        hix = max(hix, bx);
        hiy = max(hiy, by);
      }
      // the record spans the iterates' taps: texels [lo - 1, hi + 10] clipped to the level
      const int rs = p.cur_s;
      const int rx0 = max(lox - 1, 0), ry0 = max(loy - 1, 0);
      const int rw = min(hix + 10, W - 1) - rx0 + 1, rh = min(hiy + 10, H - 1) - ry0 + 1;
      for (int k = lane; k < rw * rh; k += 32) sm.acc[(k / rw) * rs + k % rw] = 0.f;
      __syncwarp();
      float p1b[kNE], ab[kNE], bb[kNE];
      // per tap and bilinear corner, dL/dP2 weighted by the corner's weight, summed over the steps
      // that share one uniform, unclamped tap base (pbx, pby); added to the record when the base
      // changes and at the end of the level
      float cs[kNE][4];
#pragma unroll
      for (int e = 0; e < kNE; ++e) {
        p1b[e] = ab[e] = bb[e] = 0.f;
        cs[e][0] = cs[e][1] = cs[e][2] = cs[e][3] = 0.f;
      }
      int pbx = INT_MIN, pby = INT_MIN;
      bool pending = false;
      auto flush = [&]() {
#pragma unroll
        for (int corner = 0; corner < 4; ++corner) {
          const int ox = corner & 1, oy = corner >> 1;
#pragma unroll
          for (int e = 0; e < kNE; ++e) {
            if (valid[e]) {
              const int o = (pby + iy[e] + oy - ry0) * rs + (pbx + ix[e] + ox - rx0);
              sm.acc[o] = __fadd_rn(sm.acc[o], cs[e][corner]);
            }
            cs[e][corner] = 0.f;
          }
          __syncwarp();
        }
        pending = false;
      };
      float hxx = 0.f, hxy = 0.f, hyx = 0.f, hyy = 0.f;
      for (int t = K - 1; t >= 0; --t) {
        const float2 c = R.it[level][t];
        const float2 v = R.v[level][t];
        const float delta = R.delta[level][t];
        const TapSet tc = cur_taps(CL, c.x, c.y, wbx, wby, sm, lane);
        float p2[kNE], dx[kNE], dy[kNE];
#pragma unroll
        for (int e = 0; e < kNE; ++e) {
          p2[e] = dx[e] = dy[e] = 0.f;
          const Tap tp = tap_of<FE_SAMPLE_EXACT>(tc, ix[e], iy[e], wbx, wby, kCAS);
          if (valid[e]) sample_vg(sm.win.cur, kCAS, tp, p2[e], dx[e], dy[e]);
        }
        // v = H^-1 e is recorded; mu = H^-1 cbar, Hbar -= mu v^T
        const float mux = __fmul_rn(__fmaf_rn(T.gyy, cbx, -__fmul_rn(T.gxy, cby)), T.det_rcp);
        const float muy = __fmul_rn(__fmaf_rn(T.gxx, cby, -__fmul_rn(T.gxy, cbx)), T.det_rcp);
        hxx = __fmaf_rn(-mux, v.x, hxx);
        hxy = __fmaf_rn(-mux, v.y, hxy);
        hyx = __fmaf_rn(-muy, v.x, hyx);
        hyy = __fmaf_rn(-muy, v.y, hyy);
        float u[kNE], su = 0.f;
#pragma unroll
        for (int e = 0; e < kNE; ++e) {
          u[e] = 0.f;
          if (valid[e]) {
            u[e] = __fmul_rn(wt[e], __fmaf_rn(mux, T.a[e], __fmul_rn(muy, T.b[e])));
            su = __fadd_rn(su, u[e]);
          }
        }
        const float mu = __fmul_rn(warp_sum(su), rcp81);
        float p2b[kNE], gx = 0.f, gy = 0.f;
#pragma unroll
        for (int e = 0; e < kNE; ++e) {
          p2b[e] = 0.f;
          if (valid[e]) {
            p2b[e] = __fsub_rn(u[e], mu);
            gx = __fmaf_rn(p2b[e], dx[e], gx);
            gy = __fmaf_rn(p2b[e], dy[e], gy);
            p1b[e] = __fsub_rn(p1b[e], p2b[e]);
            const float wr = __fmul_rn(wt[e], __fsub_rn(__fsub_rn(p2[e], T.p1[e]), delta));
            ab[e] = __fmaf_rn(wr, mux, ab[e]);
            bb[e] = __fmaf_rn(wr, muy, bb[e]);
          }
        }
        const int b0x = __shfl_sync(kFull, tc.base, 0), b0y = __shfl_sync(kFull, tc.base, 16);
        const bool fast = tc.uniform && b0x >= 0 && b0y >= 0 && b0x + 9 <= W - 1 && b0y + 9 <= H - 1;
        if (pending && !(fast && b0x == pbx && b0y == pby)) flush();
        if (fast) {
          const float fx = tc.u.w00, fy = tc.u.w10;
          const float qx = __fsub_rn(1.f, fx), qy = __fsub_rn(1.f, fy);
          const float wc[4] = {__fmul_rn(qx, qy), __fmul_rn(fx, qy), __fmul_rn(qx, fy), __fmul_rn(fx, fy)};
#pragma unroll
          for (int e = 0; e < kNE; ++e)
#pragma unroll
            for (int corner = 0; corner < 4; ++corner) cs[e][corner] = __fmaf_rn(wc[corner], p2b[e], cs[e][corner]);
          pbx = b0x;
          pby = b0y;
          pending = true;
        } else {
          float* const dst[1] = {sm.acc};
          const float c1[1][kNE] = {{p2b[0], p2b[1], p2b[2]}};
          scatter_taps<1>(dst, rs, rx0, ry0, tc, c1, valid, ix, iy, W, H, sm, lane);
        }
        warp_sum2(gx, gy, lane);
        cbx = __fadd_rn(cbx, gx);
        cby = __fadd_rn(cby, gy);
      }
      if (pending) flush();
      const float hs = __fadd_rn(hxy, hyx);
      float sa = 0.f, sb = 0.f;
#pragma unroll
      for (int e = 0; e < kNE; ++e) {
        if (valid[e]) {
          ab[e] = __fmaf_rn(wt[e], __fmaf_rn(2.f * hxx, T.a[e], __fmul_rn(hs, T.b[e])), ab[e]);
          bb[e] = __fmaf_rn(wt[e], __fmaf_rn(hs, T.a[e], __fmul_rn(2.f * hyy, T.b[e])), bb[e]);
          sa = __fadd_rn(sa, ab[e]);
          sb = __fadd_rn(sb, bb[e]);
        }
      }
      warp_sum2(sa, sb, lane);
      const float ma = __fmul_rn(sa, rcp81), mb = __fmul_rn(sb, rcp81);
      float gxb[kNE], gyb[kNE];
#pragma unroll
      for (int e = 0; e < kNE; ++e) {
        gxb[e] = valid[e] ? __fsub_rn(ab[e], ma) : 0.f;
        gyb[e] = valid[e] ? __fsub_rn(bb[e], mb) : 0.f;
      }
      // current-image record of the level
      {
        const size_t slot = (size_t)level * p.total + g;
        store_record(p.data_cur + slot * (rs * rs), rs, sm.acc, rs, rw, rh, lane);
        if (lane == 0) p.hdr[(size_t)3 * p.L * p.total + slot] = make_int4(rx0, ry0, rw, rh);
      }
      float dsx, dsy;
      finish_template(p, g, level, W, H, T, p1b, gxb, gyb, valid, ix, iy, sm, lane, dsx, dsy);
      const float sl = 1.f / (float)(1 << level);
      gtx = __fmaf_rn(dsx, sl, gtx);
      gty = __fmaf_rn(dsy, sl, gty);
    } else {
      empty_level(p, g, level, lane);
    }
    if (level < top) {
      cbx = __fmul_rn(cbx, 2.f);
      cby = __fmul_rn(cby, 2.f);
    }
  }
  for (int l = levels; l < p.L; ++l) empty_level(p, g, l, lane);
  const float st = 1.f / (float)(1 << top);
  finish_track(cam, i, __fmaf_rn(cbx, st, gtx), __fmaf_rn(cby, st, gty), __fmul_rn(cbx, st), __fmul_rn(cby, st),
               lane);
}

template <int MODE>
__global__ void __launch_bounds__(kAdjWarps * 32, MODE == kLkImplicit ? 5 : 4) adjoint_kernel(const __grid_constant__ AdjLaunch p) {
  __shared__ AdjSmem smem[kAdjWarps];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (;;) {
    int v = 0;
    if (lane == 0) v = atomicAdd(p.counter, 1);
    const int g = __shfl_sync(kFull, v, 0);
    if (g >= p.total) return;  // warp-uniform
    int lo = 0, hi = p.ncams - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (p.cams[mid].lk.begin <= g) lo = mid; else hi = mid - 1;
    }
    adjoint_one<MODE>(p, p.cams[lo], g, smem[wid], lane);
  }
}

template <int MODE>
int adjoint_blocks() {
  // blocks resident on the device, found once per process
  static const int blocks = [] {
    int per_sm = 0, dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, adjoint_kernel<MODE>, kAdjWarps * 32, 0);
    return (per_sm > 0 ? per_sm : 1) * (sms > 0 ? sms : 1);
  }();
  return blocks;
}

// ---------------------------------------------------------------- tile-segmented reduction
__device__ __forceinline__ int slot_camera(const AdjGather& G, int g) {
  int lo = 0, hi = G.ncams - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (G.cams[mid].lk.begin <= g) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Visits the tiles a record covers: count (FILL = false) or list fill (FILL = true).
template <bool FILL>
__global__ void bin_kernel(const __grid_constant__ AdjGather G) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= G.nslots) return;
  const int4 h = G.hdr[s];
  if (h.z <= 0 || h.w <= 0) return;
  const int per_q = G.L * G.total;
  const int q = s / per_q, rem = s - q * per_q;
  const int l = rem / G.total, g = rem - l * G.total;
  const AdjPlane& P = G.planes[(slot_camera(G, g) * 4 + q) * G.L + l];
  if (P.ntiles <= 0) return;
  const int tiles_y = P.ntiles / P.tiles_x;
  const int tx0 = h.x / kTile, tx1 = min((h.x + h.z - 1) / kTile, P.tiles_x - 1);
  const int ty0 = h.y / kTile, ty1 = min((h.y + h.w - 1) / kTile, tiles_y - 1);
  for (int ty = ty0; ty <= ty1; ++ty)
    for (int tx = tx0; tx <= tx1; ++tx) {
      const int t = P.tile_begin + ty * P.tiles_x + tx;
      if (FILL) G.list[G.off[t] + atomicAdd(&G.cursor[t], 1)] = s;
      else atomicAdd(&G.count[t], 1);
    }
}

// Exclusive prefix sum of the per-tile counts (one CTA, four tiles per thread per pass); clears the
// fill cursors and lists the tiles with more than kWarpList records.
__global__ void __launch_bounds__(1024) scan_kernel(const __grid_constant__ AdjGather G) {
  __shared__ int warp_tot[32];
  __shared__ int carry;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  if (tid == 0) {
    carry = 0;
    *G.long_count = 0;
  }
  __syncthreads();
  for (int base = 0; base < G.total_tiles; base += 4096) {
    const int t0 = base + 4 * tid;
    int v[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      v[k] = t0 + k < G.total_tiles ? G.count[t0 + k] : 0;
      if (v[k] > kWarpList) G.long_tiles[atomicAdd(G.long_count, 1)] = t0 + k;  // processing order is free
    }
    const int mine = v[0] + v[1] + v[2] + v[3];
    int x = mine;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, d);
      if (lane >= d) x += y;
    }
    if (lane == 31) warp_tot[wid] = x;
    __syncthreads();
    if (wid == 0) {
      int w = warp_tot[lane];
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, w, d);
        if (lane >= d) w += y;
      }
      warp_tot[lane] = w;  // inclusive
    }
    __syncthreads();
    int before = carry + (wid > 0 ? warp_tot[wid - 1] : 0) + x - mine;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (t0 + k < G.total_tiles) {
        G.off[t0 + k] = before;
        G.cursor[t0 + k] = 0;
      }
      before += v[k];
    }
    __syncthreads();
    if (tid == 0) carry += warp_tot[31];
    __syncthreads();
  }
  if (tid == 0) G.off[G.total_tiles] = carry;
}

__device__ __forceinline__ const float* record_data(const AdjGather& G, int s, int& S) {
  const int per_q = G.L * G.total;
  if (s < 3 * per_q) {
    S = kRP;
    return G.data_prev + (size_t)s * (kRP * kRP);
  }
  S = G.cur_s;
  return G.data_cur + (size_t)(s - 3 * per_q) * (G.cur_s * G.cur_s);
}

__device__ __forceinline__ const AdjPlane& tile_plane(const AdjGather& G, int t) {
  // the last plane that begins at or before t (an empty plane shares its begin with the next one)
  int lo = 0, hi = G.nplanes - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (G.planes[mid].tile_begin <= t) lo = mid; else hi = mid - 1;
  }
  return G.planes[lo];
}

// One warp adds records to its 32x32 tile at (X0, Y0): lane = column X0 + lane, acc[r] = row Y0 + r.
// `key` is this lane's record slot (lanes 0..m-1 hold m records, in the order they are added).
__device__ __forceinline__ void warp_add_records(const AdjGather& G, int key, int m, int X0, int Y0, float (&acc)[kTile],
                                                 int lane) {
  const int4 mine = lane < m ? G.hdr[key] : make_int4(0, 0, 0, 0);
  const int X = X0 + lane;
  if (lane < m) {
    // every record of the group is requested into L2 up front (lane r: record r's rows inside the
    // tile), so that the in-order adds below wait on L2 rather than on DRAM
    int S;
    const float* d = record_data(G, key, S) + max(0, X0 - mine.x);
    const int r1 = min(mine.w, Y0 + kTile - mine.y);
    for (int row = max(0, Y0 - mine.y); row < r1; ++row)
      asm volatile("prefetch.global.L2 [%0];" ::"l"(d + (size_t)row * S));
  }
  for (int r = 0; r < m; ++r) {
    const int k = __shfl_sync(kFull, key, r);
    const int hx = __shfl_sync(kFull, mine.x, r), hy = __shfl_sync(kFull, mine.y, r);
    const int hz = __shfl_sync(kFull, mine.z, r), hw = __shfl_sync(kFull, mine.w, r);
    if (X < hx || X >= hx + hz || hy >= Y0 + kTile || hy + hw <= Y0) continue;
    int S;
    const float* d = record_data(G, k, S) + (X - hx);
#pragma unroll
    for (int row = 0; row < kTile; ++row) {
      const int dy = Y0 + row - hy;
      if (dy >= 0 && dy < hw) acc[row] += d[dy * S];
    }
  }
}

// Ascending sort of one key per lane across the warp (bitonic network on shuffles).
__device__ __forceinline__ int warp_sort(int key, int lane) {
#pragma unroll
  for (int size = 2; size <= 32; size <<= 1) {
#pragma unroll
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      const int other = __shfl_xor_sync(kFull, key, stride);
      const bool up = (lane & size) == 0 || size == 32;
      const bool lower = (lane & stride) == 0;
      key = (lower == up) ? min(key, other) : max(key, other);
    }
  }
  return key;
}

// Tiles with at most kWarpList records (nearly all): one warp per tile, 8 tiles per CTA; the warp
// sorts the slots (track order) and adds the records in that order into its registers.
__global__ void __launch_bounds__(kGatherThreads) gather_warp_kernel(const __grid_constant__ AdjGather G) {
  const int lane = threadIdx.x & 31;
  const int t = blockIdx.x * kGatherWarps + (threadIdx.x >> 5);
  if (t >= G.total_tiles) return;  // warp-uniform
  const int begin = G.off[t], n = G.off[t + 1] - begin;
  if (n > kWarpList) return;       // gather_long_kernel
  const AdjPlane& P = tile_plane(G, t);
  const int lt = t - P.tile_begin;
  const int X0 = (lt % P.tiles_x) * kTile, Y0 = (lt / P.tiles_x) * kTile;
  const int key = warp_sort(lane < n ? G.list[begin + lane] : INT_MAX, lane);
  float acc[kTile];
#pragma unroll
  for (int r = 0; r < kTile; ++r) acc[r] = 0.f;
  warp_add_records(G, key, n, X0, Y0, acc, lane);
  const int X = X0 + lane;
  if (X < P.w) {
#pragma unroll
    for (int r = 0; r < kTile; ++r)
      if (Y0 + r < P.h) P.dst[(size_t)(Y0 + r) * P.pitch + X] = acc[r];
  }
}

// Tiles with more than kWarpList records (coarse levels), from the scan's list: a CTA orders the
// tile's slots by track, warp k of 32 adds the k-th contiguous part of the sorted list (32 records at a time)
// into its registers, and the 32 partial tiles are summed in warp order.  Each record costs its warp
// one memory round trip, so the records of a tile are spread over as many warps as one CTA holds.
__global__ void __launch_bounds__(kLongThreads, 1) gather_long_kernel(const __grid_constant__ AdjGather G) {
  extern __shared__ __align__(16) unsigned char gsm[];
  float* part = reinterpret_cast<float*>(gsm);                                // [kLongWarps][1024]
  int* keys = reinterpret_cast<int*>(gsm + kLongWarps * kTile * kTile * 4);  // [list_cap]
  const int nwords = (G.list_cap + 31) >> 5;                                  // bitmap words (<= 1024)
  uint32_t* bits = reinterpret_cast<uint32_t*>(keys + G.list_cap);            // [nwords]
  int* prefix = reinterpret_cast<int*>(bits + nwords);                        // [nwords]
  __shared__ int wsum[32];
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int nlong = *G.long_count;
  for (int li = blockIdx.x; li < nlong; li += gridDim.x) {
    const int t = G.long_tiles[li];
    const AdjPlane& P = tile_plane(G, t);
    const int lt = t - P.tile_begin;
    const int X0 = (lt % P.tiles_x) * kTile, Y0 = (lt / P.tiles_x) * kTile;
    const int begin = G.off[t], n = min(G.off[t + 1] - begin, G.list_cap);
    // the tile's records in track order without a comparison sort: a tile belongs to one plane of
    // one camera, so each record is a distinct track of that camera; mark the tracks in a bitmap,
    // then a record's rank is the number of marked tracks before it
    const int pi = (int)(&P - G.planes);
    const int cbegin = G.cams[pi / (4 * G.L)].lk.begin;
    __syncthreads();  // the previous tile's readers of keys, bitmap and part are done
    for (int k = tid; k < nwords; k += kLongThreads) bits[k] = 0u;
    __syncthreads();
    for (int k = tid; k < n; k += kLongThreads) {
      const int rel = G.list[begin + k] % G.total - cbegin;
      atomicOr(&bits[rel >> 5], 1u << (rel & 31));
    }
    __syncthreads();
    // exclusive prefix of the words' population counts (nwords <= kLongThreads)
    {
      const int c = tid < nwords ? __popc(bits[tid]) : 0;
      int x = c;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const int y = __shfl_up_sync(kFull, x, d);
        if (lane >= d) x += y;
      }
      if (lane == 31) wsum[wid] = x;
      __syncthreads();
      if (wid == 0) {
        int w = wsum[lane];
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
          const int y = __shfl_up_sync(kFull, w, d);
          if (lane >= d) w += y;
        }
        wsum[lane] = w;
      }
      __syncthreads();
      if (tid < nwords) prefix[tid] = (wid > 0 ? wsum[wid - 1] : 0) + x - c;
    }
    __syncthreads();
    for (int k = tid; k < n; k += kLongThreads) {
      const int key = G.list[begin + k];
      const int rel = key % G.total - cbegin;
      keys[prefix[rel >> 5] + __popc(bits[rel >> 5] & ((1u << (rel & 31)) - 1u))] = key;
    }
    __syncthreads();
    float acc[kTile];
#pragma unroll
    for (int r = 0; r < kTile; ++r) acc[r] = 0.f;
    const int r0 = (int)((long long)n * wid / kLongWarps), r1 = (int)((long long)n * (wid + 1) / kLongWarps);
    for (int g0 = r0; g0 < r1; g0 += 32) {
      const int m = min(32, r1 - g0);
      warp_add_records(G, lane < m ? keys[g0 + lane] : 0, m, X0, Y0, acc, lane);
    }
#pragma unroll
    for (int r = 0; r < kTile; ++r) part[wid * kTile * kTile + r * kTile + lane] = acc[r];
    __syncthreads();
    for (int k = tid; k < kTile * kTile; k += kLongThreads) {
      const int X = X0 + (k & (kTile - 1)), Y = Y0 + k / kTile;
      if (X < P.w && Y < P.h) {
        float v = part[k];
        for (int w = 1; w < kLongWarps; ++w) v += part[w * kTile * kTile + k];
        P.dst[(size_t)Y * P.pitch + X] = v;
      }
    }
  }
}

// ---------------------------------------------------------------- pyramid adjoint
__device__ __forceinline__ float binom5(int k) {
  return k == 2 ? 6.f / 16.f : (k == 1 || k == 3) ? 4.f / 16.f : 1.f / 16.f;
}

// Complete gradient of pixel (x, y) of one level: the summed records, the transposed 7-tap
// derivatives of the gradient planes' adjoints (previous frame only) and the transposed 5x5
// decimation of the next level's complete gradient.  Taps are added in a fixed order: derivative
// taps j = 0..6 along x, then along y, then the decimation's rows and columns in ascending order.
__device__ float adjoint_pixel(const AdjPyrJob& J, int x, int y) {
  float v = J.img[(size_t)y * J.pitch + x];
  if (J.gx) {
    // transposed 7-tap derivatives: gx(x') = sum_j D_j img(x' - 3 + j) for 2 < x' < w - 3
#pragma unroll
    for (int j = 0; j < 7; ++j) {
      const int xp = x - j + 3;
      if (xp > 2 && xp < J.w - 3) v = __fmaf_rn(dsp_tap(j), J.gx[(size_t)y * J.gpitch + xp], v);
    }
#pragma unroll
    for (int j = 0; j < 7; ++j) {
      const int yp = y - j + 3;
      if (yp > 2 && yp < J.h - 3) v = __fmaf_rn(dsp_tap(j), J.gy[(size_t)yp * J.gpitch + x], v);
    }
  }
  if (J.up && x >= 2 && x <= J.w - 3 && y >= 2 && y <= J.h - 3) {
    // interior: only unmirrored sources, 2X - 2 + k == x with k of x's parity (2 or 3 per axis)
    for (int ky = y & 1; ky < 5; ky += 2) {
      const int Y = (y + 2 - ky) >> 1;
      if (Y >= J.up_h) continue;
      const float* row = J.up + (size_t)Y * J.up_pitch;
      const float wy = binom5(ky);
      for (int kx = x & 1; kx < 5; kx += 2) {
        const int X = (x + 2 - kx) >> 1;
        if (X >= J.up_w) continue;
        v = __fmaf_rn(__fmul_rn(wy, binom5(kx)), row[X], v);
      }
    }
  } else if (J.up) {
    // transposed decimation: the outputs (X, Y) of the next level whose 5x5 taps read (x, y), either
    // directly (unmirrored source coordinate 2X - 2 + k == x) or through the mirror (-x-1 below 0,
    // 2n-x-1 above n-1); taps outside in both directions are skipped as the forward skips them
    for (int a = 0; a < 3; ++a) {
      const int yc = a == 0 ? y : a == 1 ? (y <= 1 ? -y - 1 : INT_MIN) : (y >= J.h - 2 ? 2 * J.h - y - 1 : INT_MIN);
      if (yc == INT_MIN) continue;
      const bool yo = yc < 0 || yc >= J.h;
      for (int ky = 0; ky < 5; ++ky) {
        const int vy = yc + 2 - ky;
        if (vy & 1) continue;
        const int Y = vy / 2;
        if (Y < 0 || Y >= J.up_h) continue;
        const float* row = J.up + (size_t)Y * J.up_pitch;
        for (int b = 0; b < 3; ++b) {
          const int xc = b == 0 ? x : b == 1 ? (x <= 1 ? -x - 1 : INT_MIN) : (x >= J.w - 2 ? 2 * J.w - x - 1 : INT_MIN);
          if (xc == INT_MIN) continue;
          const bool xo = xc < 0 || xc >= J.w;
          if (xo && yo) continue;
          for (int kx = 0; kx < 5; ++kx) {
            const int vx = xc + 2 - kx;
            if (vx & 1) continue;
            const int X = vx / 2;
            if (X < 0 || X >= J.up_w) continue;
            v = __fmaf_rn(__fmul_rn(binom5(ky), binom5(kx)), row[X], v);
          }
        }
      }
    }
  }
  return v;
}

__device__ __forceinline__ void load4(const float* p, float* out) {
  const float4 q = *reinterpret_cast<const float4*>(p);
  out[0] = q.x;
  out[1] = q.y;
  out[2] = q.z;
  out[3] = q.w;
}

// One launch per level; blockIdx.y = job (one pyramid of one camera).  A thread takes four pixels
// x .. x+3 (x a multiple of 4) of a row, 128x8-pixel blocks.  Away from the borders, with 16-byte
// aligned planes, the taps come from 16-byte loads: the gradient row x-4 .. x+7, seven gradient
// rows at x .. x+3, and two or three rows of the next level's gradient from the 4-aligned column at
// or below x/2 - 1; every pixel adds the same taps in the same order as adjoint_pixel.  Elsewhere
// each pixel runs adjoint_pixel.
__global__ void __launch_bounds__(256) pyramid_adjoint_kernel(const __grid_constant__ AdjPyrLevel L) {
  const AdjPyrJob& J = L.job[blockIdx.y];
  const int bx = (J.w + 127) >> 7;
  const int x = ((int)(blockIdx.x % bx) * 32 + (threadIdx.x & 31)) * 4;
  const int y = (int)(blockIdx.x / bx) * 8 + (threadIdx.x >> 5);
  if (x >= J.w || y >= J.h) return;
  const bool aligned = ((reinterpret_cast<uintptr_t>(J.img) | reinterpret_cast<uintptr_t>(J.gx) |
                         reinterpret_cast<uintptr_t>(J.gy) | reinterpret_cast<uintptr_t>(J.up)) & 15) == 0 &&
                       ((J.pitch | J.gpitch | J.up_pitch) & 3) == 0;
  const int ub = (x >> 1) - 1 >= 0 ? (((x >> 1) - 1) & ~3) : 0;  // first next-level column loaded
  const bool fast = aligned && x >= 8 && x + 10 <= J.w && y >= 6 && y + 7 <= J.h &&
                    (!J.up || (ub + 8 <= J.up_w && ((y + 2) >> 1) < J.up_h));
  if (!fast) {
    for (int i = 0; i < 4 && x + i < J.w; ++i) {
      const float v = adjoint_pixel(J, x + i, y);
      J.img[(size_t)y * J.pitch + x + i] = v;
    }
    return;
  }
  float v[4];
  load4(J.img + (size_t)y * J.pitch + x, v);
  if (J.gx) {
    // x' = x + i - j + 3 runs over x - 3 .. x + 6, all inside (2, w - 3): row values x - 4 .. x + 7
    float r[12];
    const float* gr = J.gx + (size_t)y * J.gpitch + x - 4;
    load4(gr, r);
    load4(gr + 4, r + 4);
    load4(gr + 8, r + 8);
#pragma unroll
    for (int j = 0; j < 7; ++j)
#pragma unroll
      for (int i = 0; i < 4; ++i) v[i] = __fmaf_rn(dsp_tap(j), r[i - j + 7], v[i]);
#pragma unroll
    for (int j = 0; j < 7; ++j) {
      float c[4];
      load4(J.gy + (size_t)(y - j + 3) * J.gpitch + x, c);
#pragma unroll
      for (int i = 0; i < 4; ++i) v[i] = __fmaf_rn(dsp_tap(j), c[i], v[i]);
    }
  }
  if (J.up) {
    // pixel x + i reads next-level columns (x + i + 2 - kx) / 2 for kx of its parity, rows likewise
    for (int ky = y & 1; ky < 5; ky += 2) {
      const int Y = (y + 2 - ky) >> 1;
      float u[8];
      const float* ur = J.up + (size_t)Y * J.up_pitch + ub;
      load4(ur, u);
      load4(ur + 4, u + 4);
      const float wy = binom5(ky);
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int kx = i & 1; kx < 5; kx += 2) v[i] = __fmaf_rn(__fmul_rn(wy, binom5(kx)), u[((x + i + 2 - kx) >> 1) - ub], v[i]);
    }
  }
  *reinterpret_cast<float4*>(J.img + (size_t)y * J.pitch + x) = make_float4(v[0], v[1], v[2], v[3]);
}

}  // namespace

int lk_max_unrolled() { return kMaxRecIt; }
size_t lk_record_bytes() { return sizeof(LkRecord); }

cudaError_t adjoint_init() {
  cudaError_t e = cudaFuncSetAttribute(gather_long_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       kLongWarps * kTile * kTile * 4 + kMaxSelectKeys * 4 + 8 * (kMaxSelectKeys / 32));
  return e;
}

cudaError_t launch_lk_adjoint(const AdjLaunch& a, cudaStream_t s) {
  if (a.total <= 0) return cudaSuccess;
  cudaError_t e = cudaMemsetAsync(a.counter, 0, sizeof(int), s);
  if (e != cudaSuccess) return e;
  const int want = (a.total + kAdjWarps - 1) / kAdjWarps;
  if (a.mode == kLkUnrolled) {
    adjoint_kernel<kLkUnrolled><<<min(want, adjoint_blocks<kLkUnrolled>()), kAdjWarps * 32, 0, s>>>(a);
  } else {
    adjoint_kernel<kLkImplicit><<<min(want, adjoint_blocks<kLkImplicit>()), kAdjWarps * 32, 0, s>>>(a);
  }
  return cudaGetLastError();
}

cudaError_t launch_adjoint_gather(const AdjGather& g, cudaStream_t s) {
  if (g.total_tiles <= 0) return cudaSuccess;
  cudaError_t e = cudaMemsetAsync(g.count, 0, sizeof(int) * g.total_tiles, s);
  if (e != cudaSuccess) return e;
  const int nb = (g.nslots + 255) / 256;
  if (nb > 0) bin_kernel<false><<<nb, 256, 0, s>>>(g);
  scan_kernel<<<1, 1024, 0, s>>>(g);
  if (nb > 0) bin_kernel<true><<<nb, 256, 0, s>>>(g);
  const size_t smem = kLongWarps * kTile * kTile * 4 + (size_t)g.list_cap * 4 + 8 * (size_t)((g.list_cap + 31) / 32);
  gather_warp_kernel<<<(g.total_tiles + kGatherWarps - 1) / kGatherWarps, kGatherThreads, 0, s>>>(g);
  static const int sms = [] {
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n > 0 ? n : 1;
  }();
  gather_long_kernel<<<sms, kLongThreads, smem, s>>>(g);
  return cudaGetLastError();
}

cudaError_t launch_pyramid_adjoint(const AdjPyrLevel& lv, cudaStream_t s) {
  if (lv.total_px <= 0) return cudaSuccess;
  pyramid_adjoint_kernel<<<dim3(lv.max_blocks, lv.njobs), 256, 0, s>>>(lv);
  return cudaGetLastError();
}

}  // namespace fe
