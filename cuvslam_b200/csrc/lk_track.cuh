// The per-track LK routine (one warp per track) shared by the tracker (lk.cu) and the replay
// inside its adjoint (lk_adjoint.cu).  Algorithm and evaluation order: lk_track_kernel /
// lk_track_horizontal_kernel (lk_tracker.cu:69-379, 381-665).
#pragma once

#include <climits>

#include "fe_internal.h"
#include "lk_common.cuh"

namespace fe {
namespace lk {

// Iteration rules: kModeRef is the reference tracker.  The differentiable tracker (exact sampling)
// adds kModeImplicit: after the reference rule has accepted level 0, up to `iters` Newton steps on
// e(c) = 0, stopping after the first with |step|^2 < tol2, so that the result sits at the fixed
// point whose implicit derivative the adjoint takes (a track fails when the refinement does not
// settle within `iters` steps, takes a step or drifts beyond 2 px, or ends where J is ill
// conditioned); and kModeUnrolled: exactly `iters` steps on
// every level (no early stop), the level accepted when the last |v| < 0.12 and the gates pass.
constexpr int kModeRef = 0, kModeImplicit = 1, kModeUnrolled = 2;

// `rec` (unrolled mode only, may be null) receives the per-level record the adjoint replays.
// `cnt` (may be null) counts the work done: [0] levels set up (previous patch and gradients sampled,
// Hessian formed), [1] Gauss-Newton steps (current patch sampled, update solved), [2] NCC
// evaluations.
template <int SAMPLING, bool HORIZ, int MODE>
__device__ void track_one(const LkCam& cam, fe_track_data& td, WarpSmem& sm, int lane, int iters, float tol2,
                          LkRecord* rec = nullptr, unsigned long long* cnt = nullptr) {
  if (MODE == kModeUnrolled && rec) {
    if (lane < kMaxLevels) rec->flags[lane] = 0;
    __syncwarp();
  }
  const float radius = td.search_radius_px;
  const float ncc_thr = td.ncc_threshold;
  if (radius < 0.f) {
    __syncwarp();
    if (lane == 0) td.track_status = 0;
    return;
  }
  const float tx = td.track[0], ty = td.track[1];
  const float cx0 = __fadd_rn(tx, td.offset[0]), cy0 = __fadd_rn(ty, td.offset[1]);
  __syncwarp();
  if (lane < 4) td.info[lane] = (lane == 0 || lane == 3) ? 1.f / 9.f : 0.f;

  const int levels = cam.prev.levels;
  const int top = levels - 1;
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
  int ix[kNE], iy[kNE];
  float wt[kNE];
  bool valid[kNE], nccm[kNE];
#pragma unroll
  for (int e = 0; e < kNE; ++e) {
    const int f = lane + 32 * e;
    valid[e] = f < 81;
    iy[e] = valid[e] ? f / 9 : 0;
    ix[e] = valid[e] ? f - (f / 9) * 9 : 0;
    nccm[e] = valid[e] && ix[e] >= 2 && ix[e] < 7 && iy[e] >= 2 && iy[e] < 7;
    wt[e] = valid[e] ? gauss9(iy[e]) * gauss9(ix[e]) : 0.f;
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
    if (MODE == kModeUnrolled && rec && lane == 0) {
      rec->s[level] = make_float2(sx, sy);
      rec->K[level] = 0;
      rec->flags[level] = 0;
    }
    if (good) {
      if (cnt && lane == 0) atomicAdd(cnt, 1ull);
      // previous-frame patch: image and gradients; the window [bx, bx + 12) is staged from the
      // 16-byte aligned column ax = bx rounded down to a multiple of 4
      const int bx = (int)floorf(__fsub_rn(xmin, 0.5f)) - 1, by = (int)floorf(__fsub_rn(ymin, 0.5f)) - 1;
      const int ax = bx & ~3;
      __syncwarp();
      if (HORIZ) {
        float* const wv[2] = {sm.img, sm.gx};
        const float* const iv[2] = {PL.img, PL.gx};
        stage_planes<kPW, kPA, kPAS, 2>(wv, iv, PL.pitch, PL.w, PL.h, ax, by, lane);
      } else {
        float* const wv[3] = {sm.img, sm.gx, sm.gy};
        const float* const iv[3] = {PL.img, PL.gx, PL.gy};
        stage_planes<kPW, kPA, kPAS, 3>(wv, iv, PL.pitch, PL.w, PL.h, ax, by, lane);
      }
      // the current frame's window for the first Gauss-Newton step (the origin gn_step would choose),
      // staged together with the previous frame's so that one wait covers both
      int wbx = INT_MIN / 2, wby = INT_MIN / 2;  // current-frame window origin (none yet)
      {
        const float cxm = __fadd_rn(cx, -4.f), cym = __fadd_rn(cy, -4.f);
        if (cxm >= 0.f && __fadd_rn(cx, 5.f) < (float)W && cym >= 0.f && __fadd_rn(cy, 5.f) < (float)H) {
          wbx = ((int)floorf(__fsub_rn(cxm, 0.5f)) - 3) & ~3;
          wby = (int)floorf(__fsub_rn(cym, 0.5f)) - 3;
          stage_aligned<kCW, kCA, kCAS>(sm.cur, CL.img, CL.pitch, CL.w, CL.h, wbx, wby, lane);
        }
      }
      cp_async_wait_all();
      __syncwarp();
      const TapSet ts = make_taps<SAMPLING, false>(xmin, ymin, ax, by, kPAS, lane);
      float gxp[kNE], gyp[kNE], p1[kNE];
      float sgx = 0.f, sgy = 0.f, sp = 0.f;
#pragma unroll
      for (int e = 0; e < kNE; ++e) {
        gxp[e] = gyp[e] = p1[e] = 0.f;
        const Tap t = tap_of<SAMPLING>(ts, ix[e], iy[e], ax, by, kPAS);
        if (valid[e]) {
          gxp[e] = sample<SAMPLING>(sm.gx, kPAS, t);
          if (!HORIZ) gyp[e] = sample<SAMPLING>(sm.gy, kPAS, t);
          p1[e] = sample<SAMPLING>(sm.img, kPAS, t);
          sgx = __fadd_rn(sgx, gxp[e]);
          if (!HORIZ) sgy = __fadd_rn(sgy, gyp[e]);
          sp = __fadd_rn(sp, p1[e]);
        }
      }
      if (HORIZ) warp_sum2(sgx, sp, lane);
      else warp_sum3(sgx, sgy, sp, lane);
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
      if (HORIZ) lxx = warp_sum(lxx);
      else warp_sum3(lxx, lxy, lyy, lane);
      const float gxx = lxx;
      const float gxy = HORIZ ? 0.f : lxy;
      const float gyy = HORIZ ? 0.f : lyy;
      float det_rcp;
      if (HORIZ) {
        if (gxx < 1.1920928955078125e-07f) {
          if (lane == 0) td.track_status = 0;
          return;
        }
        det_rcp = __frcp_rn(gxx);  // correctly rounded: equals __fdiv_rn(1.f, gxx)
      } else {
        const float det = __fmaf_rn(gxx, gyy, -__fmul_rn(gxy, gxy));
        if (det < 1.1920928955078125e-07f) {
          if (lane == 0) td.track_status = 0;
          return;
        }
        det_rcp = __frcp_rn(det);  // correctly rounded: equals __fdiv_rn(1.f, det)
      }
      if (MODE == kModeUnrolled && rec && lane == 0) rec->flags[level] = 1;
      const float savex = cx, savey = cy;
      float p2[kNE];
#pragma unroll
      for (int e = 0; e < kNE; ++e) p2[e] = 0.f;
      float last_delta = 0.f;
      // One Gauss-Newton step at (cx, cy): samples p2 and returns the update; false when the patch
      // leaves the level.
      auto gn_step = [&](float& vx, float& vy) -> bool {
        xmin = __fadd_rn(cx, -4.f);
        ymin = __fadd_rn(cy, -4.f);
        if (!(xmin >= 0.f && __fadd_rn(cx, 5.f) < (float)W && ymin >= 0.f && __fadd_rn(cy, 5.f) < (float)H)) return false;
        // taps reach texels [base0 - 1, base0 + 10]; keep the window (20 columns from the aligned
        // wbx, 16 rows from wby) while it covers them
        const int nbx = (int)floorf(__fsub_rn(xmin, 0.5f)) - 1, nby = (int)floorf(__fsub_rn(ymin, 0.5f)) - 1;
        if (nbx < wbx || nbx + kPW > wbx + 4 * kCA || nby < wby || nby + kPW > wby + kCW) {
          wbx = (nbx - 2) & ~3;
          wby = nby - 2;
          __syncwarp();
          stage_aligned<kCW, kCA, kCAS>(sm.cur, CL.img, CL.pitch, CL.w, CL.h, wbx, wby, lane);
          cp_async_wait_all();
          __syncwarp();
        }
        const TapSet tc = make_taps<SAMPLING, false>(xmin, ymin, wbx, wby, kCAS, lane);
        float sc = 0.f;
#pragma unroll
        for (int e = 0; e < kNE; ++e) {
          const Tap t = tap_of<SAMPLING>(tc, ix[e], iy[e], wbx, wby, kCAS);
          if (valid[e]) {
            p2[e] = sample<SAMPLING>(sm.cur, kCAS, t);
            sc = __fadd_rn(sc, p2[e]);
          }
        }
        sc = warp_sum(sc);
        const float delta = __fmul_rn(__fsub_rn(sc, sp), rcp81);
        last_delta = delta;
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
        if (HORIZ) {
          ex = warp_sum(ex);
          vx = __fmul_rn(ex, det_rcp);
          vy = 0.f;
        } else {
          warp_sum2(ex, ey, lane);
          vx = __fmul_rn(__fmaf_rn(gyy, ex, -__fmul_rn(gxy, ey)), det_rcp);
          vy = __fmul_rn(__fmaf_rn(gxx, ey, -__fmul_rn(gxy, ex)), det_rcp);
        }
        return true;
      };
      const int max_it = MODE == kModeUnrolled ? iters : 11;
      int steps = 0;
      for (int it = 0; it < max_it; ++it) {
        if (MODE == kModeUnrolled && rec && lane == 0) rec->it[level][it] = make_float2(cx, cy);
        float vx, vy;
        if (!gn_step(vx, vy)) {
          good = false;
          break;
        }
        if (cnt && lane == 0) atomicAdd(cnt + 1, 1ull);
        conv = HORIZ ? fabsf(vx) < 0.12f : __fmaf_rn(vx, vx, __fmul_rn(vy, vy)) < thr2;
        if (MODE != kModeUnrolled && conv) break;
        if (MODE == kModeUnrolled && rec && lane == 0) {
          rec->v[level][it] = make_float2(vx, vy);
          rec->delta[level][it] = last_delta;
        }
        cx = __fadd_rn(cx, vx);
        cy = __fadd_rn(cy, vy);
        ++steps;
      }
      if (MODE == kModeUnrolled && !good) conv = false;
      if (MODE == kModeUnrolled && rec && lane == 0) {
        rec->it[level][steps] = make_float2(cx, cy);
        rec->K[level] = steps;
      }
      if (conv) {
        // radius / 2^level, exact as a product with 2^-level (no subnormal for a pixel radius)
        const float r = __fmul_rn(radius, __int_as_float((127 - level) << 23));
        const float dx = __fsub_rn(cx, savex), dy = __fsub_rn(cy, savey);
        if (__fmaf_rn(dx, dx, __fmul_rn(dy, dy)) > __fmul_rn(r, r)) conv = false;
      }
      if (conv) {
        if (cnt && lane == 0) atomicAdd(cnt + 2, 1ull);
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
        warp_sum3(s1, s2, s11, lane);
        warp_sum2(s22, s12, lane);
        const float a1 = __fmul_rn(s1, rcp25), a2 = __fmul_rn(s2, rcp25);
        const float d1 = __fmaf_rn(s11, rcp25, -__fmul_rn(a1, a1));
        const float d2 = __fmaf_rn(s22, rcp25, -__fmul_rn(a2, a2));
        const float d12 = __fmaf_rn(s12, rcp25, -__fmul_rn(a1, a2));
        const float d1d2 = __fmul_rn(d1, d2);
        const float ncc = d1d2 < 1.1920928955078125e-07f ? 0.f : __fmul_rn(d12, __frsqrt_rn(d1d2));
        conv = ncc > ncc_thr;
      }
      if (MODE == kModeUnrolled && rec && lane == 0 && conv) rec->flags[level] |= 2;
      if (!conv && level > 0) {
        cx = savex;
        cy = savey;
      }
      if (MODE == kModeImplicit && level == 0 && conv) {
        // Newton steps on e(c) = 0 with its exact Jacobian J = sum w g (dP2/dc - mean)^T: the same
        // fixed point the Gauss-Newton steps approach (linearly, as the derivative filter's gain
        // under-relaxes them), reached quadratically.  The track is kept only if the steps settle.
        bool settled = false;
        const float rx = cx, ry = cy;  // the reference rule's result
        for (int it = 0; it < iters; ++it) {
          xmin = __fadd_rn(cx, -4.f);
          ymin = __fadd_rn(cy, -4.f);
          if (!(xmin >= 0.f && __fadd_rn(cx, 5.f) < (float)W && ymin >= 0.f && __fadd_rn(cy, 5.f) < (float)H)) break;
          const int nbx = (int)floorf(__fsub_rn(xmin, 0.5f)) - 1, nby = (int)floorf(__fsub_rn(ymin, 0.5f)) - 1;
          if (nbx < wbx || nbx + kPW > wbx + 4 * kCA || nby < wby || nby + kPW > wby + kCW) {
            wbx = (nbx - 2) & ~3;
            wby = nby - 2;
            __syncwarp();
            stage_aligned<kCW, kCA, kCAS>(sm.cur, CL.img, CL.pitch, CL.w, CL.h, wbx, wby, lane);
            cp_async_wait_all();
            __syncwarp();
          }
          const TapSet tc = make_taps<SAMPLING, false>(xmin, ymin, wbx, wby, kCAS, lane);
          float dxs[kNE], dys[kNE];
          float sc = 0.f, sdx = 0.f, sdy = 0.f;
#pragma unroll
          for (int e = 0; e < kNE; ++e) {
            dxs[e] = dys[e] = 0.f;
            const Tap t = tap_of<SAMPLING>(tc, ix[e], iy[e], wbx, wby, kCAS);
            if (valid[e]) {
              sample_vg(sm.cur, kCAS, t, p2[e], dxs[e], dys[e]);
              sc = __fadd_rn(sc, p2[e]);
              sdx = __fadd_rn(sdx, dxs[e]);
              sdy = __fadd_rn(sdy, dys[e]);
            }
          }
          warp_sum3(sc, sdx, sdy, lane);
          const float mdx = __fmul_rn(sdx, rcp81), mdy = __fmul_rn(sdy, rcp81);
          const float delta = __fmul_rn(__fsub_rn(sc, sp), rcp81);
          float ex = 0.f, ey = 0.f, j00 = 0.f, j01 = 0.f, j10 = 0.f, j11 = 0.f;
#pragma unroll
          for (int e = 0; e < kNE; ++e) {
            if (valid[e]) {
              const float wd = __fmul_rn(wt[e], __fsub_rn(__fsub_rn(p2[e], p1[e]), delta));
              ex = __fmaf_rn(wd, gxp[e], ex);
              ey = __fmaf_rn(wd, gyp[e], ey);
              const float wa = __fmul_rn(wt[e], gxp[e]), wb = __fmul_rn(wt[e], gyp[e]);
              const float ddx = __fsub_rn(dxs[e], mdx), ddy = __fsub_rn(dys[e], mdy);
              j00 = __fmaf_rn(wa, ddx, j00);
              j01 = __fmaf_rn(wa, ddy, j01);
              j10 = __fmaf_rn(wb, ddx, j10);
              j11 = __fmaf_rn(wb, ddy, j11);
            }
          }
          warp_sum3(ex, ey, j00, lane);
          warp_sum3(j01, j10, j11, lane);
          const float detj = __fmaf_rn(j00, j11, -__fmul_rn(j01, j10));
          if (!(fabsf(detj) > 0.f)) break;
          // c -= J^-1 e
          const float vx = -__fdiv_rn(__fmaf_rn(j11, ex, -__fmul_rn(j01, ey)), detj);
          const float vy = -__fdiv_rn(__fmaf_rn(j00, ey, -__fmul_rn(j10, ex)), detj);
          // steps and the drift from the reference result stay within 2 px (else another zero of e,
          // far from the tracked feature, could be reached)
          const float step2 = __fmaf_rn(vx, vx, __fmul_rn(vy, vy));
          if (!(step2 <= 4.f)) break;
          cx = __fadd_rn(cx, vx);
          cy = __fadd_rn(cy, vy);
          const float ddx = __fsub_rn(cx, rx), ddy = __fsub_rn(cy, ry);
          if (!(__fmaf_rn(ddx, ddx, __fmul_rn(ddy, ddy)) <= 4.f)) break;
          if (step2 < tol2) {
            // kept only when J is well conditioned: |det J| >= 0.01 |J|_F^2 (sigma_min / sigma_max
            // above about 0.01), so that the adjoint's FP32 solve J^T lambda = dL/dc is accurate
            const float fro = __fmaf_rn(j00, j00, __fmaf_rn(j01, j01, __fmaf_rn(j10, j10, __fmul_rn(j11, j11))));
            settled = fabsf(detj) >= __fmul_rn(0.01f, fro);
            break;
          }
        }
        conv = settled;
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

}  // namespace lk
}  // namespace fe
