// Pyramidal LK with the texture unit's own bilinear filtering (FE_SAMPLE_HARDWARE): the reference
// rule of lk_track_kernel / lk_track_horizontal_kernel (lk_tracker.cu:69-379, 381-665), sampled as
// the reference samples (tex2D on linear-filtered, clamped texture objects of the pyramid planes, at
// the coordinates xmin + i, ymin + j).
//
// One warp per track (a one-warp block per track, so that a long track holds no other warp), tap
// f = lane + 32 e (e < 3) as in lk.cu, window sums as lane partial sums then the xor butterfly over
// masks 1, 2, 4, 8, 16, which pairs lanes as the reference's warp reduction does.  The arithmetic is
// written plainly, as the reference writes it, and left to the compiler to contract into fused
// multiply-adds as the reference's build does, with the reference's fast reciprocal of the
// determinant: the records equal lk_track_kernel's bit for bit (the emulated modes cannot, their
// samples differ from the texture unit's in the last bits).  A level's texture handles are read once
// into registers before its samples.
#include <cuda_runtime.h>

#include "fe_common.cuh"
#include "fe_internal.h"

namespace fe {

namespace {

constexpr int kTE = 3;  // taps per lane: ceil(81 / 32)

__device__ __forceinline__ float tex(cudaTextureObject_t t, float x, float y) { return tex2D<float>(t, x, y); }

// COUNT: `cnt` counts the work done, as lk_track.cuh's: [0] levels set up, [1] Gauss-Newton steps,
// [2] NCC evaluations (a separate instantiation, so that the timed kernel carries no counting code).
template <bool HORIZ, bool COUNT>
__device__ void track_hw(const LkCam& cam, const LkTex& T, fe_track_data& td, float ncc_thr, int lane,
                         unsigned long long* cnt) {
  const float radius = td.search_radius_px;
  if (radius < 0.f) {
    __syncwarp();
    if (lane == 0) td.track_status = 0;
    return;
  }
  const float tx = td.track[0], ty = td.track[1];
  const float cx0 = (tx + td.offset[0]), cy0 = (ty + td.offset[1]);
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
  float sx = (tx - 0.5f) * scale + 0.5f, sy = (ty - 0.5f) * scale + 0.5f;
  float cx = (cx0 - 0.5f) * scale + 0.5f, cy = (cy0 - 0.5f) * scale + 0.5f;

  float fx[kTE], fy[kTE], wt[kTE];
  bool valid[kTE], nccm[kTE];
#pragma unroll
  for (int e = 0; e < kTE; ++e) {
    const int f = lane + 32 * e;
    valid[e] = f < 81;
    const int iy = valid[e] ? f / 9 : 0, ix = valid[e] ? f - (f / 9) * 9 : 0;
    fx[e] = (float)ix;
    fy[e] = (float)iy;
    nccm[e] = valid[e] && ix >= 2 && ix < 7 && iy >= 2 && iy < 7;
    wt[e] = valid[e] ? gauss9(iy) * gauss9(ix) : 0.f;
  }
  const float rcp81 = 1.f / 81.f, rcp25 = 1.f / 25.f;
  const float thr2 = 0.12f * 0.12f;
  bool conv = false;

  for (int i = 0; i < levels; ++i) {
    const int level = top - i;
    const Level& CL = cam.cur.lv[level];
    const int W = CL.w, H = CL.h;
    float xmin = (sx + -4.f), ymin = (sy + -4.f);
    bool good = xmin >= 0.f && (sx + 5.f) < (float)W && ymin >= 0.f && (sy + 5.f) < (float)H;
    if (good) {
      if (COUNT && lane == 0) atomicAdd(cnt, 1ull);
      const cudaTextureObject_t t_gx = (cudaTextureObject_t)T.prev_gx[level];
      const cudaTextureObject_t t_gy = HORIZ ? 0 : (cudaTextureObject_t)T.prev_gy[level];
      const cudaTextureObject_t t_p1 = (cudaTextureObject_t)T.prev_img[level];
      const cudaTextureObject_t t_p2 = (cudaTextureObject_t)T.cur_img[level];
      // the first Gauss-Newton step's patch (the loop's first iterate, same coordinates), fetched
      // together with the template's so that both wait on one texture round trip
      float p2[kTE];
      {
        const float xm = (cx + -4.f), ym = (cy + -4.f);
#pragma unroll
        for (int e = 0; e < kTE; ++e) p2[e] = valid[e] ? tex(t_p2, (xm + fx[e]), (ym + fy[e])) : 0.f;
      }
      float gxp[kTE], gyp[kTE], p1[kTE];
      float sgx = 0.f, sgy = 0.f, sp = 0.f;
#pragma unroll
      for (int e = 0; e < kTE; ++e) {
        gxp[e] = gyp[e] = p1[e] = 0.f;
        if (valid[e]) {
          const float px = (xmin + fx[e]), py = (ymin + fy[e]);
          gxp[e] = tex(t_gx, px, py);
          if (!HORIZ) gyp[e] = tex(t_gy, px, py);
          p1[e] = tex(t_p1, px, py);
          sgx = (sgx + gxp[e]);
          if (!HORIZ) sgy = (sgy + gyp[e]);
          sp = (sp + p1[e]);
        }
      }
      if (HORIZ) warp_sum2(sgx, sp, lane);
      else warp_sum3(sgx, sgy, sp, lane);
      float lxx = 1.f / 32.f, lxy = 0.f, lyy = 1.f / 32.f;
#pragma unroll
      for (int e = 0; e < kTE; ++e) {
        if (valid[e]) {
          const float a = (-sgx * rcp81 + gxp[e]);
          gxp[e] = a;
          if (HORIZ) {
            lxx = wt[e] * a * a + lxx;
          } else {
            const float bq = (-sgy * rcp81 + gyp[e]);
            gyp[e] = bq;
            lxx = a * a * wt[e] + lxx;
            lxy = a * bq * wt[e] + lxy;
            lyy = bq * bq * wt[e] + lyy;
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
        det_rcp = __fdividef(1.0f, gxx);
      } else {
        const float det = gxx * gyy - gxy * gxy;
        if (det < 1.1920928955078125e-07f) {
          if (lane == 0) td.track_status = 0;
          return;
        }
        det_rcp = __fdividef(1.0f, det);
      }
      const float savex = cx, savey = cy;
      for (int it = 0; it < 11; ++it) {
        xmin = (cx + -4.f);
        ymin = (cy + -4.f);
        if (!(xmin >= 0.f && (cx + 5.f) < (float)W && ymin >= 0.f && (cy + 5.f) < (float)H)) break;
        if (COUNT && lane == 0) atomicAdd(cnt + 1, 1ull);
        float sc = 0.f;
#pragma unroll
        for (int e = 0; e < kTE; ++e) {
          if (valid[e]) {
            if (it > 0) p2[e] = tex(t_p2, (xmin + fx[e]), (ymin + fy[e]));
            sc = (sc + p2[e]);
          }
        }
        sc = warp_sum(sc);
        const float delta = (sc - sp) * rcp81;
        float ex = 0.f, ey = 0.f;
#pragma unroll
        for (int e = 0; e < kTE; ++e) {
          if (valid[e]) {
            const float wd = wt[e] * ((p2[e] - p1[e]) - delta);
            ex = (wd * gxp[e] + ex);
            if (!HORIZ) ey = (wd * gyp[e] + ey);
          }
        }
        float vx, vy;
        if (HORIZ) {
          ex = warp_sum(ex);
          vx = (ex * det_rcp);
          vy = 0.f;
        } else {
          warp_sum2(ex, ey, lane);
          vx = (gyy * ex - gxy * ey) * det_rcp;
          vy = (gxx * ey - gxy * ex) * det_rcp;
        }
        conv = HORIZ ? fabsf(vx) < 0.12f : (vx * vx +  (vy * vy)) < thr2;
        if (conv) break;
        cx = (cx + vx);
        cy = (cy + vy);
      }
      if (conv) {
        const float r = __fdiv_rn(radius, (float)(1 << level));
        const float dx = (cx - savex), dy = (cy - savey);
        if ((dx * dx +  (dy * dy)) > (r * r)) conv = false;
      }
      if (conv) {
        if (COUNT && lane == 0) atomicAdd(cnt + 2, 1ull);
        float s1 = 0.f, s2 = 0.f, s11 = 0.f, s22 = 0.f, s12 = 0.f;
#pragma unroll
        for (int e = 0; e < kTE; ++e) {
          if (nccm[e]) {
            s1 = (s1 + p1[e]);
            s2 = (s2 + p2[e]);
            s11 = (p1[e] * p1[e] + s11);
            s22 = (p2[e] * p2[e] + s22);
            s12 = (p2[e] * p1[e] + s12);
          }
        }
        warp_sum3(s1, s2, s11, lane);
        warp_sum2(s22, s12, lane);
        const float a1 = (s1 * rcp25), a2 = (s2 * rcp25);
        const float d1 = s11 * rcp25 - a1 * a1;
        const float d2 = s22 * rcp25 - a2 * a2;
        const float d12 = s12 * rcp25 - a1 * a2;
        const float d1d2 = (d1 * d2);
        const float ncc = d1d2 < 1.1920928955078125e-07f ? 0.f : (d12 * __frsqrt_rn(d1d2));
        conv = ncc > ncc_thr;
      }
      if (!conv && level > 0) {
        cx = savex;
        cy = savey;
      }
      conv = (level == 0) && conv;
    }
    if (i != levels - 1) {
      sx = (sx * 2.f + -0.5f);
      sy = (sy * 2.f + -0.5f);
      cx = (cx * 2.f + -0.5f);
      cy = (cy * 2.f + -0.5f);
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

template <bool HORIZ, bool COUNT>
__global__ void __launch_bounds__(32) lk_hw_kernel(const __grid_constant__ LkLaunch p) {
  const int lane = threadIdx.x;
  const int g = blockIdx.x;
  if (g >= p.total) return;
  const LkCam* cams = p.cams ? p.cams : &p.single;
  int lo = 0, hi = p.ncams - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (cams[mid].begin <= g) lo = mid; else hi = mid - 1;
  }
  const LkCam& cam = cams[lo];
  const LkTex& T = p.texs ? p.texs[lo] : p.single_tex;
  fe_track_data& td = cam.tracks[g - cam.begin];
  if (cam.tracks_in) {
    // out-of-place: the 80-byte record is copied first, then tracked in place
    if (lane < 20)
      reinterpret_cast<uint32_t*>(&td)[lane] = reinterpret_cast<const uint32_t*>(&cam.tracks_in[g - cam.begin])[lane];
    __syncwarp();
  }
  track_hw<HORIZ, COUNT>(cam, T, td, td.ncc_threshold, lane, p.counts);
  if (cam.retrack_ncc > 0.f) {
    // MonoSOFGPU's retrack pass (as lk.cu): a track the first pass lost runs again from the same
    // inputs with the retrack NCC threshold
    __syncwarp();
    if (td.track_status == 0 && td.search_radius_px >= 0.f)
      track_hw<HORIZ, COUNT>(cam, T, td, cam.retrack_ncc, lane, p.counts);
  }
}

}  // namespace

cudaError_t launch_lk_hw(const LkLaunch& p, cudaStream_t s) {
  if (p.total <= 0) return cudaSuccess;
  if (!p.texs && p.cams) return cudaErrorInvalidValue;
  if (p.counts) {
    if (p.horizontal)
      lk_hw_kernel<true, true><<<p.total, 32, 0, s>>>(p);
    else
      lk_hw_kernel<false, true><<<p.total, 32, 0, s>>>(p);
  } else if (p.horizontal) {
    lk_hw_kernel<true, false><<<p.total, 32, 0, s>>>(p);
  } else {
    lk_hw_kernel<false, false><<<p.total, 32, 0, s>>>(p);
  }
  return cudaGetLastError();
}

}  // namespace fe
