// Affine (Shi-Tomasi) feature tracker: st_track_kernel, st_build_cache_kernel and
// st_track_with_cache_kernel (libs/cuda_modules/cuda_kernels/st_tracker.cu:320-1370), one warp per
// track.
//
// Algorithm (the reference's): coarse to fine from level min(levels - 1, (int)log1p(search radius));
// on each level the previous frame's 9x9 patch (or the cached one) against the current frame's patch
// under the affine map: shift-only Gauss-Newton steps, then full affine steps (dx, dy and the 2x2
// map) from Gaussian-weighted moments of the mean-subtracted current-frame gradients, each solved by
// a column-pivoting Householder QR with the reference's rank rule; a step stops early when the
// shift of the 2x2 system is below 0.04 px; level 0 needs that convergence and a 5x5 NCC above the
// track's threshold.  Levels whose patches leave the image are skipped (level 0 fails).
//
// Layout: the 81 taps are spread over the lanes (tap f = lane + 32 e, e < 3), each lane samples its
// taps straight from global memory (4 texels per plane, clamped; the texture unit's weight rule
// emulated as in the LK tracker), patch sums are lane-major partial sums then an xor butterfly, and
// every lane solves the small systems redundantly so the control flow stays warp-uniform.  Operations
// are unfused (__fmul_rn / __fadd_rn) so the oracle restates them exactly.
#include <cuda_runtime.h>

#include "fe_common.cuh"
#include "fe_internal.h"
#include "lk_common.cuh"

namespace fe {

namespace {

using lk::Tap;
using lk::kFull;
constexpr int kWarps = 8;
constexpr float kEps = 1.1920928955078125e-07f;

// One bilinear sample at texture coordinate (x, y) of a level plane, clamped (or_tex_sample).
template <int SAMPLING>
__device__ __forceinline__ float tex_at(const float* img, int pitch, int w, int h, float x, float y) {
  const float xb = __fsub_rn(x, 0.5f), yb = __fsub_rn(y, 0.5f);
  const float fx = floorf(xb), fy = floorf(yb);
  const float a = __fsub_rn(xb, fx), b = __fsub_rn(yb, fy);
  int i0 = (int)fx, j0 = (int)fy;
  int i1 = i0 + 1, j1 = j0 + 1;
  i0 = min(max(i0, 0), w - 1);
  i1 = min(max(i1, 0), w - 1);
  j0 = min(max(j0, 0), h - 1);
  j1 = min(max(j1, 0), h - 1);
  const float t00 = __ldg(img + (size_t)j0 * pitch + i0), t10 = __ldg(img + (size_t)j0 * pitch + i1);
  const float t01 = __ldg(img + (size_t)j1 * pitch + i0), t11 = __ldg(img + (size_t)j1 * pitch + i1);
  if (SAMPLING == FE_SAMPLE_EXACT) {
    const float top = __fmaf_rn(a, __fsub_rn(t10, t00), t00);
    const float bot = __fmaf_rn(a, __fsub_rn(t11, t01), t01);
    return __fmaf_rn(b, __fsub_rn(bot, top), top);
  }
  Tap t;
  lk::tex_weights((int)floorf(__fmaf_rn(a, 256.f, 0.5f)), (int)floorf(__fmaf_rn(b, 256.f, 0.5f)), t);
  if (SAMPLING == FE_SAMPLE_TEXTURE_WIDE) {
    double v = __dmul_rn((double)t.w00, (double)t00);
    v = __fma_rn((double)t.w10, (double)t10, v);
    v = __fma_rn((double)t.w01, (double)t01, v);
    return __double2float_rn(__fma_rn((double)t.w11, (double)t11, v));
  }
  float v = __fmul_rn(t.w00, t00);
  v = __fmaf_rn(t.w10, t10, v);
  v = __fmaf_rn(t.w01, t01, v);
  return __fmaf_rn(t.w11, t11, v);
}

__device__ __forceinline__ float wsum(float x) {
#pragma unroll
  for (int m = 1; m < 32; m <<= 1) x = __fadd_rn(x, __shfl_xor_sync(kFull, x, m));
  return x;
}

__device__ __forceinline__ bool inside(float x, float y, int w, int h) {
  return x >= 0.f && x < (float)w && y >= 0.f && y < (float)h;
}

// Column-pivoting Householder QR solve of the D x D system a z = b (row-major), as or_st_qr_solve.
template <int D>
__device__ bool qr_solve(const float* a, const float* b, float* z) {
  float R[D * D], qb[D], cn[D], cnd[D];
  int perm[D];
#pragma unroll
  for (int i = 0; i < D * D; ++i) R[i] = a[i];
#pragma unroll
  for (int i = 0; i < D; ++i) qb[i] = b[i];
  float max_norm = -1.f;
#pragma unroll
  for (int c = 0; c < D; ++c) {
    float s = 0.f;
#pragma unroll
    for (int r = 0; r < D; ++r) s = __fadd_rn(s, __fmul_rn(R[r * D + c], R[r * D + c]));
    cn[c] = __fsqrt_rn(s);
    cnd[c] = cn[c];
    if (cn[c] > max_norm) max_norm = cn[c];
    perm[c] = c;
  }
  float th = __fmul_rn(max_norm, kEps);
  th = __fdiv_rn(__fmul_rn(th, th), (float)D);
  int nzp = D;
#pragma unroll
  for (int q = 0; q < D - 1; ++q) {
    float mn = -1.f;
    int mc = -1;
#pragma unroll
    for (int c = q; c < D; ++c)
      if (cn[c] > mn) {
        mn = cn[c];
        mc = c;
      }
    if (nzp == D && __fmul_rn(mn, mn) < __fmul_rn(th, (float)(D - q))) nzp = q;
    if (q != mc) {
      // swap columns q and mc (mc is a runtime index: select instead of indexing)
#pragma unroll
      for (int c = q + 1; c < D; ++c)
        if (c == mc) {
          int t = perm[q];
          perm[q] = perm[c];
          perm[c] = t;
          float f = cn[q];
          cn[q] = cn[c];
          cn[c] = f;
          f = cnd[q];
          cnd[q] = cnd[c];
          cnd[c] = f;
#pragma unroll
          for (int r = 0; r < D; ++r) {
            f = R[r * D + q];
            R[r * D + q] = R[r * D + c];
            R[r * D + c] = f;
          }
        }
    }
    const float c0 = R[q * D + q];
    if (c0 >= 0.f) mn = -mn;
    const float div = __fadd_rn(__fmul_rn(mn, mn), __fmul_rn(c0, mn));
    float tau = __fdiv_rn(1.f, div);
    if (fabsf(div) < kEps) tau = 0.f;
    float v[D];
#pragma unroll
    for (int r = 0; r < D; ++r) v[r] = r < q ? 0.f : R[r * D + q];
    v[q] = __fadd_rn(c0, mn);
#pragma unroll
    for (int c = 0; c < D; ++c) {
      float s = 0.f;
#pragma unroll
      for (int r = q; r < D; ++r) s = __fadd_rn(s, __fmul_rn(v[r], R[r * D + c]));
      const float ts = __fmul_rn(tau, s);
#pragma unroll
      for (int r = q; r < D; ++r) R[r * D + c] = __fsub_rn(R[r * D + c], __fmul_rn(ts, v[r]));
    }
    {
      float s = 0.f;
#pragma unroll
      for (int r = q; r < D; ++r) s = __fadd_rn(s, __fmul_rn(v[r], qb[r]));
      const float ts = __fmul_rn(tau, s);
#pragma unroll
      for (int r = q; r < D; ++r) qb[r] = __fsub_rn(qb[r], __fmul_rn(ts, v[r]));
    }
#pragma unroll
    for (int c = q + 1; c < D; ++c) {
      if (cn[c] != 0.f) {
        float t = __fdiv_rn(fabsf(R[q * D + c]), cn[c]);
        t = __fmul_rn(__fadd_rn(1.f, t), __fsub_rn(1.f, t));
        if (t < 0.f) t = 0.f;
        const float rr = __fdiv_rn(cn[c], cnd[c]);
        const float t2 = __fmul_rn(__fmul_rn(t, rr), rr);
        if (t2 <= kEps) {
          float s = 0.f;
#pragma unroll
          for (int r = q + 1; r < D; ++r) s = __fadd_rn(s, __fmul_rn(R[r * D + c], R[r * D + c]));
          cnd[c] = __fsqrt_rn(s);
          cn[c] = cnd[c];
        } else {
          cn[c] = __fmul_rn(cn[c], __fsqrt_rn(t));
        }
      }
    }
  }
#pragma unroll
  for (int i = D - 1; i >= 0; --i) {
    if (i < nzp) {
      if (fabsf(R[i * D + i]) < kEps) {
        if (fabsf(qb[i]) > kEps) return false;
      } else {
        qb[i] = __fdiv_rn(qb[i], R[i * D + i]);
      }
#pragma unroll
      for (int j = i - 1; j >= 0; --j) qb[j] = __fsub_rn(qb[j], __fmul_rn(qb[i], R[j * D + i]));
    }
  }
#pragma unroll
  for (int i = 0; i < D; ++i)
#pragma unroll
    for (int k = 0; k < D; ++k)
      if (perm[i] == k) z[k] = qb[i];
  return true;
}

struct Taps {
  float wt[3], ox[3], oy[3];
  bool valid[3], ncc[3];
  int ix[3], iy[3];
};

__device__ __forceinline__ Taps make_taps(int lane) {
  Taps t;
#pragma unroll
  for (int e = 0; e < 3; ++e) {
    const int f = lane + 32 * e;
    t.valid[e] = f < 81;
    t.iy[e] = t.valid[e] ? f / 9 : 0;
    t.ix[e] = t.valid[e] ? f - t.iy[e] * 9 : 0;
    t.wt[e] = t.valid[e] ? __fmul_rn(gauss9(t.iy[e]), gauss9(t.ix[e])) : 0.f;
    t.ox[e] = (float)(t.ix[e] - 4);
    t.oy[e] = (float)(t.iy[e] - 4);
    t.ncc[e] = t.valid[e] && t.ix[e] >= 2 && t.ix[e] < 7 && t.iy[e] >= 2 && t.iy[e] < 7;
  }
  return t;
}

// Lane-major partial sum of a per-tap expression, then the butterfly.
#define TAP_SUM(T, expr)                              \
  ({                                                  \
    float acc_ = 0.f;                                 \
    _Pragma("unroll") for (int e = 0; e < 3; ++e) if ((T).valid[e]) acc_ = __fadd_rn(acc_, (expr)); \
    wsum(acc_);                                       \
  })

// The current patch (image and, when g is set, gradients) at map m around (cx, cy); false when it
// leaves the level.  Warp-uniform.
template <int SAMPLING>
__device__ bool sample_current(const Level& L, float cx, float cy, const float* m, const Taps& T, float* p, float* gx,
                               float* gy, bool g) {
  const bool id = m[0] == 1.f && m[1] == 0.f && m[2] == 0.f && m[3] == 1.f;
  float sx[3], sy[3];
  bool ok = true;
  if (id) {
    const float xmin = __fadd_rn(__fsub_rn(cx, 4.5f), 0.5f), ymin = __fadd_rn(__fsub_rn(cy, 4.5f), 0.5f);
    if (xmin < 0.f || __fadd_rn(xmin, 9.f) >= (float)L.w || ymin < 0.f || __fadd_rn(ymin, 9.f) >= (float)L.h) return false;
#pragma unroll
    for (int e = 0; e < 3; ++e) {
      sx[e] = __fadd_rn(xmin, (float)T.ix[e]);
      sy[e] = __fadd_rn(ymin, (float)T.iy[e]);
    }
  } else {
    const float x00 = __fsub_rn(__fsub_rn(cx, 0.5f), __fdiv_rn(__fmul_rn(8.f, __fadd_rn(m[0], m[1])), 2.f));
    const float y00 = __fsub_rn(__fsub_rn(cy, 0.5f), __fdiv_rn(__fmul_rn(8.f, __fadd_rn(m[2], m[3])), 2.f));
#pragma unroll
    for (int e = 0; e < 3; ++e) {
      const float x = __fadd_rn(__fadd_rn(x00, __fmul_rn(m[0], (float)T.ix[e])), __fmul_rn(m[1], (float)T.iy[e]));
      const float y = __fadd_rn(__fadd_rn(y00, __fmul_rn(m[2], (float)T.ix[e])), __fmul_rn(m[3], (float)T.iy[e]));
      if (T.valid[e] && (x < 0.f || x >= (float)L.w || y < 0.f || y >= (float)L.h)) ok = false;
      sx[e] = __fadd_rn(x, 0.5f);
      sy[e] = __fadd_rn(y, 0.5f);
    }
    if (!__all_sync(kFull, ok)) return false;
  }
#pragma unroll
  for (int e = 0; e < 3; ++e) {
    if (!T.valid[e]) {
      p[e] = 0.f;
      if (g) gx[e] = gy[e] = 0.f;
      continue;
    }
    p[e] = tex_at<SAMPLING>(L.img, L.pitch, L.w, L.h, sx[e], sy[e]);
    if (g) {
      gx[e] = tex_at<SAMPLING>(L.gx, L.pitch, L.w, L.h, sx[e], sy[e]);
      gy[e] = tex_at<SAMPLING>(L.gy, L.pitch, L.w, L.h, sx[e], sy[e]);
    }
  }
  return true;
}

template <int SAMPLING>
__device__ bool sample_previous(const Level& L, float u, float v, const Taps& T, float* p, float& sum) {
  const float xmin = __fadd_rn(__fsub_rn(u, 4.5f), 0.5f), ymin = __fadd_rn(__fsub_rn(v, 4.5f), 0.5f);
  if (xmin < 0.f || __fadd_rn(xmin, 9.f) >= (float)L.w || ymin < 0.f || __fadd_rn(ymin, 9.f) >= (float)L.h) return false;
#pragma unroll
  for (int e = 0; e < 3; ++e)
    p[e] = T.valid[e] ? tex_at<SAMPLING>(L.img, L.pitch, L.w, L.h, __fadd_rn(xmin, (float)T.ix[e]),
                                         __fadd_rn(ymin, (float)T.iy[e]))
                      : 0.f;
  sum = TAP_SUM(T, p[e]);
  return true;
}

struct State {
  float cx, cy, m[4];
  bool converged;
};

// Gauss-Newton refinement against the previous patch; false when a patch leaves the level or a
// solve fails (or_st refine()).
template <int SAMPLING>
__device__ bool refine(const Level& L, const float* prev, float prev_sum, int n_shift, int n_full, const Taps& T,
                       State& s) {
  float m[4] = {s.m[0], s.m[1], s.m[2], s.m[3]};
  float cx = s.cx, cy = s.cy;
  for (int it = 0; it < n_shift + n_full; ++it) {
    const bool full = it >= n_shift;
    if (!inside(cx, cy, L.w, L.h)) return false;
    float p[3], gx[3], gy[3], r[3];
    if (!sample_current<SAMPLING>(L, cx, cy, m, T, p, gx, gy, true)) return false;
    const float cs = TAP_SUM(T, p[e]), gxs = TAP_SUM(T, gx[e]), gys = TAP_SUM(T, gy[e]);
    const float delta = __fdiv_rn(__fsub_rn(cs, prev_sum), 81.f);
    const float gxm = __fdiv_rn(gxs, 81.f), gym = __fdiv_rn(gys, 81.f);
#pragma unroll
    for (int e = 0; e < 3; ++e) {
      gx[e] = __fsub_rn(gx[e], gxm);
      gy[e] = __fsub_rn(gy[e], gym);
      r[e] = __fsub_rn(__fsub_rn(p[e], prev[e]), delta);
    }
    const float sxx = TAP_SUM(T, __fmul_rn(__fmul_rn(T.wt[e], gx[e]), gx[e]));
    const float sxy = TAP_SUM(T, __fmul_rn(__fmul_rn(T.wt[e], gx[e]), gy[e]));
    const float syy = TAP_SUM(T, __fmul_rn(__fmul_rn(T.wt[e], gy[e]), gy[e]));
    const float rx = TAP_SUM(T, __fmul_rn(__fmul_rn(T.wt[e], r[e]), gx[e]));
    const float ry = TAP_SUM(T, __fmul_rn(__fmul_rn(T.wt[e], r[e]), gy[e]));
    const float det = __fsub_rn(__fmul_rn(sxx, syy), __fmul_rn(sxy, sxy));
    const float vx = __fdiv_rn(__fsub_rn(__fmul_rn(syy, rx), __fmul_rn(sxy, ry)), det);
    const float vy = __fdiv_rn(__fsub_rn(__fmul_rn(sxx, ry), __fmul_rn(sxy, rx)), det);
    s.converged = __fsqrt_rn(__fadd_rn(__fmul_rn(vx, vx), __fmul_rn(vy, vy))) < 0.04f;
    if (s.converged) break;
    if (full) {
      // moments (position weight x, y, x^2, xy, y^2) x (gx gx, gx gy, gy gy), and residual moments
      float mm[6][3];
      mm[0][0] = sxx;
      mm[0][1] = sxy;
      mm[0][2] = syy;
#pragma unroll
      for (int k = 1; k < 6; ++k) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          mm[k][c] = TAP_SUM(T, __fmul_rn(
              __fmul_rn(k == 1 ? T.ox[e] : k == 2 ? T.oy[e] : k == 3 ? __fmul_rn(T.ox[e], T.ox[e])
                        : k == 4 ? __fmul_rn(T.ox[e], T.oy[e]) : __fmul_rn(T.oy[e], T.oy[e]), T.wt[e]),
              c == 0 ? __fmul_rn(gx[e], gx[e]) : c == 1 ? __fmul_rn(gx[e], gy[e]) : __fmul_rn(gy[e], gy[e])));
        }
      }
      float rr[4];
#pragma unroll
      for (int k = 0; k < 4; ++k)
        rr[k] = TAP_SUM(T, __fmul_rn(__fmul_rn(r[e], __fmul_rn(k < 2 ? T.ox[e] : T.oy[e], T.wt[e])),
                                     (k % 2 == 0) ? gx[e] : gy[e]));
      const float A[36] = {mm[3][0], mm[3][1], mm[4][0], mm[4][1], mm[1][0], mm[1][1],
                           mm[3][1], mm[3][2], mm[4][1], mm[4][2], mm[1][1], mm[1][2],
                           mm[4][0], mm[4][1], mm[5][0], mm[5][1], mm[2][0], mm[2][1],
                           mm[4][1], mm[4][2], mm[5][1], mm[5][2], mm[2][1], mm[2][2],
                           mm[1][0], mm[1][1], mm[2][0], mm[2][1], mm[0][0], mm[0][1],
                           mm[1][1], mm[1][2], mm[2][1], mm[2][2], mm[0][1], mm[0][2]};
      const float bv[6] = {rr[0], rr[1], rr[2], rr[3], rx, ry};
      float z[6];
      if (!qr_solve<6>(A, bv, z)) return false;
      m[0] = __fadd_rn(m[0], z[0]);
      m[1] = __fadd_rn(m[1], z[1]);
      m[2] = __fadd_rn(m[2], z[2]);
      m[3] = __fadd_rn(m[3], z[3]);
      cx = __fadd_rn(cx, z[4]);
      cy = __fadd_rn(cy, z[5]);
    } else {
      const float A[4] = {sxx, sxy, sxy, syy}, bv[2] = {rx, ry};
      float z[2];
      if (!qr_solve<2>(A, bv, z)) return false;
      cx = __fadd_rn(cx, z[0]);
      cy = __fadd_rn(cy, z[1]);
    }
  }
  if (!inside(cx, cy, L.w, L.h)) return false;
  s.cx = cx;
  s.cy = cy;
#pragma unroll
  for (int k = 0; k < 4; ++k) s.m[k] = m[k];
  return true;
}

__device__ __forceinline__ void up(float& x, float& y) {
  x = __fsub_rn(__fmul_rn(x, 2.f), 0.5f);
  y = __fsub_rn(__fmul_rn(y, 2.f), 0.5f);
}

template <int SAMPLING, bool CACHED>
__global__ void __launch_bounds__(kWarps * 32) st_track_kernel(const __grid_constant__ StLaunch P) {
  const int lane = threadIdx.x & 31;
  const int g = blockIdx.x * kWarps + (threadIdx.x >> 5);
  if (g >= P.n) return;
  fe_track_data& td = P.tracks[g];
  const Taps T = make_taps(lane);
  const fe_affine_cache* cd = nullptr;
  if (CACHED) {
    if (td.cache_index < 0 || td.cache_index >= P.n_cache) {
      if (lane == 0) td.track_status = 0;
      return;
    }
    cd = P.cache + td.cache_index;
  }
  const float radius = td.search_radius_px;
  if (radius < 0.f) {
    if (lane == 0) td.track_status = 0;
    return;
  }
  const int levels = P.cur.levels;
  const int top = min(levels - 1, (int)log1pf(radius));
  const float tx = td.track[0], ty = td.track[1];
  if (!CACHED && !inside(tx, ty, P.prev.lv[0].w, P.prev.lv[0].h)) {
    if (lane == 0) td.track_status = 0;
    return;
  }
  const float scale = 1.f / (float)(1 << top);
  float pu = __fadd_rn(__fmul_rn(__fsub_rn(tx, 0.5f), scale), 0.5f);
  float pv = __fadd_rn(__fmul_rn(__fsub_rn(ty, 0.5f), scale), 0.5f);
  State s;
  s.m[0] = td.initial_guess_map[0];
  s.m[1] = td.initial_guess_map[1];
  s.m[2] = td.initial_guess_map[2];
  s.m[3] = td.initial_guess_map[3];
  s.cx = __fadd_rn(__fmul_rn(__fsub_rn(__fadd_rn(tx, td.offset[0]), 0.5f), scale), 0.5f);
  s.cy = __fadd_rn(__fmul_rn(__fsub_rn(__fadd_rn(ty, td.offset[1]), 0.5f), scale), 0.5f);
  s.converged = false;
  float ncc_out = 0.f;
  for (int level = top; level >= 0; --level) {
    const Level& L = P.cur.lv[level];
    if (!CACHED && !inside(pu, pv, L.w, L.h)) {
      if (lane == 0) td.track_status = 0;
      return;
    }
    if (!inside(s.cx, s.cy, L.w, L.h)) {
      if (lane == 0) td.track_status = 0;
      return;
    }
    float prev[3], prev_sum = 0.f;
    bool have = true;
    if (CACHED) {
      if (!((cd->level_mask >> level) & 1u) && level > 0) {
        up(s.cx, s.cy);
        up(pu, pv);
        continue;
      }
#pragma unroll
      for (int e = 0; e < 3; ++e) prev[e] = T.valid[e] ? cd->patch[81 * level + lane + 32 * e] : 0.f;
      prev_sum = cd->patch_sums[level];
    } else {
      have = sample_previous<SAMPLING>(P.prev.lv[level], pu, pv, T, prev, prev_sum);
      if (!have && level > 0) {
        up(s.cx, s.cy);
        up(pu, pv);
        continue;
      }
    }
    __syncwarp();
    if (lane < 4) td.info[lane] = (lane == 0 || lane == 3) ? 1.f / 9.f : 0.f;
    const bool ok = have && refine<SAMPLING>(L, prev, prev_sum, P.n_shift, P.n_full, T, s);
    if (!ok) {
      if (level > 0) {
        up(s.cx, s.cy);
        up(pu, pv);
        continue;
      }
      if (lane == 0) td.track_status = 0;
      return;
    }
    float cur[3];
    if (!sample_current<SAMPLING>(L, s.cx, s.cy, s.m, T, cur, nullptr, nullptr, false)) {
      if (lane == 0) td.track_status = 0;
      return;
    }
    if (level == 0) {
      const float cs = TAP_SUM(T, T.ncc[e] ? cur[e] : 0.f), ps = TAP_SUM(T, T.ncc[e] ? prev[e] : 0.f);
      const float css = TAP_SUM(T, T.ncc[e] ? __fmul_rn(cur[e], cur[e]) : 0.f);
      const float pss = TAP_SUM(T, T.ncc[e] ? __fmul_rn(prev[e], prev[e]) : 0.f);
      const float cps = TAP_SUM(T, T.ncc[e] ? __fmul_rn(cur[e], prev[e]) : 0.f);
      const float cm = __fdiv_rn(cs, 25.f), pm = __fdiv_rn(ps, 25.f);
      const float cv = __fsub_rn(__fdiv_rn(css, 25.f), __fmul_rn(cm, cm));
      const float pvv = __fsub_rn(__fdiv_rn(pss, 25.f), __fmul_rn(pm, pm));
      const float cov = __fsub_rn(__fdiv_rn(cps, 25.f), __fmul_rn(cm, pm));
      const float d = __fmul_rn(cv, pvv);
      const float c = d < kEps ? 0.f : __fdiv_rn(cov, __fsqrt_rn(d));
      if (c <= td.ncc_threshold || !s.converged) {
        __syncwarp();
        if (lane == 0) td.track_status = 0;
        return;
      }
      ncc_out = c;
    } else {
      up(s.cx, s.cy);
      up(pu, pv);
    }
  }
  __syncwarp();
  if (lane == 0) {
    td.ncc = ncc_out;
    td.track[0] = s.cx;
    td.track[1] = s.cy;
    td.track_status = inside(s.cx, s.cy, P.cur.lv[0].w, P.cur.lv[0].h) ? 1 : 0;
  }
}

template <int SAMPLING>
__global__ void __launch_bounds__(kWarps * 32) st_build_kernel(const __grid_constant__ StLaunch P) {
  const int lane = threadIdx.x & 31;
  const int g = blockIdx.x * kWarps + (threadIdx.x >> 5);
  if (g >= P.n) return;
  fe_track_data& td = P.tracks[g];
  fe_affine_cache& c = P.cache_out[g];
  const int levels = P.prev.levels;
  if (levels == 0) {
    if (lane == 0) td.cache_index = -1;
    return;
  }
  const Taps T = make_taps(lane);
  int level = levels - 1;
  const float scale = 1.f / (float)(1 << level);
  float pu = __fadd_rn(__fmul_rn(__fsub_rn(td.track[0], 0.5f), scale), 0.5f);
  float pv = __fadd_rn(__fmul_rn(__fsub_rn(td.track[1], 0.5f), scale), 0.5f);
  uint32_t mask = 0;
  for (;; --level) {
    const Level& L = P.prev.lv[level];
    if (inside(pu, pv, L.w, L.h)) {
      float p[3], sum;
      if (sample_previous<SAMPLING>(L, pu, pv, T, p, sum)) {
#pragma unroll
        for (int e = 0; e < 3; ++e)
          if (T.valid[e]) c.patch[81 * level + lane + 32 * e] = p[e];
        if (lane == 0) c.patch_sums[level] = sum;
        mask |= 1u << level;
      }
    }
    if (level > 0) up(pu, pv);
    if (level == 0) break;
  }
  if (lane == 0) {
    c.level_mask = mask;
    td.cache_index = g;
  }
}

template <int SAMPLING>
cudaError_t launch_sampling(const StLaunch& p, int kind, cudaStream_t s) {
  const int blocks = (p.n + kWarps - 1) / kWarps;
  if (kind == 0)
    st_track_kernel<SAMPLING, false><<<blocks, kWarps * 32, 0, s>>>(p);
  else if (kind == 1)
    st_track_kernel<SAMPLING, true><<<blocks, kWarps * 32, 0, s>>>(p);
  else
    st_build_kernel<SAMPLING><<<blocks, kWarps * 32, 0, s>>>(p);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_st(const StLaunch& p, int kind, cudaStream_t s) {
  if (p.n <= 0) return cudaSuccess;
  if (p.sampling == FE_SAMPLE_EXACT) return launch_sampling<FE_SAMPLE_EXACT>(p, kind, s);
  if (p.sampling == FE_SAMPLE_TEXTURE_WIDE) return launch_sampling<FE_SAMPLE_TEXTURE_WIDE>(p, kind, s);
  return launch_sampling<FE_SAMPLE_TEXTURE>(p, kind, s);
}

}  // namespace fe
