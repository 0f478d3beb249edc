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
// Layout: persistent warps take tracks from a counter.  The 81 taps are spread over the lanes
// (tap f = lane + 32 e, e < 3); each lane samples its taps straight from global memory (4 texels per
// plane, clamped, one bilinear set-up shared by the image and both gradients; the texture unit's
// weight rule emulated as in the LK tracker).  A patch sum is a lane-major partial sum then an xor
// butterfly; the 19 moments of a full step are summed by recursive halving (value k ends in lane k,
// each addition pairing the same partial sums as the butterfly) and gathered straight into the
// columns of the 6x6 system.  The QR solve is spread over the warp: lane c holds column c, lane D the
// right side, so each reflector and norm update runs once per column in parallel.  Operations are
// unfused (__fmul_rn / __fadd_rn) so the oracle restates them exactly.
#include <cuda_runtime.h>

#include "fe_common.cuh"
#include "fe_internal.h"
#include "lk_common.cuh"

namespace fe {

namespace {

using lk::kFull;
using lk::Tap;
constexpr int kWarps = 8;
#ifndef FE_ST_MIN_BLOCKS
#define FE_ST_MIN_BLOCKS 3  // tracking blocks per SM the register budget is sized for (80 registers)
#endif
constexpr int kMinBlocks = FE_ST_MIN_BLOCKS;
constexpr float kEps = 1.1920928955078125e-07f;

// Bilinear set-up of one sample at texture coordinate (x, y) of a level: the four clamped texel
// offsets and the weights (or_tex_sample).
template <int SAMPLING>
struct Bilerp {
  int o00, o10, o01, o11;
  float a, b;  // exact fractions (FE_SAMPLE_EXACT)
  Tap w;       // texture-unit weights
};

template <int SAMPLING>
__device__ __forceinline__ Bilerp<SAMPLING> bilerp(const Level& L, float x, float y) {
  Bilerp<SAMPLING> s;
  const float xb = __fsub_rn(x, 0.5f), yb = __fsub_rn(y, 0.5f);
  const float fx = floorf(xb), fy = floorf(yb);
  s.a = __fsub_rn(xb, fx);
  s.b = __fsub_rn(yb, fy);
  const int i0 = (int)fx, j0 = (int)fy;
  const int i0c = min(max(i0, 0), L.w - 1), i1c = min(max(i0 + 1, 0), L.w - 1);
  const int r0 = min(max(j0, 0), L.h - 1) * L.pitch, r1 = min(max(j0 + 1, 0), L.h - 1) * L.pitch;
  s.o00 = r0 + i0c;
  s.o10 = r0 + i1c;
  s.o01 = r1 + i0c;
  s.o11 = r1 + i1c;
  if (SAMPLING != FE_SAMPLE_EXACT)
    lk::tex_weights((int)floorf(__fmaf_rn(s.a, 256.f, 0.5f)), (int)floorf(__fmaf_rn(s.b, 256.f, 0.5f)), s.w);
  return s;
}

template <int SAMPLING>
__device__ __forceinline__ float sample(const float* plane, const Bilerp<SAMPLING>& s) {
  const float t00 = __ldg(plane + s.o00), t10 = __ldg(plane + s.o10);
  const float t01 = __ldg(plane + s.o01), t11 = __ldg(plane + s.o11);
  if (SAMPLING == FE_SAMPLE_EXACT) {
    const float top = __fmaf_rn(s.a, __fsub_rn(t10, t00), t00);
    const float bot = __fmaf_rn(s.a, __fsub_rn(t11, t01), t01);
    return __fmaf_rn(s.b, __fsub_rn(bot, top), top);
  }
  if (SAMPLING == FE_SAMPLE_TEXTURE_WIDE) {
    double v = __dmul_rn((double)s.w.w00, (double)t00);
    v = __fma_rn((double)s.w.w10, (double)t10, v);
    v = __fma_rn((double)s.w.w01, (double)t01, v);
    return __double2float_rn(__fma_rn((double)s.w.w11, (double)t11, v));
  }
  float v = __fmul_rn(s.w.w00, t00);
  v = __fmaf_rn(s.w.w10, t10, v);
  v = __fmaf_rn(s.w.w01, t01, v);
  return __fmaf_rn(s.w.w11, t11, v);
}

__device__ __forceinline__ float wsum(float x) {
#pragma unroll
  for (int m = 1; m < 32; m <<= 1) x = __fadd_rn(x, __shfl_xor_sync(kFull, x, m));
  return x;
}

// Warp sums of N <= 32 per-lane values, value k ending in lane k: recursive halving over the masks
// 1, 2, 4, 8, 16.  Each addition joins the same two partial sums as the butterfly of wsum does
// (a + b and b + a round alike), so lane k's result equals wsum(v[k]) bit for bit.
template <int N>
__device__ __forceinline__ float reduce_scatter(const float (&v)[N], int lane) {
  constexpr int N1 = (N + 1) / 2, N2 = (N1 + 1) / 2, N3 = (N2 + 1) / 2, N4 = (N3 + 1) / 2;
  float h1[N1], h2[N2], h3[N3], h4[N4], h5[1];
  const bool b0 = lane & 1, b1 = lane & 2, b2 = lane & 4, b3 = lane & 8, b4 = lane & 16;
#define RS_STEP(SRC, NS, DST, ND, BIT, MASK)                                 \
  _Pragma("unroll") for (int j = 0; j < ND; ++j) {                           \
    const float lo = SRC[2 * j], hi = 2 * j + 1 < NS ? SRC[2 * j + 1] : 0.f; \
    const float keep = BIT ? hi : lo, send = BIT ? lo : hi;                  \
    DST[j] = __fadd_rn(keep, __shfl_xor_sync(kFull, send, MASK));            \
  }
  RS_STEP(v, N, h1, N1, b0, 1)
  RS_STEP(h1, N1, h2, N2, b1, 2)
  RS_STEP(h2, N2, h3, N3, b2, 4)
  RS_STEP(h3, N3, h4, N4, b3, 8)
  RS_STEP(h4, N4, h5, 1, b4, 16)
#undef RS_STEP
  return h5[0];
}

__device__ __forceinline__ bool inside(float x, float y, int w, int h) {
  return x >= 0.f && x < (float)w && y >= 0.f && y < (float)h;
}

template <int D>
__device__ __forceinline__ float pick(const float (&a)[D], int i) {
  float x = a[0];
#pragma unroll
  for (int r = 1; r < D; ++r)
    if (r == i) x = a[r];
  return x;
}

// Column-pivoting Householder QR solve of the D x D system A z = b with or_st_qr_solve's operations,
// spread over the warp: lane c < D holds column c of A in `col`, lane D holds b, the other lanes
// zeros.  Each column (and b) sees the same operations, in the same order, as in a one-thread solve;
// the pivot choice (largest column norm, first on ties) is a reduction over lanes 0-7.  Every lane
// returns the same z and status (false: no solution).
template <int D>
__device__ bool qr_solve_warp(float (&col)[D], int lane, float (&z)[D]) {
  static_assert(D < 8, "columns live in lanes 0-7");
  const bool is_col = lane < D;
  float s = 0.f;
#pragma unroll
  for (int r = 0; r < D; ++r) s = __fadd_rn(s, __fmul_rn(col[r], col[r]));
  float cn = is_col ? __fsqrt_rn(s) : -1.f;
  float cnd = cn;
  int perm = lane;
  float max_norm = cn > -1.f ? cn : -1.f;
#pragma unroll
  for (int m = 1; m < 8; m <<= 1) max_norm = fmaxf(max_norm, __shfl_xor_sync(kFull, max_norm, m));
  max_norm = __shfl_sync(kFull, max_norm, 0);
  float th = __fmul_rn(max_norm, kEps);
  th = __fdiv_rn(__fmul_rn(th, th), (float)D);
  int nzp = D;
#pragma unroll 1
  for (int q = 0; q < D - 1; ++q) {
    // pivot: the largest remaining column norm, the first column on ties
    float key = (lane >= q && is_col && cn > -1.f) ? cn : -1.f;
    int idx = lane;
#pragma unroll
    for (int m = 1; m < 8; m <<= 1) {
      const float ok = __shfl_xor_sync(kFull, key, m);
      const int oi = __shfl_xor_sync(kFull, idx, m);
      if (ok > key || (ok == key && oi < idx)) {
        key = ok;
        idx = oi;
      }
    }
    key = __shfl_sync(kFull, key, 0);
    idx = __shfl_sync(kFull, idx, 0);
    const int mc = key > -1.f ? idx : -1;
    float mn = key > -1.f ? key : -1.f;
    if (nzp == D && __fmul_rn(mn, mn) < __fmul_rn(th, (float)(D - q))) nzp = q;
    if (mc >= 0 && mc != q) {
      const int src = lane == q ? mc : (lane == mc ? q : lane);
#pragma unroll
      for (int r = 0; r < D; ++r) col[r] = __shfl_sync(kFull, col[r], src);
      cn = __shfl_sync(kFull, cn, src);
      cnd = __shfl_sync(kFull, cnd, src);
      perm = __shfl_sync(kFull, perm, src);
    }
    const float c0 = __shfl_sync(kFull, pick(col, q), q);
    if (c0 >= 0.f) mn = -mn;
    const float div = __fadd_rn(__fmul_rn(mn, mn), __fmul_rn(c0, mn));
    float tau = __fdiv_rn(1.f, div);
    if (fabsf(div) < kEps) tau = 0.f;
    float v[D];
#pragma unroll
    for (int r = 0; r < D; ++r) {
      const float x = __shfl_sync(kFull, col[r], q);
      v[r] = r < q ? 0.f : (r == q ? __fadd_rn(c0, mn) : x);
    }
    // the reflector on this lane's column (or b)
    s = 0.f;
#pragma unroll
    for (int r = 0; r < D; ++r)
      if (r >= q) s = __fadd_rn(s, __fmul_rn(v[r], col[r]));
    const float ts = __fmul_rn(tau, s);
#pragma unroll
    for (int r = 0; r < D; ++r)
      if (r >= q) col[r] = __fsub_rn(col[r], __fmul_rn(ts, v[r]));
    // norm down-date of the remaining columns
    if (lane > q && is_col && cn != 0.f) {
      float t = __fdiv_rn(fabsf(pick(col, q)), cn);
      t = __fmul_rn(__fadd_rn(1.f, t), __fsub_rn(1.f, t));
      if (t < 0.f) t = 0.f;
      const float rr = __fdiv_rn(cn, cnd);
      const float t2 = __fmul_rn(__fmul_rn(t, rr), rr);
      if (t2 <= kEps) {
        float u = 0.f;
#pragma unroll
        for (int r = 0; r < D; ++r)
          if (r > q) u = __fadd_rn(u, __fmul_rn(col[r], col[r]));
        cnd = __fsqrt_rn(u);
        cn = cnd;
      } else {
        cn = __fmul_rn(cn, __fsqrt_rn(t));
      }
    }
  }
  float qb[D];
#pragma unroll
  for (int r = 0; r < D; ++r) qb[r] = __shfl_sync(kFull, col[r], D);
#pragma unroll
  for (int i = D - 1; i >= 0; --i) {
    if (i < nzp) {
      float ri[D];
#pragma unroll
      for (int r = 0; r <= i; ++r) ri[r] = __shfl_sync(kFull, col[r], i);
      if (fabsf(ri[i]) < kEps) {
        if (fabsf(qb[i]) > kEps) return false;
      } else {
        qb[i] = __fdiv_rn(qb[i], ri[i]);
      }
#pragma unroll
      for (int j = i - 1; j >= 0; --j) qb[j] = __fsub_rn(qb[j], __fmul_rn(qb[i], ri[j]));
    }
  }
#pragma unroll
  for (int i = 0; i < D; ++i) {
    const int p = __shfl_sync(kFull, perm, i);
#pragma unroll
    for (int k = 0; k < D; ++k)
      if (p == k) z[k] = qb[i];
  }
  return true;
}

// Slots of the 19 full-step moments after reduce_scatter: moment (m, c) of position weight m
// (1 x, 2 y, 3 x^2, 4 xy, 5 y^2) and gradient product c (0 gx gx, 1 gx gy, 2 gy gy) in slot
// 3 (m - 1) + c; the residual moments (x gx, x gy, y gx, y gy) in slots 15-18.  Row r of column c of
// the symmetric 6x6 system in the reference's layout (st_tracker.cu:632-636), and b in column 6; 31
// marks the moments with weight 1 (held by every lane).
constexpr int kColSlot[7][6] = {{6, 7, 9, 10, 0, 1},    {7, 8, 10, 11, 1, 2},   {9, 10, 12, 13, 3, 4},
                                {10, 11, 13, 14, 4, 5}, {0, 1, 3, 4, 31, 31},   {1, 2, 4, 5, 31, 31},
                                {15, 16, 17, 18, 31, 31}};

constexpr unsigned long long col_slots(int r) {
  unsigned long long v = 0;
  for (int c = 0; c < 7; ++c) v |= (unsigned long long)kColSlot[c][r] << (5 * c);
  return v;
}

// kColSlot row r packed 5 bits per column, as scalar literals for device code (a host array is not
// device data), checked against the table.
constexpr unsigned long long kSlots0 = 0x3c20524e6ull, kSlots1 = 0x40415a907ull, kSlots2 = 0x44836b149ull;
constexpr unsigned long long kSlots3 = 0x48a47356aull, kSlots4 = 0x7fff20c20ull, kSlots5 = 0x7fff29041ull;
static_assert(kSlots0 == col_slots(0) && kSlots1 == col_slots(1) && kSlots2 == col_slots(2) &&
                  kSlots3 == col_slots(3) && kSlots4 == col_slots(4) && kSlots5 == col_slots(5),
              "packed slots");

__device__ __forceinline__ int col_slot(int c, int r) {
  const unsigned long long v = r == 0   ? kSlots0
                               : r == 1 ? kSlots1
                               : r == 2 ? kSlots2
                               : r == 3 ? kSlots3
                               : r == 4 ? kSlots4
                                        : kSlots5;
  return (int)((v >> (5 * c)) & 31ull);
}

struct Taps {
  float wt[3];
  int ix[3], iy[3];
  bool valid[3];
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
  }
  return t;
}

// Lane-major partial sum of a per-tap expression (taps e = 0, 1, 2 of this lane).
#define LANE_SUM(T, expr)                                                                           \
  ({                                                                                                \
    float acc_ = 0.f;                                                                               \
    _Pragma("unroll") for (int e = 0; e < 3; ++e) if ((T).valid[e]) acc_ = __fadd_rn(acc_, (expr)); \
    acc_;                                                                                           \
  })
#define TAP_SUM(T, expr) wsum(LANE_SUM(T, expr))

// Sample coordinates of this lane's taps of the current patch at map m around (cx, cy); false (warp-
// uniform) when the patch leaves the level.
__device__ __forceinline__ bool current_coords(const Level& L, float cx, float cy, const float* m, const Taps& T,
                                               float* sx, float* sy) {
  if (m[0] == 1.f && m[1] == 0.f && m[2] == 0.f && m[3] == 1.f) {
    const float xmin = __fadd_rn(__fsub_rn(cx, 4.5f), 0.5f), ymin = __fadd_rn(__fsub_rn(cy, 4.5f), 0.5f);
    if (xmin < 0.f || __fadd_rn(xmin, 9.f) >= (float)L.w || ymin < 0.f || __fadd_rn(ymin, 9.f) >= (float)L.h)
      return false;
#pragma unroll
    for (int e = 0; e < 3; ++e) {
      sx[e] = __fadd_rn(xmin, (float)T.ix[e]);
      sy[e] = __fadd_rn(ymin, (float)T.iy[e]);
    }
    return true;
  }
  const float x00 = __fsub_rn(__fsub_rn(cx, 0.5f), __fdiv_rn(__fmul_rn(8.f, __fadd_rn(m[0], m[1])), 2.f));
  const float y00 = __fsub_rn(__fsub_rn(cy, 0.5f), __fdiv_rn(__fmul_rn(8.f, __fadd_rn(m[2], m[3])), 2.f));
  bool ok = true;
#pragma unroll
  for (int e = 0; e < 3; ++e) {
    const float x = __fadd_rn(__fadd_rn(x00, __fmul_rn(m[0], (float)T.ix[e])), __fmul_rn(m[1], (float)T.iy[e]));
    const float y = __fadd_rn(__fadd_rn(y00, __fmul_rn(m[2], (float)T.ix[e])), __fmul_rn(m[3], (float)T.iy[e]));
    if (T.valid[e] && (x < 0.f || x >= (float)L.w || y < 0.f || y >= (float)L.h)) ok = false;
    sx[e] = __fadd_rn(x, 0.5f);
    sy[e] = __fadd_rn(y, 0.5f);
  }
  return __all_sync(kFull, ok);
}

template <int SAMPLING>
__device__ bool sample_previous(const Level& L, float u, float v, const Taps& T, float* p, float& sum) {
  const float xmin = __fadd_rn(__fsub_rn(u, 4.5f), 0.5f), ymin = __fadd_rn(__fsub_rn(v, 4.5f), 0.5f);
  if (xmin < 0.f || __fadd_rn(xmin, 9.f) >= (float)L.w || ymin < 0.f || __fadd_rn(ymin, 9.f) >= (float)L.h) return false;
#pragma unroll
  for (int e = 0; e < 3; ++e)
    p[e] = T.valid[e] ? sample<SAMPLING>(L.img, bilerp<SAMPLING>(L, __fadd_rn(xmin, (float)T.ix[e]),
                                                                 __fadd_rn(ymin, (float)T.iy[e])))
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
                       int lane, State& s) {
  float m[4] = {s.m[0], s.m[1], s.m[2], s.m[3]};
  float cx = s.cx, cy = s.cy;
  for (int it = 0; it < n_shift + n_full; ++it) {
    const bool full = it >= n_shift;
    if (!inside(cx, cy, L.w, L.h)) return false;
    float sx[3], sy[3], p[3], gx[3], gy[3], r[3];
    if (!current_coords(L, cx, cy, m, T, sx, sy)) return false;
#pragma unroll
    for (int e = 0; e < 3; ++e) {
      if (T.valid[e]) {
        const Bilerp<SAMPLING> bl = bilerp<SAMPLING>(L, sx[e], sy[e]);
        p[e] = sample<SAMPLING>(L.img, bl);
        gx[e] = sample<SAMPLING>(L.gx, bl);
        gy[e] = sample<SAMPLING>(L.gy, bl);
      } else {
        p[e] = gx[e] = gy[e] = 0.f;
      }
    }
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
      float part[19];
#pragma unroll
      for (int k = 1; k < 6; ++k) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          part[3 * (k - 1) + c] = LANE_SUM(
              T, __fmul_rn(__fmul_rn(k == 1   ? (float)(T.ix[e] - 4)
                                     : k == 2 ? (float)(T.iy[e] - 4)
                                     : k == 3 ? __fmul_rn((float)(T.ix[e] - 4), (float)(T.ix[e] - 4))
                                     : k == 4 ? __fmul_rn((float)(T.ix[e] - 4), (float)(T.iy[e] - 4))
                                              : __fmul_rn((float)(T.iy[e] - 4), (float)(T.iy[e] - 4)),
                                     T.wt[e]),
                           c == 0   ? __fmul_rn(gx[e], gx[e])
                           : c == 1 ? __fmul_rn(gx[e], gy[e])
                                    : __fmul_rn(gy[e], gy[e])));
        }
      }
#pragma unroll
      for (int k = 0; k < 4; ++k)
        part[15 + k] = LANE_SUM(
            T, __fmul_rn(__fmul_rn(r[e], __fmul_rn(k < 2 ? (float)(T.ix[e] - 4) : (float)(T.iy[e] - 4), T.wt[e])),
                         (k % 2 == 0) ? gx[e] : gy[e]));
      const float slot = reduce_scatter(part, lane);
      float col[6], z[6];
      const int c = lane < 7 ? lane : 0;
#pragma unroll
      for (int rr = 0; rr < 6; ++rr) col[rr] = __shfl_sync(kFull, slot, col_slot(c, rr));
      if (lane == 4) {
        col[4] = sxx;
        col[5] = sxy;
      } else if (lane == 5) {
        col[4] = sxy;
        col[5] = syy;
      } else if (lane == 6) {
        col[4] = rx;
        col[5] = ry;
      } else if (lane >= 7) {
#pragma unroll
        for (int rr = 0; rr < 6; ++rr) col[rr] = 0.f;
      }
      if (!qr_solve_warp<6>(col, lane, z)) return false;
      m[0] = __fadd_rn(m[0], z[0]);
      m[1] = __fadd_rn(m[1], z[1]);
      m[2] = __fadd_rn(m[2], z[2]);
      m[3] = __fadd_rn(m[3], z[3]);
      cx = __fadd_rn(cx, z[4]);
      cy = __fadd_rn(cy, z[5]);
    } else {
      float col[2], z[2];
      col[0] = lane == 0 ? sxx : lane == 1 ? sxy : lane == 2 ? rx : 0.f;
      col[1] = lane == 0 ? sxy : lane == 1 ? syy : lane == 2 ? ry : 0.f;
      if (!qr_solve_warp<2>(col, lane, z)) return false;
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

// One track (st_track_kernel / st_track_with_cache_kernel).
template <int SAMPLING, bool CACHED>
__device__ void track_one(const StLaunch& P, fe_track_data& td, const Taps& T, int lane) {
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
    if ((!CACHED && !inside(pu, pv, L.w, L.h)) || !inside(s.cx, s.cy, L.w, L.h)) {
      __syncwarp();
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
    const bool ok = have && refine<SAMPLING>(L, prev, prev_sum, P.n_shift, P.n_full, T, lane, s);
    if (!ok) {
      if (level > 0) {
        up(s.cx, s.cy);
        up(pu, pv);
        continue;
      }
      __syncwarp();
      if (lane == 0) td.track_status = 0;
      return;
    }
    float sx[3], sy[3];
    if (!current_coords(L, s.cx, s.cy, s.m, T, sx, sy)) {
      __syncwarp();
      if (lane == 0) td.track_status = 0;
      return;
    }
    if (level == 0) {
      float cur[3];
      bool nc[3];
#pragma unroll
      for (int e = 0; e < 3; ++e) {
        cur[e] = T.valid[e] ? sample<SAMPLING>(L.img, bilerp<SAMPLING>(L, sx[e], sy[e])) : 0.f;
        nc[e] = T.valid[e] && T.ix[e] >= 2 && T.ix[e] < 7 && T.iy[e] >= 2 && T.iy[e] < 7;
      }
      const float cs = TAP_SUM(T, nc[e] ? cur[e] : 0.f), ps = TAP_SUM(T, nc[e] ? prev[e] : 0.f);
      const float css = TAP_SUM(T, nc[e] ? __fmul_rn(cur[e], cur[e]) : 0.f);
      const float pss = TAP_SUM(T, nc[e] ? __fmul_rn(prev[e], prev[e]) : 0.f);
      const float cps = TAP_SUM(T, nc[e] ? __fmul_rn(cur[e], prev[e]) : 0.f);
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

// Persistent warps: each takes the next track from P.counter (zeroed before the launch).
template <int SAMPLING, bool CACHED>
__global__ void __launch_bounds__(kWarps * 32, kMinBlocks) st_track_kernel(const __grid_constant__ StLaunch P) {
  const int lane = threadIdx.x & 31;
  const Taps T = make_taps(lane);
  for (;;) {
    int g = 0;
    if (lane == 0) g = atomicAdd(P.counter, 1);
    g = __shfl_sync(kFull, g, 0);
    if (g >= P.n) return;
    track_one<SAMPLING, CACHED>(P, P.tracks[g], T, lane);
    __syncwarp();
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
  __syncwarp();
  if (lane == 0) {
    c.level_mask = mask;
    td.cache_index = g;
  }
}

template <int SAMPLING, bool CACHED>
cudaError_t launch_track(const StLaunch& p, cudaStream_t s) {
  // blocks resident on the device (persistent grid), found once per process
  static const int resident = [] {
    int per_sm = 0, dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, st_track_kernel<SAMPLING, CACHED>, kWarps * 32, 0);
    return (per_sm > 0 ? per_sm : 1) * (sms > 0 ? sms : 1);
  }();
  cudaError_t e = cudaMemsetAsync(p.counter, 0, sizeof(int), s);
  if (e != cudaSuccess) return e;
  const int blocks = min((p.n + kWarps - 1) / kWarps, resident);
  st_track_kernel<SAMPLING, CACHED><<<blocks, kWarps * 32, 0, s>>>(p);
  return cudaGetLastError();
}

template <int SAMPLING>
cudaError_t launch_sampling(const StLaunch& p, int kind, cudaStream_t s) {
  if (kind == 0) return launch_track<SAMPLING, false>(p, s);
  if (kind == 1) return launch_track<SAMPLING, true>(p, s);
  st_build_kernel<SAMPLING><<<(p.n + kWarps - 1) / kWarps, kWarps * 32, 0, s>>>(p);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_st(const StLaunch& p, int kind, cudaStream_t s) {
  if (p.n <= 0) return cudaSuccess;
  if (kind != 2 && !p.counter) return cudaErrorInvalidValue;
  if (p.sampling == FE_SAMPLE_EXACT) return launch_sampling<FE_SAMPLE_EXACT>(p, kind, s);
  if (p.sampling == FE_SAMPLE_TEXTURE_WIDE) return launch_sampling<FE_SAMPLE_TEXTURE_WIDE>(p, kind, s);
  return launch_sampling<FE_SAMPLE_TEXTURE>(p, kind, s);
}

}  // namespace fe
