// Pyramidal Lucas-Kanade, one warp per track.
//
// Warps are persistent: each takes the next track of the flattened (camera, track) list from an
// atomic counter, so a warp whose track fails early moves on at once instead of idling in its CTA.
// Per level (coarse to fine) a warp stages the previous frame's window under the 9x9 patch in
// shared memory (12x12 texels of image, grad_x, grad_y) and samples the 81 bilinear taps from it (3
// per lane, lane-major like the reference); the current frame has a 16x16 window that is re-staged
// only when the Gauss-Newton iterate leaves it.  Reductions are xor-butterfly shuffles.
//
// Tap weights: the 81 taps of a patch share the fractional offset unless the FP32 coordinate
// xmin + i rounds (near a power of two).  Lanes 0-8 and 16-24 evaluate the 9 columns and 9 rows
// exactly as the reference's per-tap coordinates, a warp vote confirms that all columns and rows
// agree with column/row 0, and then every tap uses one set of weights; otherwise each tap takes
// its own column's and row's values.  Either way the result equals the per-tap evaluation.
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

#include <climits>

#include "fe_common.cuh"
#include "fe_internal.h"

namespace fe {

namespace {

constexpr int kWarps = 8;
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

template <int SAMPLING>
__device__ __forceinline__ TapSet make_taps(float xmin, float ymin, int bx, int by, int stride, int lane) {
  TapSet s;
  const bool is_col = lane < 9, is_row = lane >= 16 && lane < 25;
  const float p = is_col ? __fadd_rn(xmin, (float)lane) : __fadd_rn(ymin, (float)(is_row ? lane - 16 : 0));
  const float pb = __fsub_rn(p, 0.5f);
  const float fl = floorf(pb);
  s.fr = __fsub_rn(pb, fl);
  s.base = (int)fl;
  s.q = (SAMPLING == FE_SAMPLE_TEXTURE) ? (int)floorf(__fmaf_rn(s.fr, 256.f, 0.5f)) : 0;
  const int base0x = __shfl_sync(kFull, s.base, 0), base0y = __shfl_sync(kFull, s.base, 16);
  const int q0x = __shfl_sync(kFull, s.q, 0), q0y = __shfl_sync(kFull, s.q, 16);
  const float fr0x = __shfl_sync(kFull, s.fr, 0), fr0y = __shfl_sync(kFull, s.fr, 16);
  bool ok = true;
  if (is_col) ok = s.base == base0x + lane && (SAMPLING == FE_SAMPLE_TEXTURE ? s.q == q0x : s.fr == fr0x);
  if (is_row) ok = s.base == base0y + (lane - 16) && (SAMPLING == FE_SAMPLE_TEXTURE ? s.q == q0y : s.fr == fr0y);
  s.uniform = __all_sync(kFull, ok);
  if (SAMPLING == FE_SAMPLE_TEXTURE) {
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
  if (SAMPLING == FE_SAMPLE_TEXTURE) {
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

template <int SAMPLING, bool HORIZ>
__device__ void track_one(const LkCam& cam, fe_track_data& td, WarpSmem& sm, int lane) {
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
    if (good) {
      // previous-frame patch: image and gradients
      const int bx = (int)floorf(__fsub_rn(xmin, 0.5f)) - 1, by = (int)floorf(__fsub_rn(ymin, 0.5f)) - 1;
      __syncwarp();
      stage<kPW, kPS>(sm.img, PL.img, PL.pitch, PL.w, PL.h, bx, by, lane);
      stage<kPW, kPS>(sm.gx, PL.gx, PL.pitch, PL.w, PL.h, bx, by, lane);
      if (!HORIZ) stage<kPW, kPS>(sm.gy, PL.gy, PL.pitch, PL.w, PL.h, bx, by, lane);
      cp_async_wait_all();
      __syncwarp();
      const TapSet ts = make_taps<SAMPLING>(xmin, ymin, bx, by, kPS, lane);
      float gxp[kNE], gyp[kNE], p1[kNE];
      float sgx = 0.f, sgy = 0.f, sp = 0.f;
#pragma unroll
      for (int e = 0; e < kNE; ++e) {
        gxp[e] = gyp[e] = p1[e] = 0.f;
        const Tap t = tap_of<SAMPLING>(ts, ix[e], iy[e], bx, by, kPS);
        if (valid[e]) {
          gxp[e] = sample<SAMPLING>(sm.gx, kPS, t);
          if (!HORIZ) gyp[e] = sample<SAMPLING>(sm.gy, kPS, t);
          p1[e] = sample<SAMPLING>(sm.img, kPS, t);
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
      int wbx = INT_MIN / 2, wby = INT_MIN / 2;  // current-frame window origin (none yet)
      for (int it = 0; it < 11; ++it) {
        xmin = __fadd_rn(cx, -4.f);
        ymin = __fadd_rn(cy, -4.f);
        if (!(xmin >= 0.f && __fadd_rn(cx, 5.f) < (float)W && ymin >= 0.f && __fadd_rn(cy, 5.f) < (float)H)) good = false;
        if (!good) break;
        // taps reach texels [base0 - 1, base0 + 10]; keep the 16x16 window while it covers them
        const int nbx = (int)floorf(__fsub_rn(xmin, 0.5f)) - 1, nby = (int)floorf(__fsub_rn(ymin, 0.5f)) - 1;
        if (nbx < wbx || nbx + kPW > wbx + kCW || nby < wby || nby + kPW > wby + kCW) {
          wbx = nbx - 2;
          wby = nby - 2;
          __syncwarp();
          stage<kCW, kCS>(sm.cur, CL.img, CL.pitch, CL.w, CL.h, wbx, wby, lane);
          cp_async_wait_all();
          __syncwarp();
        }
        const TapSet tc = make_taps<SAMPLING>(xmin, ymin, wbx, wby, kCS, lane);
        float sc = 0.f;
#pragma unroll
        for (int e = 0; e < kNE; ++e) {
          const Tap t = tap_of<SAMPLING>(tc, ix[e], iy[e], wbx, wby, kCS);
          if (valid[e]) {
            p2[e] = sample<SAMPLING>(sm.cur, kCS, t);
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

template <int SAMPLING, bool HORIZ>
__global__ void __launch_bounds__(kWarps * 32, 4) lk_kernel(const __grid_constant__ LkLaunch p) {
  __shared__ WarpSmem smem[kWarps];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const LkCam* cams = p.cams ? p.cams : &p.single;
  int g = p.counter ? 0 : (int)blockIdx.x * kWarps + wid;
  for (;;) {
    if (p.counter) {
      int v = 0;
      if (lane == 0) v = atomicAdd(p.counter, 1);
      g = __shfl_sync(kFull, v, 0);
    }
    if (g >= p.total) return;  // warp-uniform
    int lo = 0, hi = p.ncams - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (cams[mid].begin <= g) lo = mid; else hi = mid - 1;
    }
    const LkCam& cam = cams[lo];
    track_one<SAMPLING, HORIZ>(cam, cam.tracks[g - cam.begin], smem[wid], lane);
    if (!p.counter) return;
  }
}

template <int SAMPLING, bool HORIZ>
int resident_blocks() {
  static int blocks = 0;
  if (!blocks) {
    int per_sm = 0, dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lk_kernel<SAMPLING, HORIZ>, kWarps * 32, 0);
    blocks = (per_sm > 0 ? per_sm : 1) * (sms > 0 ? sms : 1);
  }
  return blocks;
}

template <int SAMPLING, bool HORIZ>
cudaError_t launch(const LkLaunch& p, cudaStream_t s) {
  int blocks = (p.total + kWarps - 1) / kWarps;
  if (p.counter) blocks = min(blocks, resident_blocks<SAMPLING, HORIZ>());
  lk_kernel<SAMPLING, HORIZ><<<blocks, kWarps * 32, 0, s>>>(p);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_lk(const LkLaunch& p, cudaStream_t s) {
  if (p.total <= 0) return cudaSuccess;
  if (p.counter) {
    cudaError_t e = cudaMemsetAsync(p.counter, 0, sizeof(int), s);
    if (e != cudaSuccess) return e;
  }
  if (p.sampling == FE_SAMPLE_EXACT)
    return p.horizontal ? launch<FE_SAMPLE_EXACT, true>(p, s) : launch<FE_SAMPLE_EXACT, false>(p, s);
  return p.horizontal ? launch<FE_SAMPLE_TEXTURE, true>(p, s) : launch<FE_SAMPLE_TEXTURE, false>(p, s);
}

}  // namespace fe
