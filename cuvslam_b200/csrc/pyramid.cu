// Fused pyramid + gradient kernel.
//
// One launch ("stage") takes an input level s that is already in memory (the uint8 frame for
// s = 0, else the FP32 level s) and produces up to NL further levels and their gradients.  Each CTA
// owns a T x T core tile of the deepest produced level and the matching 2^k-times larger core tiles
// of the shallower levels.  It stages the input region (with the halo the deeper levels and the
// 7-tap derivatives need) in shared memory, computes every intermediate level in shared memory,
// and writes each level's core image, grad_x and grad_y once, coalesced.  Level l+1 therefore never
// re-reads level l from HBM inside a stage.
//
// Arithmetic follows the reference exactly:
//   gaussian_scaling_kernel (image_pyramid.cu:56-102): 25 taps visited row-major, each as an FMA
//     into the accumulator, mirror addressing -x-1 / 2n-x-1, taps outside in both x and y skipped;
//   conv_grad_x/y_kernel (convolutions.cu:74-139): 7 taps j = -3..3 as FMAs, 0 within 3 px of
//     the border.
// so every level and gradient is bit-identical to the reference.
//
// Region geometry (1-D; the same in y).  With the deepest core [X, X+T) at level s+NL:
//   level s+NL is needed on [X-3, X+T+3)                (its own gradient halo), size S_NL = T+6;
//   level s+k  is needed on [2a-2, 2b+1) given [a, b) at level s+k+1, size S_k = 2 S_{k+1} + 3.
// Mirrored taps near the image border fall inside these regions (the region always reaches the
// border it is mirrored about), so a CTA never reads outside its shared-memory tiles.
#include <cuda_runtime.h>

#include "fe_common.cuh"
#include "fe_internal.h"

namespace fe {

namespace {

// Generic stages: the deepest level's core tile is KT x KT (8 or 16, chosen by the batch autotuner).
constexpr int kThreads = 256;

__host__ __device__ constexpr int region_size(int kt, int nl, int k) {
  return k == nl ? kt + 6 : 2 * region_size(kt, nl, k + 1) + 3;
}
__host__ __device__ constexpr int smem_floats(int kt, int nl) {
  int s = 0;
  for (int k = 0; k <= nl; ++k) s += region_size(kt, nl, k) * region_size(kt, nl, k);
  return s;
}

template <typename InT>
__device__ __forceinline__ float load_px(const InT* base, int64_t pitch_bytes, int x, int y) {
  const InT* row = reinterpret_cast<const InT*>(reinterpret_cast<const char*>(base) + (int64_t)y * pitch_bytes);
  return (float)__ldg(row + x);
}

// One output of gaussian_scaling_kernel at level coordinates (x, y), reading the source level from
// a shared-memory region whose origin is (ax, ay) and row length is `stride`.
__device__ __forceinline__ float downscale_px(const float* src, int stride, int ax, int ay, int sw, int sh, int x,
                                              int y) {
  const float k1[5] = {1.f / 16.f, 4.f / 16.f, 6.f / 16.f, 4.f / 16.f, 1.f / 16.f};
  const int x0 = 2 * x - 2, y0 = 2 * y - 2;
  float acc = 0.f;
  if (x0 >= 0 && y0 >= 0 && x0 + 4 < sw && y0 + 4 < sh) {
    const float* p = src + (y0 - ay) * stride + (x0 - ax);
#pragma unroll
    for (int k = 0; k < 5; ++k)
#pragma unroll
      for (int l = 0; l < 5; ++l) acc = __fmaf_rn(k1[k] * k1[l], p[k * stride + l], acc);
    return acc;
  }
#pragma unroll
  for (int k = 0; k < 5; ++k) {
#pragma unroll
    for (int l = 0; l < 5; ++l) {
      int xc = x0 + l, yc = y0 + k;
      const bool xo = xc < 0 || xc >= sw, yo = yc < 0 || yc >= sh;
      if (xo && yo) continue;
      xc = mirror_index(xc, sw);
      yc = mirror_index(yc, sh);
      acc = __fmaf_rn(k1[k] * k1[l], src[(yc - ay) * stride + (xc - ax)], acc);
    }
  }
  return acc;
}

// Levels tail[0..n) of one camera from the complete level `src` (global), by one CTA: the source
// level is copied to shared memory (L2, bypassing L1), each tail level's image is computed there
// with the 25-tap rule and its gradients from it.  `smem` holds kTailFloats floats.
__device__ void stage_tail(const Level& src, const Level* tail, int n, float* smem) {
  float* a = smem;                              // current source level (w x h, row stride w)
  int sw = src.w, sh = src.h;
  for (int i = threadIdx.x; i < sw * sh; i += kThreads) {
    const int r = i / sw, c = i - r * sw;
    cp_async4(a + i, src.img + (size_t)r * src.pitch + c);
  }
  cp_async_wait_all();
  __syncthreads();
  for (int t = 0; t < n; ++t) {
    const Level& L = tail[t];
    float* b = a + sw * sh;                     // this level, right after its source
    for (int i = threadIdx.x; i < L.w * L.h; i += kThreads) {
      const int y = i / L.w, x = i - y * L.w;
      const float v = downscale_px(a, sw, 0, 0, sw, sh, x, y);
      b[i] = v;
      L.img[(size_t)y * L.pitch + x] = v;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < L.w * L.h; i += kThreads) {
      const int y = i / L.w, x = i - y * L.w;
      const float* p = b + i;
      float gx = 0.f, gy = 0.f;
      if (x > 2 && x < L.w - 3) {
#pragma unroll
        for (int j = 0; j < 7; ++j)
          if (j != 3) gx = __fmaf_rn(dsp_tap(j), p[j - 3], gx);
      }
      if (y > 2 && y < L.h - 3) {
#pragma unroll
        for (int j = 0; j < 7; ++j)
          if (j != 3) gy = __fmaf_rn(dsp_tap(j), p[(j - 3) * L.w], gy);
      }
      L.gx[(size_t)y * L.pitch + x] = gx;
      if (L.gy) L.gy[(size_t)y * L.pitch + x] = gy;
    }
    __syncthreads();
    // the next level's source: move this level to the front (it is smaller than its source)
    for (int i = threadIdx.x; i < L.w * L.h; i += kThreads) a[i] = b[i];  // disjoint ranges
    __syncthreads();
    sw = L.w;
    sh = L.h;
  }
}

template <typename InT, int NL, int KT>
__global__ void __launch_bounds__(kThreads) pyramid_stage_kernel(const __grid_constant__ StageBatch batch) {
  extern __shared__ float smem[];
  // camera of this CTA: last job whose tile_begin <= blockIdx.x
  int lo = 0, hi = batch.njobs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (batch.job[mid].tile_begin <= (int)blockIdx.x) lo = mid; else hi = mid - 1;
  }
  const StageJob& job = batch.job[lo];
  const int t = (int)blockIdx.x - job.tile_begin;
  const int X = (t % job.tiles_x) * KT, Y = (t / job.tiles_x) * KT;

  int a[NL + 1], S[NL + 1], off[NL + 1];
  a[NL] = X - 3;
  int ay[NL + 1];
  ay[NL] = Y - 3;
#pragma unroll
  for (int k = NL - 1; k >= 0; --k) {
    a[k] = 2 * a[k + 1] - 2;
    ay[k] = 2 * ay[k + 1] - 2;
  }
  int o = 0;
#pragma unroll
  for (int k = 0; k <= NL; ++k) {
    S[k] = region_size(KT, NL, k);
    off[k] = o;
    o += S[k] * S[k];
  }

  // 1. stage the input region (FP32 sources as asynchronous copies, all in flight at once), scaled
  //    by job.scale (the first stage of a scaled build; 1 otherwise)
  {
    const int w = job.src_w, h = job.src_h;
    const InT* src = static_cast<const InT*>(job.src);
    float* dst = smem + off[0];
    for (int i = threadIdx.x; i < S[0] * S[0]; i += kThreads) {
      const int r = i / S[0], c = i - r * S[0];
      const int gx = a[0] + c, gy = ay[0] + r;
      const bool in = gx >= 0 && gy >= 0 && gx < w && gy < h;
      if constexpr (sizeof(InT) == 4) {
        if (in) {
          cp_async4(dst + i, reinterpret_cast<const float*>(reinterpret_cast<const char*>(src) +
                                                            (int64_t)gy * job.src_pitch_bytes) + gx);
        } else {
          dst[i] = 0.f;
        }
      } else {
        dst[i] = in ? load_px(src, job.src_pitch_bytes, gx, gy) : 0.f;
      }
    }
    if constexpr (sizeof(InT) == 4) cp_async_wait_all();
    __syncthreads();
    if (job.scale != 1.f) {
      for (int i = threadIdx.x; i < S[0] * S[0]; i += kThreads) dst[i] = __fmul_rn(dst[i], job.scale);
      __syncthreads();
    }
  }

  // 2. deeper levels inside shared memory
#pragma unroll
  for (int k = 1; k <= NL; ++k) {
    const int sw = job.out[k - 1].w, sh = job.out[k - 1].h;
    const int w = job.out[k].w, h = job.out[k].h;
    const float* src = smem + off[k - 1];
    float* dst = smem + off[k];
    for (int i = threadIdx.x; i < S[k] * S[k]; i += kThreads) {
      const int r = i / S[k], c = i - r * S[k];
      const int gx = a[k] + c, gy = ay[k] + r;
      if (gx >= 0 && gy >= 0 && gx < w && gy < h)
        dst[i] = downscale_px(src, S[k - 1], a[k - 1], ay[k - 1], sw, sh, gx, gy);
    }
    __syncthreads();
  }

  // 3. core outputs: image, grad_x, grad_y
#pragma unroll
  for (int k = (job.write_level0 ? 0 : 1); k <= NL; ++k) {
    const Level& L = job.out[k];
    const int C = KT << (NL - k);
    const int cx0 = X << (NL - k), cy0 = Y << (NL - k);
    const float* reg = smem + off[k];
    for (int i = threadIdx.x; i < C * C; i += kThreads) {
      const int r = i / C, c = i - r * C;
      const int x = cx0 + c, y = cy0 + r;
      if (x >= L.w || y >= L.h) continue;
      const float* p = reg + (y - ay[k]) * S[k] + (x - a[k]);
      float sx = 0.f, sy = 0.f;
      if (x > 2 && x < L.w - 3) {
#pragma unroll
        for (int j = 0; j < 7; ++j)
          if (j != 3) sx = __fmaf_rn(dsp_tap(j), p[j - 3], sx);
      }
      if (y > 2 && y < L.h - 3) {
#pragma unroll
        for (int j = 0; j < 7; ++j)
          if (j != 3) sy = __fmaf_rn(dsp_tap(j), p[(j - 3) * S[k]], sy);
      }
      const int64_t o2 = (int64_t)y * L.pitch + x;
      L.img[o2] = p[0];
      L.gx[o2] = sx;
      if (L.gy) L.gy[o2] = sy;
    }
  }

  // 4. tail: the last CTA of the job computes the remaining (small) levels from the complete
  //    deepest level, in shared memory (threadfence + counter: every CTA's stores precede its count)
  if (job.tail_levels > 0) {
    __shared__ int last;
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      last = atomicAdd(job.done, 1) == job.tiles_x * job.tiles_y - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    stage_tail(job.out[NL], job.tail, job.tail_levels, smem);
    if (threadIdx.x == 0) *job.done = 0;
  }
}

// ---------------------------------------------------------------- levels 0-2 from the uint8 frame
//
// The first stage dominates the pyramid's HBM traffic (it writes ~98% of the bytes), so it has its
// own kernel.  A CTA owns a 32x32 level-2 core tile (128x128 at level 0) and
//   1. stages its 176x163 uint8 tile with one TMA copy (zero fill outside the frame), or with plain
//      loads when the frame's base/pitch are not 16-byte aligned, and applies the optional box
//      prefilter to it (integer arithmetic, exact);
//   2. computes level 1 on its 79x79 region as column strips with a sliding 5-row window of
//      horizontal 5-tap sums, in integers;
//   3. computes level 2 on its 38x38 region the same way from level 1, in FP32;
//   4. writes the three core tiles (image, grad_x, grad_y) with 16-byte stores.
// Levels 1 and 2 are exact in any summation order (all partial sums are multiples of 2^-16 below
// 2^8), so the separable sums equal gaussian_scaling_kernel's 25-tap FMA chain bit for bit; only the
// four image-corner pixels, where the reference skips the taps outside in both x and y, are redone
// with the 25-tap rule.
namespace l012 {

constexpr int kT2 = 32;
constexpr int kThreads = 512;
constexpr int kS0W = 176, kS0H = 163;  // uint8 tile: cols [4X2-32, 4X2+144), rows [4Y2-19, 4Y2+144)
constexpr int kS1 = 79, kS1S = 80;     // level 1: [2X2-8, 2X2+71) in x and y
constexpr int kS2 = 38, kS2S = 40;     // level 2: rows [Y2-3, Y2+35); columns stored from X2-4
constexpr int kB0Bytes = kS0W * kS0H;
constexpr int kOffB1 = (kB0Bytes + 127) / 128 * 128;
constexpr int kOffB2 = kOffB1 + kS1 * kS1S * 4;
constexpr int kOffBar = kOffB2 + kS2 * kS2S * 4;
constexpr int kSmem = kOffBar + 64;
// with the box prefilter: the prefiltered tile after the rest
constexpr int kOffBox = (kSmem + 127) / 128 * 128;
constexpr int kSmemBox = kOffBox + kB0Bytes;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Bounded wait on an mbarrier phase: false when `limit` polls all found it incomplete (the caller
// reports it and gives up).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase, int limit) {
  for (int i = 0; i < limit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(phase)
        : "memory");
    if (done) return true;
  }
  return false;
}

// Bytes k and k+1 of a word as exact floats: 0x4B0000bb is 2^23 + b, then subtract 2^23.
__device__ __forceinline__ float2 bytes_to_float2(uint32_t wd, int k) {
  const float lo = __uint_as_float(__byte_perm(wd, 0x4B000000u, 0x7540u + k));
  const float hi = __uint_as_float(__byte_perm(wd, 0x4B000000u, 0x7540u + k + 1));
  return __fadd2_rn(make_float2(lo, hi), make_float2(-8388608.f, -8388608.f));
}

// 25-tap value with the reference's corner rule (taps outside in x and y skipped), uint8 source.
__device__ float corner_l1(const uint8_t* B0, int a0x, int a0y, int w0, int h0, int x1, int y1) {
  int acc = 0;
  for (int k = 0; k < 5; ++k)
    for (int l = 0; l < 5; ++l) {
      const int xc = 2 * x1 - 2 + l, yc = 2 * y1 - 2 + k;
      if ((xc < 0 || xc >= w0) && (yc < 0 || yc >= h0)) continue;
      const int wk = k == 2 ? 6 : (k & 1 ? 4 : 1), wl = l == 2 ? 6 : (l & 1 ? 4 : 1);
      acc += wk * wl * (int)B0[(mirror_index(yc, h0) - a0y) * kS0W + (mirror_index(xc, w0) - a0x)];
    }
  return (float)acc * (1.f / 256.f);
}

// Deeper levels (3 and below) inside the same launch.  Every tile CTA also writes its 16x16 core of
// level 3's image (its sources lie in the tile's level-2 region).  The launch's CTAs take work items
// from an atomic queue: each camera's tiles, then (placed after the next camera's tiles, so that
// their inputs are usually complete when they are taken) its deeper-level items:
//   band items of phase d (d = level 3, then level 4 when needed): level d's gradients and level
//     d+1's image for a band of rows, from level d's rows staged in shared memory;
//   one rest item: the remaining levels from the first one that fits in shared memory, staged once,
//     each further level computed there.
// An item waits (bounded) until the items it reads from are counted complete: tiles for phase 3,
// phase-3 bands for phase 4, the last banded phase (or the tiles) for the rest.  Items are taken in
// queue order and only wait on earlier items, which are running or done, so the waits end.  Pixels
// follow the reference's rules (25-tap decimation with mirror and corner skip, 7-tap derivatives),
// so every level is bit-identical to the reference's.
constexpr int kDeepFloats = (kOffBar / 4) & ~3;

// Rows [lo, lo + rows) of level L into sm (row stride `stride` floats, a multiple of 4), through L2.
__device__ __forceinline__ void stage_rows(const Level& L, int lo, int rows, int stride, float* sm) {
  const int q4 = L.w >> 2, rem = L.w & 3;
  for (int i = threadIdx.x; i < rows * q4; i += kThreads) {
    const int r = i / q4, c = (i - r * q4) * 4;
    const float* g = L.img + (size_t)(lo + r) * L.pitch + c;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(sm + r * stride + c)), "l"(g) : "memory");
  }
  if (rem)
    for (int i = threadIdx.x; i < rows * rem; i += kThreads) {
      const int r = i / rem, c = (q4 << 2) + (i - r * rem);
      sm[r * stride + c] = __ldcg(L.img + (size_t)(lo + r) * L.pitch + c);
    }
  cp_async_wait_all();
  __syncthreads();
}

// Gradients of rows [y0, y1) of level D whose image rows [lo, ...) are in sm (row stride `stride`).
__device__ __forceinline__ void smem_gradients(const Level& D, const float* a, int stride, int lo, int y0, int y1) {
  const int w = D.w, h = D.h;
  for (int i = threadIdx.x; i < (y1 - y0) * w; i += kThreads) {
    const int y = y0 + i / w, x = i - (i / w) * w;
    const float* p = a + (y - lo) * stride + x;
    float gx = 0.f, gy = 0.f;
    if (x > 2 && x < w - 3) {
#pragma unroll
      for (int j = 0; j < 7; ++j)
        if (j != 3) gx = __fmaf_rn(dsp_tap(j), p[j - 3], gx);
    }
    if (y > 2 && y < h - 3) {
#pragma unroll
      for (int j = 0; j < 7; ++j)
        if (j != 3) gy = __fmaf_rn(dsp_tap(j), p[(j - 3) * stride], gy);
    }
    D.gx[(size_t)y * D.pitch + x] = gx;
    if (D.gy) D.gy[(size_t)y * D.pitch + x] = gy;
  }
}

// Band item: level S's gradients on rows [2 r0, 2 r1) and level N's image on rows [r0, r1).
__device__ void band_item(const Level& S, const Level& N, int r0, int nrows, float* sm) {
  const int r1 = min(N.h, r0 + nrows);
  const int ss = (S.w + 3) & ~3;
  const int lo = max(0, 2 * r0 - 3), hi = min(S.h - 1, 2 * r1 + 2);
  stage_rows(S, lo, hi - lo + 1, ss, sm);
  smem_gradients(S, sm, ss, lo, min(S.h, 2 * r0), min(S.h, 2 * r1));
  for (int i = threadIdx.x; i < (r1 - r0) * N.w; i += kThreads) {
    const int y = r0 + i / N.w, x = i - (i / N.w) * N.w;
    N.img[(size_t)y * N.pitch + x] = downscale_px(sm, ss, 0, lo, S.w, S.h, x, y);
  }
}

// Rest item: levels tail[0..n): tail[0]'s image is complete; its gradients and every further level.
__device__ void rest_item(const Level* tail, int n, float* sm) {
  const int s0 = (tail[0].w + 3) & ~3;
  stage_rows(tail[0], 0, tail[0].h, s0, sm);
  const float* a = sm;
  int as = s0;
  float* b = sm + s0 * tail[0].h;
  for (int t = 0; t < n; ++t) {
    const Level& D = tail[t];
    if (t > 0) {
      const Level& S = tail[t - 1];
      for (int i = threadIdx.x; i < D.w * D.h; i += kThreads) {
        const int y = i / D.w, x = i - y * D.w;
        const float v = downscale_px(a, as, 0, 0, S.w, S.h, x, y);
        b[i] = v;
        D.img[(size_t)y * D.pitch + x] = v;
      }
      __syncthreads();
      a = b;
      as = D.w;
      b += D.w * D.h;
    }
    smem_gradients(D, a, as, 0, 0, D.h);
  }
}

// Thread 0 waits (at most batch.wait_limit polls) until *ctr >= target; false (and status bit 1)
// when the wait ran out.
__device__ bool wait_count(const StageBatch& batch, int* ctr, int target) {
  __shared__ int s_ok;
  if (threadIdx.x == 0) {
    int ok = 0;
    for (int i = 0; i < batch.wait_limit; ++i) {
      if (*reinterpret_cast<volatile int*>(ctr) >= target) {
        ok = 1;
        break;
      }
      __nanosleep(64);
    }
    if (!ok && batch.status) atomicOr(batch.status, 2);
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// Deeper-level item idx of job J.  J.done: [0] tiles finished, [1] phase-3 bands, [2] phase-4
// bands; the launch's last CTA returns them to zero for the next launch (not the rest item: if one
// of its waits gave up, tiles and bands may still be counting).
__device__ void deep_item(const StageBatch& batch, const StageJob& J, int idx, float* sm) {
  int* ctr = J.done;
  const int ntiles = J.tiles_x * J.tiles_y;
  const int nb0 = J.deep_bands[0], nb1 = J.deep_bands[1];
  if (idx < nb0 + nb1) {
    const int ph = idx < nb0 ? 0 : 1, b = ph ? idx - nb0 : idx;
    if (wait_count(batch, ph ? ctr + 1 : ctr, ph ? nb0 : ntiles))
      band_item(J.tail[ph], J.tail[ph + 1], b * J.deep_band_rows[ph], J.deep_band_rows[ph], sm);
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      atomicAdd(ctr + 1 + ph, 1);
    }
  } else {
    const int r = J.deep_rest;
    if (wait_count(batch, r == 0 ? ctr : ctr + r, r == 0 ? ntiles : J.deep_bands[r - 1]))
      rest_item(J.tail + r, J.tail_levels - r, sm);
  }
}

// The box prefilter of the reference (CudaBoxPrefilter::prefilter, box_prefilter.cpp:31-38: a
// [1 2 1]/4 pass along x, then along y truncated to an integer, then the frame's one-pixel border ring
// copied from the input) on the staged uint8 tile: on integer input every partial sum is exact, so
// an interior pixel is (sum of [1 2 1] x [1 2 1] weighted bytes) >> 4.  Four columns per thread
// item, as packed 16-bit lanes (sums stay below 2^12); rows 1..kS0H-2 and every column are written
// (the tile's outermost rows and columns, never read, keep their input bytes).  Pixels on the
// frame's border ring take the input byte.
__device__ void box3_tile(const uint8_t* raw, uint8_t* out, int a0x, int a0y, int w0, int h0) {
  constexpr int kWords = kS0W / 4;            // 44 four-column groups per row
  constexpr int kBand = 15;                   // rows per thread item
  constexpr int kBands = (kS0H - 2 + kBand - 1) / kBand;
  const uint32_t* rw = reinterpret_cast<const uint32_t*>(raw);
  for (int it = threadIdx.x; it < kWords * kBands; it += kThreads) {
    const int c4 = it % kWords, band = it / kWords;
    const int r0 = 1 + band * kBand, r1 = min(kS0H - 1, r0 + kBand);
    // horizontal [1 2 1] of four columns as two words of 16-bit lanes (columns c, c+1 | c+2, c+3)
    auto hsum = [&](int r, uint32_t& lo, uint32_t& hi) {
      const uint32_t w = rw[r * kWords + c4];
      const uint32_t wl = c4 > 0 ? rw[r * kWords + c4 - 1] : 0u;
      const uint32_t wr = c4 + 1 < kWords ? rw[r * kWords + c4 + 1] : 0u;
      // zero-extended byte pairs (selector nibbles 4-7 pick the second operand; masks clear the rest)
      const uint32_t cl = __byte_perm(w, 0u, 0x4140), ch = __byte_perm(w, 0u, 0x4342);  // c, c+1 | c+2, c+3
      const uint32_t mid = __byte_perm(w, 0u, 0x4241);                                   // c+1, c+2
      const uint32_t left = __byte_perm(wl, w, 0x4443) & 0x00ff00ffu;                    // c-1, c
      const uint32_t right = __byte_perm(w, wr, 0x4443) & 0x00ff00ffu;                   // c+3, c+4
      lo = left + 2u * cl + mid;
      hi = mid + 2u * ch + right;
    };
    uint32_t a_lo, a_hi, b_lo, b_hi, c_lo, c_hi;
    hsum(r0 - 1, a_lo, a_hi);
    hsum(r0, b_lo, b_hi);
    for (int r = r0; r < r1; ++r) {
      hsum(r + 1, c_lo, c_hi);
      const uint32_t vlo = ((a_lo + 2u * b_lo + c_lo) >> 4) & 0x0fff0fffu;
      const uint32_t vhi = ((a_hi + 2u * b_hi + c_hi) >> 4) & 0x0fff0fffu;
      reinterpret_cast<uint32_t*>(out)[r * kWords + c4] = __byte_perm(vlo, vhi, 0x6420);
      a_lo = b_lo; a_hi = b_hi;
      b_lo = c_lo; b_hi = c_hi;
    }
  }
  // rows 0 and kS0H-1 of the tile: input bytes
  for (int i = threadIdx.x; i < 2 * kS0W; i += kThreads) {
    const int r = i < kS0W ? 0 : kS0H - 1, c = i < kS0W ? i : i - kS0W;
    out[r * kS0W + c] = raw[r * kS0W + c];
  }
  __syncthreads();
  // the frame's border ring: input bytes (rows 0 and h0-1, columns 0 and w0-1 inside the tile)
  for (int i = threadIdx.x; i < 2 * (kS0W + kS0H); i += kThreads) {
    int r, c;
    if (i < 2 * kS0W) {
      r = (i < kS0W ? 0 : h0 - 1) - a0y;
      c = i % kS0W;
    } else {
      const int k = i - 2 * kS0W;
      c = (k < kS0H ? 0 : w0 - 1) - a0x;
      r = k % kS0H;
    }
    if (r >= 0 && r < kS0H && c >= 0 && c < kS0W) out[r * kS0W + c] = raw[r * kS0W + c];
  }
}

// Tile t of job: levels 0-2, and when the launch computes the deeper levels, level 3's image core
// (after which the tile counts itself complete in job.done[0]).
__device__ __forceinline__ void l012_tile(const StageBatch& batch, const StageJob& job, int t, unsigned char* sm) {
  uint8_t* B0 = sm;
  float* B1 = reinterpret_cast<float*>(sm + kOffB1);
  float* B2 = reinterpret_cast<float*>(sm + kOffB2);
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + kOffBar);
  const int tid = threadIdx.x;
  const int X2 = (t % job.tiles_x) * kT2, Y2 = (t / job.tiles_x) * kT2;
  const Level& L0 = job.out[0];
  const Level& L1 = job.out[1];
  const Level& L2 = job.out[2];
  const int w0 = L0.w, h0 = L0.h, w1 = L1.w, h1 = L1.h, w2 = L2.w, h2 = L2.h;
  const int a0x = 4 * X2 - 32, a0y = 4 * Y2 - 19;
  const int a1x = 2 * X2 - 8, a1y = 2 * Y2 - 8;
  const int a2x = X2 - 4, a2y = Y2 - 3;  // level-2 storage origin (column X2-4 is never computed)

  // 1. the uint8 tile
  if (job.use_tma) {
    if (tid == 0) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)));
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (tid == 0) {
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(kB0Bytes)
                   : "memory");
      asm volatile(
          "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
          "[%4];" ::"r"(smem_u32(B0)),
          "l"(reinterpret_cast<uint64_t>(&job.tmap)), "r"(a0x), "r"(a0y), "r"(smem_u32(bar))
          : "memory");
    }
    const bool ok = mbar_wait(bar, 0, batch.wait_limit);
    if (__syncthreads_or(!ok)) {
      if (tid == 0 && batch.status) atomicOr(batch.status, 1);
      // the copy may still land: wait once more, with the full bound whatever the launch's limit, so
      // no write targets a retired CTA
      mbar_wait(bar, 0, kDefaultWaitLimit);
      if (job.tail_levels > 0 && tid == 0) atomicAdd(job.done, 1);  // still counted (its level 3 is not written)
      return;
    }
  } else {
    const uint8_t* src = static_cast<const uint8_t*>(job.src);
    for (int i = tid; i < kS0H * kS0W; i += kThreads) {
      const int r = i / kS0W, c = i - r * kS0W;
      const int gx = a0x + c, gy = a0y + r;
      B0[i] = (gx >= 0 && gy >= 0 && gx < w0 && gy < h0) ? __ldg(src + (int64_t)gy * job.src_pitch_bytes + gx) : 0;
    }
  }
  __syncthreads();
  if (job.box3) {
    uint8_t* F = sm + kOffBox;
    box3_tile(B0, F, a0x, a0y, w0, h0);
    B0 = F;
    __syncthreads();
  }

  // 2. level 1 (integer sums: exact in any order): a thread takes a pair of columns (c, c + 1) and a
  //    band of 7 rows, sliding the 5-row window of horizontal sums down the band.  Away from the
  //    image's edges the taps of both columns are bytes 4 pp + 14 .. 4 pp + 20 of a staged row: three
  //    words, one byte permute and two dp4a with the weights (1, 4, 6, 4) plus the fifth tap; near an
  //    edge each column takes its mirrored taps one by one.
  if (tid < 40 * 12) {
    const int pp = tid % 40, band = tid / 40;
    const int c = 2 * pp;
    const int ys = max(a1y + band * 7, 0), ye = min(a1y + min(band * 7 + 7, kS1), h1);
    const int x1 = a1x + c;
    if (ys < ye) {
      if (2 * x1 - 2 >= 0 && 2 * x1 + 4 < w0 && c + 1 < kS1 && 2 * ys - 2 >= 0 && 2 * ye < h0) {
        const uint8_t* p = B0 + (2 * ys - 2 - a0y) * kS0W + 4 * pp + 12;
        auto H2 = [&](const uint8_t* q, int& ha, int& hb) {
          const uint32_t wa = *reinterpret_cast<const uint32_t*>(q);
          const uint32_t wb = *reinterpret_cast<const uint32_t*>(q + 4);
          const uint32_t wc = *reinterpret_cast<const uint32_t*>(q + 8);
          ha = (int)__dp4a(__byte_perm(wa, wb, 0x5432u), 0x04060401u, (wb >> 16) & 0xffu);
          hb = (int)__dp4a(wb, 0x04060401u, wc & 0xffu);
        };
        int a0_, b0_, a1_, b1_, a2_, b2_, a3_, b3_, a4_, b4_;
        H2(p, a0_, b0_);
        H2(p + kS0W, a1_, b1_);
        H2(p + 2 * kS0W, a2_, b2_);
        p += 3 * kS0W;
        for (int y = ys;;) {
          H2(p, a3_, b3_);
          H2(p + kS0W, a4_, b4_);
          const int Sa = a0_ + a4_ + 4 * (a1_ + a3_) + 6 * a2_;
          const int Sb = b0_ + b4_ + 4 * (b1_ + b3_) + 6 * b2_;
          *reinterpret_cast<float2*>(B1 + (y - a1y) * kS1S + c) =
              make_float2((float)Sa * (1.f / 256.f), (float)Sb * (1.f / 256.f));
          if (++y >= ye) break;
          a0_ = a2_;
          b0_ = b2_;
          a1_ = a3_;
          b1_ = b3_;
          a2_ = a4_;
          b2_ = b4_;
          p += 2 * kS0W;
        }
      } else {
#pragma unroll 1
        for (int k = 0; k < 2; ++k) {
          const int cc = c + k, xx = x1 + k;
          if (cc >= kS1 || xx < 0 || xx >= w1) continue;
          int col[5];
#pragma unroll
          for (int l = 0; l < 5; ++l) col[l] = mirror_index(2 * xx - 2 + l, w0) - a0x;
          auto H = [&](int r) {
            const uint8_t* q = B0 + (mirror_index(r, h0) - a0y) * kS0W;
            return (int)q[col[0]] + (int)q[col[4]] + 4 * ((int)q[col[1]] + (int)q[col[3]]) + 6 * (int)q[col[2]];
          };
          int h0_ = H(2 * ys - 2), h1_ = H(2 * ys - 1), h2_ = H(2 * ys), h3_ = H(2 * ys + 1), h4_ = H(2 * ys + 2);
          for (int y = ys;;) {
            const int S = h0_ + h4_ + 4 * (h1_ + h3_) + 6 * h2_;
            B1[(y - a1y) * kS1S + cc] = (float)S * (1.f / 256.f);
            if (++y >= ye) break;
            h0_ = h2_;
            h1_ = h3_;
            h2_ = h4_;
            h3_ = H(2 * y + 1);
            h4_ = H(2 * y + 2);
          }
        }
      }
    }
  }
  __syncthreads();
  if (tid < 4) {
    const int x1 = (tid & 1) ? w1 - 1 : 0, y1 = (tid & 2) ? h1 - 1 : 0;
    if (x1 >= a1x && x1 < a1x + kS1 && y1 >= a1y && y1 < a1y + kS1)
      B1[(y1 - a1y) * kS1S + (x1 - a1x)] = corner_l1(B0, a0x, a0y, w0, h0, x1, y1);
  }
  __syncthreads();

  // 3. level 2 from level 1, same scheme in FP32 (exact: level 1 holds multiples of 1/256 below 256
  //    and every partial sum fits FP32's 24 bits): a pair of columns and a band of 3 rows per thread;
  //    away from the edges both columns' taps are the level-1 values 4 pp .. 4 pp + 6 of a row (two
  //    16-byte loads)
  if (tid < 19 * 13) {
    const int pp = tid % 19, band = tid / 19;
    const int c = 2 * pp;
    const int x2 = X2 - 3 + c;
    const int ys = max(a2y + band * 3, 0), ye = min(a2y + min(band * 3 + 3, kS2), h2);
    if (ys < ye) {
      if (2 * x2 - 2 >= 0 && 2 * x2 + 4 < w1 && 2 * ys - 2 >= 0 && 2 * ye < h1) {
        const float* p = B1 + (2 * ys - 2 - a1y) * kS1S + 4 * pp;
        auto H2 = [&](const float* q, float& ha, float& hb) {
          const float4 u = *reinterpret_cast<const float4*>(q);
          const float4 v = *reinterpret_cast<const float4*>(q + 4);
          ha = (u.x + v.x) + 4.f * (u.y + u.w) + 6.f * u.z;
          hb = (u.z + v.z) + 4.f * (u.w + v.y) + 6.f * v.x;
        };
        float a0_, b0_, a1_, b1_, a2_, b2_, a3_, b3_, a4_, b4_;
        H2(p, a0_, b0_);
        H2(p + kS1S, a1_, b1_);
        H2(p + 2 * kS1S, a2_, b2_);
        p += 3 * kS1S;
        for (int y = ys;;) {
          H2(p, a3_, b3_);
          H2(p + kS1S, a4_, b4_);
          float* o = B2 + (y - a2y) * kS2S + (x2 - a2x);
          o[0] = ((a0_ + a4_) + 4.f * (a1_ + a3_) + 6.f * a2_) * (1.f / 256.f);
          o[1] = ((b0_ + b4_) + 4.f * (b1_ + b3_) + 6.f * b2_) * (1.f / 256.f);
          if (++y >= ye) break;
          a0_ = a2_;
          b0_ = b2_;
          a1_ = a3_;
          b1_ = b3_;
          a2_ = a4_;
          b2_ = b4_;
          p += 2 * kS1S;
        }
      } else {
#pragma unroll 1
        for (int k = 0; k < 2; ++k) {
          const int xx = x2 + k;
          if (xx < 0 || xx >= w2) continue;
          int col[5];
#pragma unroll
          for (int l = 0; l < 5; ++l) col[l] = mirror_index(2 * xx - 2 + l, w1) - a1x;
          auto H = [&](int r) {
            const float* q = B1 + (mirror_index(r, h1) - a1y) * kS1S;
            return (q[col[0]] + q[col[4]]) + 4.f * (q[col[1]] + q[col[3]]) + 6.f * q[col[2]];
          };
          float h0_ = H(2 * ys - 2), h1_ = H(2 * ys - 1), h2_ = H(2 * ys), h3_ = H(2 * ys + 1), h4_ = H(2 * ys + 2);
          for (int y = ys;;) {
            const float S = (h0_ + h4_) + 4.f * (h1_ + h3_) + 6.f * h2_;
            B2[(y - a2y) * kS2S + (xx - a2x)] = S * (1.f / 256.f);
            if (++y >= ye) break;
            h0_ = h2_;
            h1_ = h3_;
            h2_ = h4_;
            h3_ = H(2 * y + 1);
            h4_ = H(2 * y + 2);
          }
        }
      }
    }
  }
  __syncthreads();
  if (tid < 4) {
    const int x2 = (tid & 1) ? w2 - 1 : 0, y2 = (tid & 2) ? h2 - 1 : 0;
    if (x2 >= X2 - 3 && x2 < X2 + 35 && y2 >= a2y && y2 < a2y + kS2)
      B2[(y2 - a2y) * kS2S + (x2 - a2x)] = downscale_px(B1, kS1S, a1x, a1y, w1, h1, x2, y2);
  }
  __syncthreads();
  // level 3's image on this tile's 16x16 core (its sources [X2-2, X2+34) lie in the level-2 region),
  // when the job's last CTA computes the deeper levels
  if (job.tail_levels > 0) {
    if (tid < 256) {
      const Level& L3 = job.tail[0];
      const int x3 = (X2 >> 1) + (tid & 15), y3 = (Y2 >> 1) + (tid >> 4);
      if (x3 < L3.w && y3 < L3.h)
        L3.img[(size_t)y3 * L3.pitch + x3] = downscale_px(B2, kS2S, a2x, a2y, w2, h2, x3, y3);
    }
    // the deeper-level items read only level 3's image: count the tile now, while its level 0-2
    // stores (issued below) are not yet outstanding, so the fence has only these writes to wait for
    __syncthreads();
    if (tid == 0) {
      __threadfence();
      atomicAdd(job.done, 1);
    }
  }

  // 4. core outputs
  // level 0: 128x128 from the uint8 tile.  Bytes become floats exactly as (2^23 + b) - 2^23 (a byte
  // permute into the mantissa, then one packed subtract per pair); the 7-tap derivatives of pixel
  // pairs run as packed FP32x2 FMAs, each lane rounding exactly as the scalar FMA chain.
  // (a) image and grad_y: a thread takes a pixel pair's column over a strip of 16 rows and slides the
  //     derivative's 7-row window down it in registers, so each byte is converted once per strip.
  {
    const int pc = tid & 63, strip = tid >> 6;  // 64 pairs x 8 strips of 16 rows
    const int x = 4 * X2 + 2 * pc, y0 = 4 * Y2 + 16 * strip;
    if (x < w0 && y0 < h0) {
      const uint8_t* colp = B0 + (y0 - a0y - 3) * kS0W + (x - a0x);  // rows y0-3 .. y0+18
      auto pair = [&](int k) {
        return bytes_to_float2((uint32_t)*reinterpret_cast<const uint16_t*>(colp + k * kS0W), 0);
      };
      const bool two = x + 1 < w0;
      float2 win[7];
#pragma unroll
      for (int k = 0; k < 6; ++k) win[k] = pair(k);
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        win[6] = pair(i + 6);
        const int y = y0 + i;
        if (y < h0) {
          float2 gy = make_float2(0.f, 0.f);
#pragma unroll
          for (int j = 0; j < 7; ++j) {
            if (j == 3) continue;
            gy = __ffma2_rn(make_float2(dsp_tap(j), dsp_tap(j)), win[j], gy);
          }
          if (!(y > 2 && y < h0 - 3)) gy = make_float2(0.f, 0.f);
          const int64_t o = (int64_t)y * L0.pitch + x;
          if (two) {
            *reinterpret_cast<float2*>(L0.img + o) = win[3];
            *reinterpret_cast<float2*>(L0.gy + o) = gy;
          } else {
            L0.img[o] = win[3].x;
            L0.gy[o] = gy.x;
          }
        }
#pragma unroll
        for (int k = 0; k < 6; ++k) win[k] = win[k + 1];
      }
    }
  }
  // (b) grad_x: a thread takes four pixels of a row and their horizontal neighbours x-4 .. x+7.
#pragma unroll 1
  for (int q = tid; q < 128 * 32; q += kThreads) {
    const int y = 4 * Y2 + (q >> 5), x = 4 * X2 + (q & 31) * 4;
    if (y >= h0 || x >= w0) continue;
    const uint8_t* p = B0 + (y - a0y) * kS0W + (x - a0x);
    const uint32_t wl = *reinterpret_cast<const uint32_t*>(p - 4);
    const uint32_t wm = *reinterpret_cast<const uint32_t*>(p);
    const uint32_t wr = *reinterpret_cast<const uint32_t*>(p + 4);
    const float2 v[6] = {bytes_to_float2(wl, 0), bytes_to_float2(wl, 2), bytes_to_float2(wm, 0),
                         bytes_to_float2(wm, 2), bytes_to_float2(wr, 0), bytes_to_float2(wr, 2)};
    // pixel x+i needs v at flat indices 1+i+j (j = 0..6); pairs (i, i+1) for i = 0, 2
    auto hv = [&](int f) { return (f & 1) ? make_float2(v[f >> 1].y, v[(f >> 1) + 1].x) : v[f >> 1]; };
    float2 gx2[2];
#pragma unroll
    for (int pp = 0; pp < 2; ++pp) {
      float2 sx = make_float2(0.f, 0.f);
#pragma unroll
      for (int j = 0; j < 7; ++j) {
        if (j == 3) continue;
        sx = __ffma2_rn(make_float2(dsp_tap(j), dsp_tap(j)), hv(1 + 2 * pp + j), sx);
      }
      gx2[pp] = sx;
    }
    float gx[4] = {gx2[0].x, gx2[0].y, gx2[1].x, gx2[1].y};
#pragma unroll
    for (int i = 0; i < 4; ++i)
      if (!(x + i > 2 && x + i < w0 - 3)) gx[i] = 0.f;
    const int64_t o = (int64_t)y * L0.pitch + x;
    if (x + 3 < w0) {
      *reinterpret_cast<float4*>(L0.gx + o) = make_float4(gx[0], gx[1], gx[2], gx[3]);
    } else {
      for (int i = 0; i < 4 && x + i < w0; ++i) L0.gx[o + i] = gx[i];
    }
  }
  // levels 1 and 2 from their shared-memory tiles
#pragma unroll 1
  for (int q = tid; q < 64 * 16 + 32 * 8; q += kThreads) {
    const bool lev1 = q < 64 * 16;
    const int qq = lev1 ? q : q - 64 * 16;
    const Level& L = lev1 ? L1 : L2;
    const int qpr = lev1 ? 16 : 8;
    const int y = (lev1 ? 2 * Y2 : Y2) + qq / qpr, x = (lev1 ? 2 * X2 : X2) + (qq % qpr) * 4;
    if (y >= L.h || x >= L.w) continue;
    const float* T = lev1 ? B1 : B2;
    const int stride = lev1 ? kS1S : kS2S;
    const int r = y - (lev1 ? a1y : a2y), c = x - (lev1 ? a1x : a2x);
    float v[12];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const float4 f = *reinterpret_cast<const float4*>(T + r * stride + c - 4 + 4 * k);
      v[4 * k] = f.x;
      v[4 * k + 1] = f.y;
      v[4 * k + 2] = f.z;
      v[4 * k + 3] = f.w;
    }
    // pixel pairs (x, x+1), (x+2, x+3): packed FP32x2 FMA chains, vertical taps as 16-byte loads
    float2 sx[2] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
    float2 sy[2] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
#pragma unroll
    for (int j = 0; j < 7; ++j) {
      if (j == 3) continue;
      const float2 d = make_float2(dsp_tap(j), dsp_tap(j));
      const float4 cv = *reinterpret_cast<const float4*>(T + (r - 3 + j) * stride + c);
      sx[0] = __ffma2_rn(d, make_float2(v[1 + j], v[2 + j]), sx[0]);
      sx[1] = __ffma2_rn(d, make_float2(v[3 + j], v[4 + j]), sx[1]);
      sy[0] = __ffma2_rn(d, make_float2(cv.x, cv.y), sy[0]);
      sy[1] = __ffma2_rn(d, make_float2(cv.z, cv.w), sy[1]);
    }
    float gx[4] = {sx[0].x, sx[0].y, sx[1].x, sx[1].y};
    float gy[4] = {sy[0].x, sy[0].y, sy[1].x, sy[1].y};
    const bool vin = y > 2 && y < L.h - 3;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      if (!(x + i > 2 && x + i < L.w - 3)) gx[i] = 0.f;
      if (!vin) gy[i] = 0.f;
    }
    const int64_t o = (int64_t)y * L.pitch + x;
    if (x + 3 < L.w) {
      *reinterpret_cast<float4*>(L.img + o) = make_float4(v[4], v[5], v[6], v[7]);
      *reinterpret_cast<float4*>(L.gx + o) = make_float4(gx[0], gx[1], gx[2], gx[3]);
      *reinterpret_cast<float4*>(L.gy + o) = make_float4(gy[0], gy[1], gy[2], gy[3]);
    } else {
      for (int i = 0; i < 4 && x + i < L.w; ++i) {
        L.img[o + i] = v[4 + i];
        L.gx[o + i] = gx[i];
        L.gy[o + i] = gy[i];
      }
    }
  }
}

// MINB: CTAs resident per SM the registers are budgeted for (2, or 3 with fewer registers).
template <int MINB>
__global__ void __launch_bounds__(kThreads, MINB) pyramid_l012_kernel(const __grid_constant__ StageBatch batch) {
  extern __shared__ __align__(128) unsigned char sm[];
  __shared__ int s_q;
  const int tid = threadIdx.x;
  if (tid == 0) s_q = batch.queue ? atomicAdd(batch.queue, 1) : (int)blockIdx.x;
  __syncthreads();
  const int q = s_q;
  int j = 0, idx = 0;
  bool deep = false;
  for (; j < batch.njobs; ++j) {
    const StageJob& J = batch.job[j];
    if (q >= J.tile_begin && q < J.tile_begin + J.tiles_x * J.tiles_y) {
      idx = q - J.tile_begin;
      break;
    }
    if (J.tail_levels > 0 && q >= J.q_deep && q < J.q_deep + J.deep_items) {
      idx = q - J.q_deep;
      deep = true;
      break;
    }
  }
  if (j < batch.njobs) {
    const StageJob& job = batch.job[j];
    if (!deep) {
      l012_tile(batch, job, idx, sm);
    } else {
      deep_item(batch, job, idx, reinterpret_cast<float*>(sm));
    }
  }
  if (batch.queue) {
    // the last CTA to finish returns the queue and the jobs' item counters to zero for the next
    // launch: every other CTA has counted itself finished after its own counter updates
    __syncthreads();
    if (tid == 0) {
      __threadfence();
      if (atomicAdd(batch.queue + 1, 1) == (int)gridDim.x - 1) {
        __threadfence();
        for (int k = 0; k < batch.njobs; ++k)
          if (batch.job[k].tail_levels > 0) {
            batch.job[k].done[0] = 0;
            batch.job[k].done[1] = 0;
            batch.job[k].done[2] = 0;
          }
        batch.queue[0] = 0;
        batch.queue[1] = 0;
      }
    }
  }
}

}  // namespace l012

constexpr size_t stage_smem(int kt, int nl, bool tail = true) {
  return sizeof(float) * (tail && kTailFloats > smem_floats(kt, nl) ? kTailFloats : smem_floats(kt, nl));
}

template <typename InT, int NL, int KT>
cudaError_t set_stage_attr() {
  return cudaFuncSetAttribute(pyramid_stage_kernel<InT, NL, KT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)stage_smem(KT, NL));
}

template <typename InT, int NL>
cudaError_t launch_stage(const StageBatch& b, int tiles, int kt, bool tail, cudaStream_t s) {
  if ((kt & 31) == 16)
    pyramid_stage_kernel<InT, NL, 16><<<tiles, kThreads, stage_smem(16, NL, tail), s>>>(b);
  else
    pyramid_stage_kernel<InT, NL, 8><<<tiles, kThreads, stage_smem(8, NL, tail), s>>>(b);
  return cudaGetLastError();
}

template <int KT>
cudaError_t set_stage_attrs() {
  cudaError_t e;
  if ((e = set_stage_attr<uint8_t, 0, KT>()) != cudaSuccess) return e;
  if ((e = set_stage_attr<uint8_t, 1, KT>()) != cudaSuccess) return e;
  if ((e = set_stage_attr<uint8_t, 2, KT>()) != cudaSuccess) return e;
  if ((e = set_stage_attr<float, 0, KT>()) != cudaSuccess) return e;
  if ((e = set_stage_attr<float, 1, KT>()) != cudaSuccess) return e;
  return set_stage_attr<float, 2, KT>();
}

// ---------------------------------------------------------------- input stage
// Level 0 from an RGB8 frame, or from a small mono frame with the box prefilter (larger mono frames
// get the prefilter inside the levels 0-2 kernel).  One thread per pixel.
template <int CH>
__device__ __forceinline__ float input_gray(const uint8_t* src, int64_t pitch, int x, int y) {
  const uint8_t* p = src + (int64_t)y * pitch + (int64_t)x * CH;
  if (CH == 1) return (float)p[0];
  const float red = p[0], green = p[1], blue = p[2];
  // the expression of cast_image_kernel_rgb (image_cast.cu:60-66), contracted by nvcc the same way
  return 0.299f * red + 0.587f * green + 0.114f * blue;
}

template <int CH>
__global__ void input_stage_kernel(const uint8_t* src, int64_t pitch, int box3, int w, int h, float* dst,
                                   int64_t dp) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= w || y >= h) return;
  float v = input_gray<CH>(src, pitch, x, y);
  if (box3 && x > 0 && x < w - 1 && y > 0 && y < h - 1) {
    // box_blur_x / box_blur_y (convolutions.cu:141-205): [1 2 1]/4 along x, then along y, truncated
    float col[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const int yy = y - 1 + k;
      float s = __fmul_rn(0.25f, input_gray<CH>(src, pitch, x - 1, yy));
      s = __fmaf_rn(0.5f, input_gray<CH>(src, pitch, x, yy), s);
      col[k] = __fmaf_rn(0.25f, input_gray<CH>(src, pitch, x + 1, yy), s);
    }
    float t = __fmul_rn(0.25f, col[0]);
    t = __fmaf_rn(0.5f, col[1], t);
    t = __fmaf_rn(0.25f, col[2], t);
    v = (float)(__float2uint_rz(t) & 0xffu);
  }
  dst[(int64_t)y * dp + x] = v;
}

}  // namespace

int l012_deep_floats() { return l012::kDeepFloats; }

int stage_tile(bool u8, int nl, int kt) { return (u8 && nl == 2) ? l012::kT2 : ((kt & 31) == 16 ? 16 : 8); }

namespace {

using TmapEncode = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// cuTensorMapEncodeTiled through the runtime's driver entry point, looked up once per process (the
// initialisation of a function-local static is thread-safe); null when unavailable.
TmapEncode tmap_encoder() {
  static const TmapEncode encode = []() -> TmapEncode {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      return reinterpret_cast<TmapEncode>(fn);
    return nullptr;
  }();
  return encode;
}

}  // namespace

bool encode_plane_tmap_f32(CUtensorMap* map, const float* base, int w, int h, int pitch_floats, int box_w, int box_h) {
  const TmapEncode encode = tmap_encoder();
  if (!encode || !map || !base || w <= 0 || h <= 0 || box_w <= 0 || box_h <= 0 || box_w > 256 || box_h > 256)
    return false;
  const int64_t pitch_bytes = (int64_t)pitch_floats * 4;
  if (((uintptr_t)base % 16) != 0 || (pitch_bytes % 16) != 0 || ((int64_t)box_w * 4) % 16 != 0) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)w, (cuuint64_t)h};
  const cuuint64_t strides[1] = {(cuuint64_t)pitch_bytes};
  const cuuint32_t box[2] = {(cuuint32_t)box_w, (cuuint32_t)box_h};
  const cuuint32_t estr[2] = {1, 1};
  return encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(base), dims, strides, box, estr,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

bool encode_frame_tmap(StageJob& job) {
  const TmapEncode encode = tmap_encoder();
  job.use_tma = 0;
  if (!encode) return false;
  // TMA needs a 16-byte aligned base and pitch; frames smaller than the box use plain loads
  if (((uintptr_t)job.src % 16) != 0 || (job.src_pitch_bytes % 16) != 0) return false;
  if (job.src_w < l012::kS0W || job.src_h < l012::kS0H) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)job.src_w, (cuuint64_t)job.src_h};
  const cuuint64_t strides[1] = {(cuuint64_t)job.src_pitch_bytes};
  const cuuint32_t box[2] = {(cuuint32_t)l012::kS0W, (cuuint32_t)l012::kS0H};
  const cuuint32_t estr[2] = {1, 1};
  if (encode(&job.tmap, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void*>(job.src), dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return false;
  job.use_tma = 1;
  return true;
}

cudaError_t pyramid_init() {
  cudaError_t e;
  if ((e = cudaFuncSetAttribute(l012::pyramid_l012_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                l012::kSmemBox)) != cudaSuccess)
    return e;
  if ((e = cudaFuncSetAttribute(l012::pyramid_l012_kernel<3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                l012::kSmemBox)) != cudaSuccess)
    return e;
  if ((e = set_stage_attrs<8>()) != cudaSuccess) return e;
  return set_stage_attrs<16>();
}

cudaError_t launch_input_stage(const uint8_t* src, int64_t src_pitch, int channels, int box3, int w, int h,
                               float* dst, int64_t dst_pitch_floats, cudaStream_t s) {
  const dim3 block(32, 8), grid((w + 31) / 32, (h + 7) / 8);
  if (channels == 3)
    input_stage_kernel<3><<<grid, block, 0, s>>>(src, src_pitch, box3, w, h, dst, dst_pitch_floats);
  else
    input_stage_kernel<1><<<grid, block, 0, s>>>(src, src_pitch, box3, w, h, dst, dst_pitch_floats);
  return cudaGetLastError();
}

cudaError_t launch_pyramid_stage(const StageBatch& b, int tiles, bool u8, int nl, int kt, bool tail, cudaStream_t s) {
  if (tiles <= 0) return cudaSuccess;
  if (u8) {
    switch (nl) {
      case 0: return launch_stage<uint8_t, 0>(b, tiles, kt, tail, s);
      case 1: return launch_stage<uint8_t, 1>(b, tiles, kt, tail, s);
      default:
        bool box = false;
        for (int j = 0; j < b.njobs; ++j) box = box || b.job[j].box3;
        const int smem = box ? l012::kSmemBox : l012::kSmem;
        if (kt & kL012Three)
          l012::pyramid_l012_kernel<3><<<tiles, l012::kThreads, smem, s>>>(b);
        else
          l012::pyramid_l012_kernel<2><<<tiles, l012::kThreads, smem, s>>>(b);
        return cudaGetLastError();
    }
  }
  switch (nl) {
    case 0: return launch_stage<float, 0>(b, tiles, kt, tail, s);
    case 1: return launch_stage<float, 1>(b, tiles, kt, tail, s);
    default: return launch_stage<float, 2>(b, tiles, kt, tail, s);
  }
}

}  // namespace fe
