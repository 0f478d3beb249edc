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

constexpr int kT = 16;        // deepest-level core tile
constexpr int kThreads = 256;

__host__ __device__ constexpr int region_size(int nl, int k) {
  return k == nl ? kT + 6 : 2 * region_size(nl, k + 1) + 3;
}
__host__ __device__ constexpr int smem_floats(int nl) {
  int s = 0;
  for (int k = 0; k <= nl; ++k) s += region_size(nl, k) * region_size(nl, k);
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

template <typename InT, int NL>
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
  const int X = (t % job.tiles_x) * kT, Y = (t / job.tiles_x) * kT;

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
    S[k] = region_size(NL, k);
    off[k] = o;
    o += S[k] * S[k];
  }

  // 1. stage the input region
  {
    const int w = job.src_w, h = job.src_h;
    const InT* src = static_cast<const InT*>(job.src);
    float* dst = smem + off[0];
    for (int i = threadIdx.x; i < S[0] * S[0]; i += kThreads) {
      const int r = i / S[0], c = i - r * S[0];
      const int gx = a[0] + c, gy = ay[0] + r;
      dst[i] = (gx >= 0 && gy >= 0 && gx < w && gy < h) ? load_px(src, job.src_pitch_bytes, gx, gy) : 0.f;
    }
  }
  __syncthreads();

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
    const int C = kT << (NL - k);
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
}

template <typename InT, int NL>
cudaError_t set_stage_attr() {
  return cudaFuncSetAttribute(pyramid_stage_kernel<InT, NL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)(sizeof(float) * smem_floats(NL)));
}

template <typename InT, int NL>
cudaError_t launch_stage(const StageBatch& b, int tiles, cudaStream_t s) {
  pyramid_stage_kernel<InT, NL><<<tiles, kThreads, sizeof(float) * smem_floats(NL), s>>>(b);
  return cudaGetLastError();
}

}  // namespace

int stage_tile() { return kT; }

cudaError_t pyramid_init() {
  cudaError_t e;
  if ((e = set_stage_attr<uint8_t, 0>()) != cudaSuccess) return e;
  if ((e = set_stage_attr<uint8_t, 1>()) != cudaSuccess) return e;
  if ((e = set_stage_attr<uint8_t, 2>()) != cudaSuccess) return e;
  if ((e = set_stage_attr<float, 0>()) != cudaSuccess) return e;
  if ((e = set_stage_attr<float, 1>()) != cudaSuccess) return e;
  return set_stage_attr<float, 2>();
}

cudaError_t launch_pyramid_stage(const StageBatch& b, int tiles, bool u8, int nl, cudaStream_t s) {
  if (tiles <= 0) return cudaSuccess;
  if (u8) {
    switch (nl) {
      case 0: return launch_stage<uint8_t, 0>(b, tiles, s);
      case 1: return launch_stage<uint8_t, 1>(b, tiles, s);
      default: return launch_stage<uint8_t, 2>(b, tiles, s);
    }
  }
  switch (nl) {
    case 0: return launch_stage<float, 0>(b, tiles, s);
    case 1: return launch_stage<float, 1>(b, tiles, s);
    default: return launch_stage<float, 2>(b, tiles, s);
  }
}

}  // namespace fe
