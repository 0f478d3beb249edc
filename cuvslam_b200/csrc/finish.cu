// Device-side track filters of a frame (MonoSOFGPU::finish after collect), so the frame step needs
// no copy back and host loop between tracking and selection.  One CTA per camera, phases separated
// by barriers, in the reference's order (sof_mono_gpu.cpp:144-170):
//   collect + age  (sof_mono_gpu.cpp:80-104, sof_mono_base.cpp:111-118): an alive track whose LK
//                  record (track and retrack passes merged) has track_status keeps it and ages by
//                  one; otherwise it dies;
//   prediction     (sof_mono_base.cpp:51-109): d = |prediction - position| over the alive tracks
//                  with a prediction; with at least 3 of them, the (count/2)-th smallest d is found
//                  by a radix select on its bits (d >= 0 orders like its bits) and tracks with
//                  d > max(3, 2 d_k) die;
//   border         (selector_stereo.cpp:109-125) and mask (sof_mono_base.cpp:121-133) kills;
//   collapse       (sof_mono_gpu.cpp:249-280): per 3x3-pixel cell, the first track in index order with
//                  the cell's largest age survives: one 64-bit atomicMax per track on
//                  (age << 32 | ~index), a survivor holds the cell's key; the cells are then cleared.
// Dead tracks get age 0 and track_status 0 (selection then ignores them).
#include <cuda_runtime.h>

#include "fe_common.cuh"
#include "fe_internal.h"

namespace fe {

namespace {

constexpr int kThreads = 1024;

__device__ __forceinline__ bool has_pred(const FinishCam& c, int i) {
  return c.pred && !isnan(c.pred[2 * i]);
}

// |prediction - position| as the reference computes it (no fused multiply-add).
__device__ __forceinline__ float pred_delta(const FinishCam& c, int i) {
  const float dx = __fsub_rn(c.pred[2 * i], c.tracks[i].track[0]);
  const float dy = __fsub_rn(c.pred[2 * i + 1], c.tracks[i].track[1]);
  return __fsqrt_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)));
}

__global__ void __launch_bounds__(kThreads) finish_kernel(const __grid_constant__ FinishBatch b) {
  const FinishCam& c = b.cam[blockIdx.x];
  __shared__ int s_count, s_bin, s_rank;
  __shared__ unsigned s_prefix;
  __shared__ int hist[256];
  const int n = c.n;

  // collect + age
  if (threadIdx.x == 0) s_count = 0;
  __syncthreads();
  int m = 0;
  for (int i = threadIdx.x; i < n; i += kThreads) {
    uint32_t a = c.age[i];
    if (a != 0) a = c.tracks[i].track_status ? a + 1 : 0;
    c.age[i] = a;
    if (a != 0 && has_pred(c, i)) ++m;
  }
  atomicAdd(&s_count, m);
  __syncthreads();
  m = s_count;

  // prediction filter
  if (c.pred && m >= 3) {
    unsigned prefix = 0, himask = 0;
    int rank = m / 2;
    for (int shift = 24; shift >= 0; shift -= 8) {
      for (int k = threadIdx.x; k < 256; k += kThreads) hist[k] = 0;
      __syncthreads();
      for (int i = threadIdx.x; i < n; i += kThreads) {
        if (c.age[i] == 0 || !has_pred(c, i)) continue;
        const unsigned u = __float_as_uint(pred_delta(c, i));
        if ((u & himask) == prefix) atomicAdd(&hist[(u >> shift) & 255u], 1);
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        int acc = 0, bin = 0;
        for (; bin < 255 && acc + hist[bin] <= rank; ++bin) acc += hist[bin];
        s_bin = bin;
        s_rank = rank - acc;
      }
      __syncthreads();
      prefix |= (unsigned)s_bin << shift;
      himask |= 255u << shift;
      rank = s_rank;
      __syncthreads();
    }
    if (threadIdx.x == 0) s_prefix = prefix;
    __syncthreads();
    const float kth = __uint_as_float(s_prefix);
    const float twice = __fmul_rn(2.f, kth);
    const float thr = 3.f < twice ? twice : 3.f;
    for (int i = threadIdx.x; i < n; i += kThreads)
      if (c.age[i] != 0 && has_pred(c, i) && pred_delta(c, i) > thr) c.age[i] = 0;
    __syncthreads();
  }

  // border and mask
  const float bl = (float)(unsigned long long)c.border[2], bt = (float)(unsigned long long)c.border[0];
  const float xr = __ull2float_rn((unsigned long long)c.w - 1ull - (unsigned long long)c.border[3]);
  const float yb = __ull2float_rn((unsigned long long)c.h - 1ull - (unsigned long long)c.border[1]);
  for (int i = threadIdx.x; i < n; i += kThreads) {
    if (c.age[i] == 0) continue;
    const float x = c.tracks[i].track[0], y = c.tracks[i].track[1];
    bool keep = bl <= x && x <= xr && bt <= y && y <= yb;
    if (keep && c.mask && x >= 0.f && y >= 0.f && x < (float)c.w && y < (float)c.h)
      keep = c.mask[(size_t)y * c.mask_pitch + (size_t)x] == 0;
    if (!keep) c.age[i] = 0;
  }
  __syncthreads();

  // collapse
  if (c.cells) {
    for (int i = threadIdx.x; i < n; i += kThreads) {
      if (c.age[i] == 0) continue;
      const int cx = (int)__fdiv_rn(c.tracks[i].track[0], 3.f), cy = (int)__fdiv_rn(c.tracks[i].track[1], 3.f);
      if (cx < 0 || cy < 0 || cx >= c.cw || cy >= c.ch) continue;
      atomicMax(&c.cells[(size_t)cy * c.cw + cx], ((unsigned long long)c.age[i] << 32) | (uint32_t)~(uint32_t)i);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += kThreads) {
      if (c.age[i] == 0) continue;
      const int cx = (int)__fdiv_rn(c.tracks[i].track[0], 3.f), cy = (int)__fdiv_rn(c.tracks[i].track[1], 3.f);
      if (cx < 0 || cy < 0 || cx >= c.cw || cy >= c.ch) continue;
      const unsigned long long mine = ((unsigned long long)c.age[i] << 32) | (uint32_t)~(uint32_t)i;
      if (c.cells[(size_t)cy * c.cw + cx] != mine) c.age[i] = 0;
    }
    __syncthreads();
    // clear the cells this camera touched (survivors' cells; every touched cell has one)
    for (int i = threadIdx.x; i < n; i += kThreads) {
      if (c.age[i] == 0) continue;
      const int cx = (int)__fdiv_rn(c.tracks[i].track[0], 3.f), cy = (int)__fdiv_rn(c.tracks[i].track[1], 3.f);
      if (cx < 0 || cy < 0 || cx >= c.cw || cy >= c.ch) continue;
      c.cells[(size_t)cy * c.cw + cx] = 0ull;
    }
  }

  // dead tracks leave selection's alive set; count the survivors
  if (threadIdx.x == 0) s_count = 0;
  __syncthreads();
  int alive = 0;
  for (int i = threadIdx.x; i < n; i += kThreads) {
    if (c.age[i] == 0)
      c.tracks[i].track_status = 0;
    else
      ++alive;
  }
  atomicAdd(&s_count, alive);
  __syncthreads();
  if (threadIdx.x == 0 && c.alive_count) *c.alive_count = s_count;
}

}  // namespace

cudaError_t launch_finish(const FinishBatch& b, cudaStream_t s) {
  if (b.ncams <= 0) return cudaSuccess;
  finish_kernel<<<b.ncams, kThreads, 0, s>>>(b);
  return cudaGetLastError();
}

}  // namespace fe
