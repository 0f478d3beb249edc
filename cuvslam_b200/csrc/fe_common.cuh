// Shared device-side types and helpers of the front-end kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "cuvslam_fe.h"

namespace fe {

constexpr int kMaxLevels = FE_MAX_LEVELS;
constexpr int kMinLevelDim = 15;
constexpr int kMaxCams = 64;  // cameras per batched launch

// One pyramid level as the kernels see it: pitch in floats.
struct Level {
  float* img;
  float* gx;
  float* gy;
  int w, h;
  int pitch;
};

struct Pyr {
  int levels;
  Level lv[kMaxLevels];
};

// 7-tap DSP derivative of the reference gradient kernels (convolutions.cu:25-26), as the same float
// constants; the centre tap is zero.
__device__ __forceinline__ float dsp_tap(int j) {
  switch (j) {
    case 0: return 112.0f / 8418.0f;
    case 1: return 913.0f / 8418.0f;
    case 2: return 3047.0f / 8418.0f;
    case 3: return 0.0f;
    case 4: return -3047.0f / 8418.0f;
    case 5: return -913.0f / 8418.0f;
    default: return -112.0f / 8418.0f;
  }
}

// 9x9 LK window weights: outer product of these (lk_tracker.cu:26-27).
__device__ __forceinline__ float gauss9(int i) {
  switch (i) {
    case 0: case 8: return 0.0135196f;
    case 1: case 7: return 0.0476622f;
    case 2: case 6: return 0.11723f;
    case 3: case 5: return 0.201168f;
    default: return 0.240841f;
  }
}

// 7-tap Gaussian of the structure tensor (gftt.cu:25).
__device__ __forceinline__ float gauss7(int i) {
  switch (i) {
    case 0: case 6: return 0.00598f;
    case 1: case 5: return 0.060626f;
    case 2: case 4: return 0.241843f;
    default: return 0.383103f;
  }
}

__device__ __forceinline__ int mirror_index(int i, int n) {
  i = i >= 0 ? i : -i - 1;
  return i < n ? i : 2 * n - i - 1;
}

// xor-butterfly warp sum: every lane ends with the same value, the order of additions is fixed.
__device__ __forceinline__ float warp_sum(float x) {
#pragma unroll
  for (int m = 1; m < 32; m <<= 1) x += __shfl_xor_sync(0xffffffffu, x, m);
  return x;
}

// Asynchronous global->shared copies (cp.async, sm_80+); both addresses aligned to the copy size.
// A thread sees its own copies after cp_async_wait_all(); other threads after a barrier
// (__syncwarp / __syncthreads) that follows the wait.
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void cp_async16(float* dst, const float* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(float* dst, const float* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async4(float* dst, const float* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

}  // namespace fe
