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

// Two warp sums at once, each bit-identical to warp_sum of its argument (the same pairs added at
// every stage): after the first stage a lane keeps one of the two partial sums (lanes with bit 0
// clear keep a's), so the later stages move one value instead of two; the totals are read from
// lanes 0 and 1.
__device__ __forceinline__ void warp_sum2(float& a, float& b, int lane) {
  const bool odd = (lane & 1) != 0;
  float keep = odd ? b : a;
  keep += __shfl_xor_sync(0xffffffffu, odd ? a : b, 1);
#pragma unroll
  for (int m = 2; m < 32; m <<= 1) keep += __shfl_xor_sync(0xffffffffu, keep, m);
  a = __shfl_sync(0xffffffffu, keep, 0);
  b = __shfl_sync(0xffffffffu, keep, 1);
}

// Three warp sums at once, each bit-identical to warp_sum of its argument: after stage 1 even lanes
// keep a's and b's partial sums and odd lanes c's, after stage 2 each lane keeps one (a on lanes with
// bits 0 and 1 clear, b with bit 1 set, c on odd lanes); the totals are read from lanes 0, 2 and 1.
__device__ __forceinline__ void warp_sum3(float& a, float& b, float& c, int lane) {
  const bool odd = (lane & 1) != 0, hi = (lane & 2) != 0;
  const float r1 = __shfl_xor_sync(0xffffffffu, odd ? a : c, 1);  // even lanes: a; odd lanes: c
  const float r2 = __shfl_xor_sync(0xffffffffu, b, 1);            // even lanes: b
  const float ka = a + r1, kb = b + r2, kc = c + r1;
  float keep = odd ? kc : (hi ? kb : ka);
  keep += __shfl_xor_sync(0xffffffffu, odd ? kc : (hi ? ka : kb), 2);
#pragma unroll
  for (int m = 4; m < 32; m <<= 1) keep += __shfl_xor_sync(0xffffffffu, keep, m);
  a = __shfl_sync(0xffffffffu, keep, 0);
  b = __shfl_sync(0xffffffffu, keep, 2);
  c = __shfl_sync(0xffffffffu, keep, 1);
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
