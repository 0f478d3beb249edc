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
// fractions; corner products rounded half up, cross products half down) with an FP32 multiply-add
// chain, FE_SAMPLE_TEXTURE_WIDE the same weights with the 4-tap sum rounded once (FP64), and
// FE_SAMPLE_EXACT exact weights.  Divisions are IEEE (the reference's __fdividef differs by <= 2 ulp).
#include <cuda_runtime.h>

#include <climits>

#include "fe_common.cuh"
#include "fe_internal.h"
#include "lk_common.cuh"
#include "lk_track.cuh"

namespace fe {

namespace {

using namespace lk;

// WARPS warps per block (one track each), at least MINB blocks per SM (which bounds the registers).
template <int SAMPLING, bool HORIZ, int MODE, int WARPS, int MINB>
__global__ void __launch_bounds__(WARPS * 32, MINB) lk_kernel(const __grid_constant__ LkLaunch p) {
  __shared__ WarpSmem smem[WARPS];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const LkCam* cams = p.cams ? p.cams : &p.single;
  int g = p.counter ? 0 : (int)blockIdx.x * WARPS + wid;
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
    fe_track_data& td = cam.tracks[g - cam.begin];
    if (cam.tracks_in) {
      // out-of-place: the 80-byte record is copied first, then tracked in place
      __syncwarp();
      if (lane < 20)
        reinterpret_cast<uint32_t*>(&td)[lane] = reinterpret_cast<const uint32_t*>(&cam.tracks_in[g - cam.begin])[lane];
      __syncwarp();
    }
    track_one<SAMPLING, HORIZ, MODE>(cam, td, smem[wid], lane, p.iters, p.tol2,
                                     MODE == kModeUnrolled && p.recs ? p.recs + g : nullptr, p.counts);
    if (MODE == kModeRef && cam.retrack_ncc > 0.f) {
      // MonoSOFGPU's retrack pass, merged as collect reads it: a track the first pass lost (its
      // record still holds the inputs) runs again with the retrack NCC threshold
      __syncwarp();
      if (td.track_status == 0 && td.search_radius_px >= 0.f) {
        const float keep = td.ncc_threshold;
        __syncwarp();
        if (lane == 0) td.ncc_threshold = cam.retrack_ncc;
        __syncwarp();
        track_one<SAMPLING, HORIZ, MODE>(cam, td, smem[wid], lane, p.iters, p.tol2, nullptr, p.counts);
        __syncwarp();
        if (lane == 0) td.ncc_threshold = keep;
      }
    }
    if (!p.counter) return;
  }
}

template <int SAMPLING, bool HORIZ, int MODE, int WARPS, int MINB>
cudaError_t launch_shape(const LkLaunch& p, cudaStream_t s) {
  // blocks of this shape resident on the device (persistent grid), found once per process
  static const int resident = [] {
    int per_sm = 0, dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lk_kernel<SAMPLING, HORIZ, MODE, WARPS, MINB>, WARPS * 32, 0);
    return (per_sm > 0 ? per_sm : 1) * (sms > 0 ? sms : 1);
  }();
  int blocks = (p.total + WARPS - 1) / WARPS;
  if (p.counter) blocks = min(blocks, resident);
  lk_kernel<SAMPLING, HORIZ, MODE, WARPS, MINB><<<blocks, WARPS * 32, 0, s>>>(p);
  return cudaGetLastError();
}

// Reference-rule launches take the block shape p.shape (kLkShapes); the differentiable modes use
// the first.
template <int SAMPLING, bool HORIZ, int MODE>
cudaError_t launch(const LkLaunch& p, cudaStream_t s) {
  if (MODE == kModeRef) {
    switch (p.shape) {
      case 1: return launch_shape<SAMPLING, HORIZ, MODE, 8, 3>(p, s);
      case 2: return launch_shape<SAMPLING, HORIZ, MODE, 4, 8>(p, s);
      case 3: return launch_shape<SAMPLING, HORIZ, MODE, 12, 2>(p, s);
      default: break;
    }
  }
  return launch_shape<SAMPLING, HORIZ, MODE, 8, 4>(p, s);
}

}  // namespace

cudaError_t launch_lk(const LkLaunch& p, cudaStream_t s) {
  if (p.total <= 0) return cudaSuccess;
  if (p.sampling == FE_SAMPLE_HARDWARE) return p.mode == kLkReference ? launch_lk_hw(p, s) : cudaErrorInvalidValue;
  if (p.counter) {
    cudaError_t e = cudaMemsetAsync(p.counter, 0, sizeof(int), s);
    if (e != cudaSuccess) return e;
  }
  if (p.mode == kLkImplicit) return launch<FE_SAMPLE_EXACT, false, kModeImplicit>(p, s);
  if (p.mode == kLkUnrolled) return launch<FE_SAMPLE_EXACT, false, kModeUnrolled>(p, s);
  if (p.sampling == FE_SAMPLE_EXACT)
    return p.horizontal ? launch<FE_SAMPLE_EXACT, true, kModeRef>(p, s) : launch<FE_SAMPLE_EXACT, false, kModeRef>(p, s);
  if (p.sampling == FE_SAMPLE_TEXTURE_WIDE)
    return p.horizontal ? launch<FE_SAMPLE_TEXTURE_WIDE, true, kModeRef>(p, s)
                        : launch<FE_SAMPLE_TEXTURE_WIDE, false, kModeRef>(p, s);
  return p.horizontal ? launch<FE_SAMPLE_TEXTURE, true, kModeRef>(p, s) : launch<FE_SAMPLE_TEXTURE, false, kModeRef>(p, s);
}

}  // namespace fe
