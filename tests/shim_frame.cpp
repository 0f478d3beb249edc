// Test driver of include/cuvslam_fe_shim.hpp: one MonoSOFGPU-style frame through the four restated
// wrapper classes, exported as a C function for the tests (ctypes).
//   ImageContext::build_gpu_image_pyramid + build_gpu_gradient_pyramid (image_context.cpp:215-255)
//     -> GaussianGPUImagePyramid::build_u8 + GPUGradientPyramid::set, for both frames;
//   MonoSOFGPU::addFeatures (sof_mono_gpu.cpp:222-247) -> GPUSelection::computeGFTTAndSelectFeatures
//     on the previous frame (no alive features, optional mask);
//   MonoSOFGPU::launch (sof_mono_gpu.cpp:34-78) -> TrackData filled on the host, copied up,
//     GPULKFeatureTracker::track_points (or the horizontal tracker), copied back;
//   then a second selection on the current frame with the tracked features alive.
// The GPU test compares every output with the same steps through the Python binding.
#include <cstdio>
#include <cstring>
#include <exception>
#include <vector>

#include "cuvslam_fe_shim.hpp"

using namespace cuvslam;
using namespace cuvslam::cuda;

namespace {
char g_error[512];
}

extern "C" const char* shim_last_error() { return g_error; }

// sel0: first selection (capacity k x 2, *n_sel0); tracks: the tracked records (capacity k);
// sel1: second selection (capacity k x 2, *n_sel1).  Returns 0, or -1 with shim_last_error().
extern "C" int shim_frame(const uint8_t* prev_host, const uint8_t* next_host, int w, int h, int k,
                          const uint8_t* mask_host, int horizontal, float* sel0, int* n_sel0, void* tracks, float* sel1,
                          int* n_sel1) {
  g_error[0] = 0;
  try {
    cudaStream_t stream = nullptr;
    shim_check_cuda(cudaStreamCreate(&stream), "cudaStreamCreate");
    uint8_t *d_prev = nullptr, *d_next = nullptr;
    shim_check_cuda(cudaMalloc((void**)&d_prev, (size_t)w * h), "frames");
    shim_check_cuda(cudaMalloc((void**)&d_next, (size_t)w * h), "frames");
    shim_check_cuda(cudaMemcpy(d_prev, prev_host, (size_t)w * h, cudaMemcpyHostToDevice), "upload");
    shim_check_cuda(cudaMemcpy(d_next, next_host, (size_t)w * h, cudaMemcpyHostToDevice), "upload");

    GaussianGPUImagePyramid prev_pyr(w, h), cur_pyr(w, h);
    GPUGradientPyramid prev_grad(w, h), cur_grad(w, h);
    prev_pyr.build_u8(d_prev, w, w, h, false, stream);
    cur_pyr.build_u8(d_next, w, w, h, false, stream);
    prev_grad.set(prev_pyr, stream, horizontal != 0);
    cur_grad.set(cur_pyr, stream, horizontal != 0);

    ImageMatrix<uint8_t> mask(h, w);
    if (mask_host) std::memcpy(mask.data(), mask_host, (size_t)w * h);
    GPUSelection selection;
    std::vector<Vector2T> alive, added;
    selection.computeGFTTAndSelectFeatures(prev_grad, 0, 0, 0, 0, mask_host ? &mask : nullptr, alive, (size_t)k, added,
                                           stream);
    *n_sel0 = (int)added.size();
    for (size_t i = 0; i < added.size(); ++i) {
      sel0[2 * i] = added[i].x();
      sel0[2 * i + 1] = added[i].y();
    }

    // MonoSOFGPU::launch fills the records on the host (sof_mono_gpu.cpp:45-63)
    const size_t n = added.size();
    GPUArrayPinned<TrackData> track_data(n > 0 ? n : 1);
    for (size_t i = 0; i < n; ++i) {
      TrackData& t = track_data[i];
      std::memset(&t, 0, sizeof(t));
      t.track[0] = added[i].x();
      t.track[1] = added[i].y();
      t.cache_index = -1;
      t.initial_guess_map[0] = 1.f;
      t.initial_guess_map[3] = 1.f;
      t.search_radius_px = (float)w;
      t.ncc_threshold = 0.8f;
    }
    track_data.copy_top_n(ToGPU, n, stream);
    GPULKFeatureTracker lk;
    GPULKTrackerHorizontal lk_h;
    GPULKFeatureTracker& tracker = horizontal ? static_cast<GPULKFeatureTracker&>(lk_h) : lk;
    if (!tracker.track_points(prev_grad, cur_grad, prev_pyr, cur_pyr, track_data, n, stream)) {
      std::snprintf(g_error, sizeof(g_error), "track_points returned false");
      return -1;
    }
    track_data.copy_top_n(ToCPU, n, stream);
    shim_check_cuda(cudaStreamSynchronize(stream), "sync");
    if (n > 0) std::memcpy(tracks, &track_data[0], n * sizeof(TrackData));

    // the next frame's selection with the tracked features alive, appended after one kept entry
    // (the reference appends and counts entries already in the vector against the limit)
    std::vector<Vector2T> survivors, added2;
    for (size_t i = 0; i < n; ++i)
      if (track_data[i].track_status) survivors.emplace_back(track_data[i].track[0], track_data[i].track[1]);
    added2.emplace_back(-1.f, -1.f);
    selection.computeGFTTAndSelectFeatures(cur_grad, 2, 3, 4, 5, nullptr, survivors,
                                           (size_t)k > survivors.size() ? (size_t)k - survivors.size() : 0, added2,
                                           stream);
    if (added2[0].x() != -1.f) {
      std::snprintf(g_error, sizeof(g_error), "the vector's first entry was overwritten");
      return -1;
    }
    *n_sel1 = (int)added2.size() - 1;
    for (size_t i = 1; i < added2.size(); ++i) {
      sel1[2 * (i - 1)] = added2[i].x();
      sel1[2 * (i - 1) + 1] = added2[i].y();
    }
    cudaFree(d_prev);
    cudaFree(d_next);
    cudaStreamDestroy(stream);
    return 0;
  } catch (const std::exception& e) {
    std::snprintf(g_error, sizeof(g_error), "%s", e.what());
    return -1;
  }
}

// Error behaviour: a gradient pyramid that was never set is refused with std::invalid_argument
// (as a null texture would make the reference fail), reported here as 1.  No kernel runs.
extern "C" int shim_unset_gradients_throws() {
  try {
    GPUGradientPyramid g;
    GPUSelection s;
    std::vector<Vector2T> alive, out;
    cudaStream_t stream = nullptr;
    s.computeGFTTAndSelectFeatures(g, 0, 0, 0, 0, nullptr, alive, 10, out, stream);
  } catch (const std::invalid_argument&) {
    return 1;
  } catch (...) {
    return 2;
  }
  return 0;
}
