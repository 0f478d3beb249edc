// Integration examples for the entry points the drop-in shim (include/cuvslam_fe_shim.hpp) does not
// wrap: left-to-right matching, the affine tracker and the differentiable tracker.  Each function is
// what a cuVSLAM maintainer would write at the named call site; a CPU test compiles this file against
// the real headers, so an example whose arguments no longer fit an entry point fails to build.
#include <cstdint>
#include <vector>

#include "cuvslam_fe_shim.hpp"

using namespace cuvslam::cuda;

#define FE_CHECK(x) shim_check_fe((x), #x)

// MultiSOFGPU::LaunchTrackingPrimaryToSecondary (sof_multicamera_gpu.cpp:69-190): one call for all
// primary -> secondary pairs instead of a launch + copy + synchronisation per candidate round.
// The epipolar table (EpipolarCurves, curves_[v][u]) lives on the device as CSR, once per pair.
void example_left_to_right(fe_context* ctx, fe_stereo_pair* pairs, int npairs, int top_w, int top_h, int top_level,
                           const int32_t* d_offsets, const float* d_xy, int32_t max_len,
                           const GaussianGPUImagePyramid& primary, const GaussianGPUImagePyramid& secondary,
                           const float* d_uvL, const uint8_t* d_valid, int n, GPUArrayPinned<TrackData>& tracks_data,
                           int32_t* d_winner, int32_t* d_stats, float kL2REarlyExitFraction, bool lk_horizontal,
                           float search_radius, cudaStream_t stream) {
  fe_epipolar_curves curves = {top_w + 1, top_h + 1, 1.f / (float)(1 << top_level), d_offsets, d_xy, max_len};
  fe_stereo_pair pair = {};
  pair.primary = &primary.desc();
  pair.secondary = &secondary.desc();
  pair.uv = d_uvL;  // primary observations (denormalizePoint)
  pair.valid = d_valid;
  pair.n = n;
  pair.curves = &curves;  // or cand_offsets / cand_xy / max_candidates
  pair.search_radius = search_radius;  // CrossCamSearchRadius(top_level)
  pair.ncc_threshold = 0.8f;
  pair.out = reinterpret_cast<fe_track_data*>(tracks_data.ptr());
  pair.winner = d_winner;
  pair.stats = d_stats;
  pairs[0] = pair;
  FE_CHECK(fe_track_stereo(ctx, pairs, npairs, kL2REarlyExitFraction, lk_horizontal ? 1 : 0, FE_SAMPLE_TEXTURE_WIDE,
                           stream));
}

// GPUSTFeatureTracker / GPUSTFeatureTrackerWithCache (cuda_modules/st_tracker.cpp:22-160): the
// current pyramid supplies image and both gradients, the previous one its image;
// PointCacheData<float, 9> is fe_affine_cache byte for byte.
void example_affine(fe_context* ctx, const GaussianGPUImagePyramid& prev, const GaussianGPUImagePyramid& cur,
                    GPUArrayPinned<TrackData>& td, GPUArrayPinned<fe_affine_cache>& cache_data, size_t n,
                    int n_shift_only_iterations, int n_full_mapping_iterations, cudaStream_t s) {
  FE_CHECK(fe_track_affine(ctx, &prev.desc(), &cur.desc(), reinterpret_cast<fe_track_data*>(td.ptr()), (int)n,
                           n_shift_only_iterations, n_full_mapping_iterations, FE_SAMPLE_TEXTURE_WIDE, s));
  FE_CHECK(fe_affine_build_cache(ctx, &prev.desc(), reinterpret_cast<fe_track_data*>(td.ptr()), (int)n,
                                 cache_data.ptr(), FE_SAMPLE_TEXTURE_WIDE, s));
  FE_CHECK(fe_track_affine_cached(ctx, &cur.desc(), cache_data.ptr(), (int)cache_data.size(),
                                  reinterpret_cast<fe_track_data*>(td.ptr()), (int)n, n_shift_only_iterations,
                                  n_full_mapping_iterations, FE_SAMPLE_TEXTURE_WIDE, s));
}

// A training or calibration loop: plan once, then forward / backward without allocation.
void example_adjoint(fe_context* ctx, const fe_pyramid& prev_desc, const fe_pyramid& cur_desc, const float* d_prev_f32,
                     const float* d_cur_f32, int w, const fe_track_data* d_tracks, fe_track_data* d_tracks_out, int n,
                     const float* d_dLdpos, float* d_gprev, float* d_gcur, float* d_gtrack, float* d_goffset,
                     cudaStream_t s) {
  fe_adjoint_job job = {};  // one per camera (<= 64), device pointers
  job.prev = &prev_desc;
  job.cur = &cur_desc;              // pyramids (built by the plan or by the caller)
  job.prev_image = d_prev_f32;      // optional: frames the plan builds the pyramids from
  job.cur_image = d_cur_f32;
  job.image_pitch_bytes = w * 4;
  job.image_scale = 255.f;          // frames in [0, 1] -> uint8 intensity scale
  job.tracks_in = d_tracks;
  job.tracks_out = d_tracks_out;
  job.n_tracks = n;
  job.grad_xy = d_dLdpos;           // n x 2, set before the backward
  job.grad_prev = d_gprev;
  job.grad_prev_pitch_bytes = w * 4;
  job.grad_cur = d_gcur;
  job.grad_cur_pitch_bytes = w * 4;
  job.grad_track = d_gtrack;        // optional, n x 2
  job.grad_offset = d_goffset;
  fe_adjoint* adj = nullptr;
  FE_CHECK(fe_adjoint_create(ctx, &job, 1, FE_ADJOINT_IMPLICIT, /*iterations=*/20, /*tolerance=*/1e-4f, &adj));
  FE_CHECK(fe_adjoint_build_pyramids(adj, s));
  FE_CHECK(fe_adjoint_forward(adj, s));   // tracks_in -> tracks_out
  // ... the loss writes dL/dpos into d_dLdpos ...
  FE_CHECK(fe_adjoint_backward(adj, s));  // -> d_gprev, d_gcur, d_gtrack, d_goffset (deterministic)
  FE_CHECK(fe_adjoint_destroy(adj));
}
