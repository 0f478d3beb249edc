/* CPU oracle for the cuVSLAM visual-tracking front-end hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product links or calls this; tests, the golden
 * fixture script, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it through
 * oracle/liboracle.so as the checker.
 *
 * Two semantics are restated:
 *   or_*     : the reference GPU path (libs/cuda_modules), the parity target of the CUDA kernels.
 *              FP32 with the reference's evaluation order; reductions follow the reference's
 *              warp layouts (lane-sequential partial sums + xor-butterfly).  Only __logf and
 *              __fdividef, whose implementations are not ours to restate, are replaced by logf
 *              and IEEE division.
 *   cpu_*    : the reference CPU path (libs/sof, use_gpu=false), the timed CPU baseline.
 * plus an FP64 LK (or_lk_track_f64) used only to state per-track error, and an FP64
 * differentiable LK with its adjoint (or64_*) that pins the CUDA adjoint.
 */
#ifndef FE_ORACLE_H
#define FE_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* cuvslam::cuda::TrackData, 80 bytes (libs/cuda_modules/cuda_kernels/cuda_kernels.h:76-87). */
typedef struct {
  float track[2];
  float offset[2];
  float info[4];
  uint8_t track_status;
  uint8_t pad0[3];
  int32_t cache_index;
  float pad1[2];
  float initial_guess_map[4];
  float search_radius_px;
  float ncc_threshold;
  float ncc;
  float pad2;
} or_track_data;

/* Bilinear sampling modes of the LK oracle. */
enum { OR_SAMPLE_TEXTURE = 0, /* emulation of cudaFilterModeLinear (8-bit-fraction weights) */
       OR_SAMPLE_EXACT = 1,    /* exact FP32 weights */
       OR_SAMPLE_TEXTURE_WIDE = 2 }; /* texture weights, sum rounded once (closest to the hardware) */

int or_level_sizes(int w, int h, int max_levels, int* ws, int* hs);
void or_cast_u8(const uint8_t* src, int w, int h, float* dst);
void or_rgb_to_gray(const uint8_t* rgb, int w, int h, int64_t pitch, float* dst, int variant);
void or_box3(const float* src, int w, int h, float* dst);
void or_gauss_downscale(const float* src, int sw, int sh, float* dst, int dw, int dh);
void or_gradients(const float* in, int w, int h, float* gx, float* gy);
void or_gftt_response(const float* gx, const float* gy, int w, int h, float* resp);
void or_bins(const float* resp, int w, int h, float* bins64);
int or_select(const float* resp, int w, int h, const float* alive_xy, int n_alive, int num_desired, int border_top,
              int border_bottom, int border_left, int border_right, const uint8_t* mask, float* nms, float* cell_max,
              uint32_t* cell_idx, float* kp, int* n_kp, float* bins, float* sel);
float or_tex_sample(const float* img, int w, int h, float x, float y, int mode);
void or_lk_track(int levels, const int* ws, const int* hs, const float* const* prev_gx, const float* const* prev_gy,
                 const float* const* prev_img, const float* const* cur_img, or_track_data* td, int n, int mode);
void or_lk_track_horizontal(int levels, const int* ws, const int* hs, const float* const* prev_gx,
                            const float* const* prev_img, const float* const* cur_img, or_track_data* td, int n,
                            int mode);
void or_lk_track_f64(int levels, const int* ws, const int* hs, const float* const* prev_gx,
                     const float* const* prev_gy, const float* const* prev_img, const float* const* cur_img,
                     or_track_data* td, int n);

/* MonoSOFGPU::finish's track filters after LK (see fe_oracle.c); returns the tracks alive. */
int or_finish_tracks(or_track_data* td, uint32_t* age, int n, const float* pred, int w, int h, const int* border,
                     const uint8_t* mask, int64_t mask_pitch, int collapse);
/* Candidates of a primary base-level point (u, v) from an epipolar table of cw x ch corner curves
 * in CSR form (offsets[cw * ch + 1], xy pairs): EpipolarCurves::Candidates
 * (libs/sof/epipolar_curves.cpp:64-101).  Writes up to `cap` x, y pairs, returns the count. */
int or_epipolar_candidates(int cw, int ch, float inv_scale, const int32_t* offsets, const float* xy, float u, float v,
                           float* out, int cap);
/* Left-to-right candidate scan of one camera pair: MultiSOFGPU::LaunchTrackingPrimaryToSecondary
 * (libs/sof/sof_multicamera_gpu.cpp:118-190) with horizontal (or 2-D) LK per round.
 * Candidates of point i: cand_xy[cand_off[i] .. cand_off[i+1]) (x, y pairs); valid may be NULL.
 * Writes out[n] (matched: the winning attempt's record; unmatched: track = uv or (0, 0) when not
 * valid, offset and info 0, status 0), winner[n] (-1 = none) and stats[4] = {matched, rounds run,
 * attempts, 0}. */
void or_stereo_scan(int levels, const int* ws, const int* hs, const float* const* prim_gx,
                    const float* const* prim_gy, const float* const* prim_img, const float* const* sec_img,
                    const float* uv, const uint8_t* valid, int n, const int32_t* cand_off, const float* cand_xy,
                    float search_radius, float ncc_threshold, float early_exit_fraction, int horizontal, int mode,
                    or_track_data* out, int32_t* winner, int32_t* stats);

/* Affine (Shi-Tomasi) tracker (st_oracle.c): st_track_kernel, st_build_cache_kernel and
 * st_track_with_cache_kernel (libs/cuda_modules/cuda_kernels/st_tracker.cu).  The cache entry is
 * PointCacheData<float, 9> (cuda_kernels.h:68-74). */
typedef struct {
  float patch[81 * 10];
  float patch_sums[10];
  uint32_t level_mask;
} or_st_cache;
int or_st_qr_solve(int D, const float* a, const float* b, float* x);
void or_st_track(int levels, const int* ws, const int* hs, const float* const* prev_img, const float* const* cur_img,
                 const float* const* cur_gx, const float* const* cur_gy, or_track_data* td, int n, int n_shift,
                 int n_full, int mode);
void or_st_track_cached(int levels, const int* ws, const int* hs, const float* const* cur_img,
                        const float* const* cur_gx, const float* const* cur_gy, const or_st_cache* cache,
                        or_track_data* td, int n, int n_shift, int n_full, int mode);
void or_st_build_cache(int levels, const int* ws, const int* hs, const float* const* prev_img, or_track_data* td, int n,
                       or_st_cache* cache, int mode);

/* FP64 differentiable LK tracker and its adjoint (lk_adjoint64.c). */
enum { OR64_IMPLICIT = 0, OR64_UNROLLED = 1 };
typedef struct or64_cam or64_cam;
or64_cam* or64_cam_create(int w, int h, int max_levels);
void or64_cam_destroy(or64_cam* c);
int or64_cam_levels(const or64_cam* c);
void or64_cam_set(or64_cam* c, const double* prev0, const double* cur0);
void or64_cam_plane(const or64_cam* c, int level, int plane, double* out);
void or64_track(const or64_cam* c, const or_track_data* in, int n, int mode, int iters, double tol, double* out_xy,
                uint8_t* status);
void or64_backward(or64_cam* c, const or_track_data* in, int n, int mode, int iters, double tol,
                   const double* grad_xy, double* grad_prev0, double* grad_cur0, double* grad_track,
                   double* grad_offset);
void or64_debug_skip_pyramid_adjoint(int on);
void or64_cam_adjoint_plane(const or64_cam* c, int level, int plane, double* out);
void or64_fd(or64_cam* c, const double* prev0, const double* cur0, const or_track_data* in, int n, int mode,
             int iters, double tol, const double* gt, const uint8_t* mask, int nq, const int* which,
             const int64_t* index, double h, double* out, int strict);

#ifdef __cplusplus
}
#endif
#endif
