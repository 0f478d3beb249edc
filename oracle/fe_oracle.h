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
 * plus an FP64 LK (or_lk_track_f64) used only to state per-track error.
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

#ifdef __cplusplus
}
#endif
#endif
