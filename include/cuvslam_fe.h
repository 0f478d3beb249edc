/* cuvslam_fe.h - C ABI of the B200-native visual-tracking front-end.
 *
 * The library replaces the hot path that cuVSLAM's MonoSOFGPU drives through four host wrappers
 * and the C-style kernel launchers of libs/cuda_modules:
 *   Gaussian image pyramid + gradient pyramid, Shi-Tomasi (GFTT) response and feature selection,
 *   pyramidal Lucas-Kanade tracking, and the affine (Shi-Tomasi) tracker,
 * with results equal to the reference GPU path (see each entry point).  All entry points:
 *   - take device pointers, sizes in elements/pixels and pitches in BYTES;
 *   - enqueue work on the caller's stream and return without synchronising, unless stated;
 *   - return an fe_status code and never throw across the ABI.
 * A context, a batch or an adjoint plan is used by one host thread at a time, as the reference's
 * wrapper objects are (not thread-safe per object); distinct contexts are independent.  Entries
 * that share state across streams say so (fe_select, fe_select_noalloc, the affine tracker).
 * Citations are to cuVSLAM 18.0.0 (libs/...).
 */
#ifndef CUVSLAM_FE_H
#define CUVSLAM_FE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define FE_API __attribute__((visibility("default")))
#else
#define FE_API
#endif

#define FE_MAX_LEVELS 10 /* PYRAMID_LEVELS, cuda_kernels.h:29 */
#define FE_ABI_VERSION 1

typedef enum {
  FE_OK = 0,
  FE_ERR_INVALID_ARGUMENT = 1, /* null pointer, bad size, misaligned pitch, ... */
  FE_ERR_CUDA = 2,             /* a CUDA runtime call failed; see fe_last_cuda_error() */
  FE_ERR_OUT_OF_MEMORY = 3,
  FE_ERR_CAPACITY = 4,         /* a documented size limit was exceeded */
  FE_ERR_DEVICE_FAULT = 5,     /* a kernel reported a bounded wait that ran out or a bad work item */
} fe_status;

typedef struct CUstream_st* fe_stream; /* identical to cudaStream_t */
typedef struct fe_context fe_context;
typedef struct fe_batch fe_batch;

/* One image pyramid and its gradient pyramid in device memory.  Level l has width[l] x height[l]
 * FP32 pixels for image, grad_x and grad_y, rows pitch_bytes[l] apart (a multiple of 16).
 * Level sizes follow the reference: (d+1)/2 while both sides stay >= 15, at most FE_MAX_LEVELS
 * (GPUImagePyramid::prepare_levels, image_pyramid.h:136-151; ScaleDownDim, image_pyramid.cpp:24).
 * Replaces GaussianGPUImagePyramid + GPUGradientPyramid (image_pyramid.h:56-162,
 * gradient_pyramid.h:30-59). */
typedef struct {
  int32_t levels;
  int32_t width[FE_MAX_LEVELS];
  int32_t height[FE_MAX_LEVELS];
  int64_t pitch_bytes[FE_MAX_LEVELS];
  float* image[FE_MAX_LEVELS];
  float* grad_x[FE_MAX_LEVELS];
  float* grad_y[FE_MAX_LEVELS];
} fe_pyramid;

/* cuvslam::cuda::TrackData, byte-for-byte (cuda_kernels.h:76-87): 80 bytes, 16-byte aligned.
 * Inputs: track (previous position, texture coordinates), offset (predicted motion),
 * search_radius_px (< 0 disables the track), ncc_threshold.  Outputs: track (new position, only
 * written when tracked), track_status, info (= diag(1/9)).  Other fields are not touched. */
typedef struct {
  float track[2];
  float offset[2];
  float info[4];
  uint8_t track_status;
  uint8_t reserved0[3];
  int32_t cache_index;
  float reserved1[2];
  float initial_guess_map[4];
  float search_radius_px;
  float ncc_threshold;
  float ncc;
  float reserved2;
} fe_track_data;

/* Bilinear sampling of LK patches. */
typedef enum {
  FE_SAMPLE_TEXTURE = 0,      /* cudaFilterModeLinear's 8-bit-fraction weights, FP32 multiply-add chain:
                                 matches the reference to well under 0.01 px */
  FE_SAMPLE_EXACT = 1,        /* exact FP32 weights (differentiable; used by the adjoint) */
  FE_SAMPLE_TEXTURE_WIDE = 2, /* the texture weights with each 4-tap sum rounded to FP32 once (FP64
                                 arithmetic), as the texture unit does: equals the hardware's samples
                                 more often, so marginal accept/reject decisions follow the reference */
  FE_SAMPLE_HARDWARE = 3,     /* the texture unit itself (linear filtering on texture objects the
                                 library creates for the pyramid planes, as the reference samples):
                                 LK only (fe_track, fe_track_mono, batches).  Planes must start on the
                                 device's texture alignment (512 bytes) with pitches on its texture
                                 pitch alignment (32 bytes), as fe_pyramid_init lays them out in
                                 512-byte aligned memory.  The context keeps a texture object per
                                 plane it tracked on until fe_destroy, at most 4096 (then
                                 FE_ERR_CAPACITY): reuse pyramids.  Equals the reference's
                                 lk_track_kernel bit for bit on the test frames (the same samples,
                                 arithmetic and summation order); not bit-identical to the
                                 emulations above.  The host wrappers' default */
} fe_sampling;

/* ---------------------------------------------------------------------------------------- */
/* Library                                                                                   */
/* ---------------------------------------------------------------------------------------- */

/* ABI version and status names: no counterpart in the reference, whose wrappers throw through
 * CUDA_CHECK (cuda_helper.h:42-56) where these entries return an fe_status. */
FE_API int fe_abi_version(void);
FE_API const char* fe_status_string(int status);
/* The CUDA error behind the last FE_ERR_CUDA on this thread (0 if none). */
FE_API int fe_last_cuda_error(void);

/* Context: owns the scratch memory of selection and batching on one device.  The device must be
 * current on the calling thread for every call that takes the context.
 * Replaces the per-wrapper state of GPUSelection / GPULKFeatureTracker (selection_v2.h:28-58,
 * lk_tracker.h:27-37) and the lazy init_* constant uploads (image_pyramid.cu:33-54, ...). */
FE_API int fe_create(int device, fe_context** out);
FE_API int fe_destroy(fe_context* ctx);

/* Device-side failure reporting.  The reference throws on every failed CUDA call (CUDA_CHECK,
 * cuda_helper.h:42-56) and has no kernel that waits on another; this library's single-launch
 * pyramid does wait (a tile for its TMA copy, a deeper level for the tiles it reads), each wait
 * bounded.  A wait that runs out skips its work and sets a flag in the context's device status word
 * instead of hanging: bit 0 = a tile's staging copy did not arrive (the tile is not written), bit 1 =
 * a deeper-level item gave up waiting for its inputs (its levels are not written), bit 2 = a
 * batch's response tile gave up waiting for its gradient window's TMA copy (its cells and sums are
 * not written).  Every pyramid launched through this context (fe_build_pyramid*, batches, adjoint
 * plans) and every batch's selection reports there.
 * fe_device_status synchronises `stream`, copies the word to *flags (may be NULL), clears it and
 * returns FE_ERR_DEVICE_FAULT when any flag was set, FE_OK otherwise. */
FE_API int fe_device_status(fe_context* ctx, fe_stream stream, int32_t* flags);
/* Iteration limit of those bounded waits for launches planned after this call (pyramid builds;
 * batches and adjoint plans created afterwards).  Default 4194304 (a few hundred milliseconds at
 * most).  0 makes every such wait give up at once, which exercises the failure path without a
 * fault: the kernels still finish and fe_device_status reports the flags. */
FE_API int fe_set_wait_limit(fe_context* ctx, int iterations);

/* ---------------------------------------------------------------------------------------- */
/* Pyramid                                                                                   */
/* ---------------------------------------------------------------------------------------- */

/* Number of levels of a width x height pyramid capped at max_levels (0 on bad arguments), by
 * GPUImagePyramid::prepare_levels (image_pyramid.h:136-151). */
FE_API int fe_pyramid_levels(int width, int height, int max_levels);
/* Bytes of device memory one pyramid (image + grad_x + grad_y, all levels) needs in this
 * library's layout (planes at multiples of 512 bytes from the start, rows padded to 256 bytes).
 * With fe_pyramid_init it replaces the pyramids ImageContext allocates at init
 * (image_context.h:101-104). */
FE_API int64_t fe_pyramid_bytes(int width, int height, int max_levels);
/* Lays a pyramid out in caller-provided device memory of at least fe_pyramid_bytes() bytes
 * (256-byte aligned; 512-byte aligned memory also suits FE_SAMPLE_HARDWARE's texture objects).
 * Host-only; allocates nothing. */
FE_API int fe_pyramid_init(void* device_memory, int64_t bytes, int width, int height, int max_levels, fe_pyramid* out);

/* Builds every level and both gradient images of `pyr` from a uint8 grayscale image in device
 * memory.  Results are bit-identical to the reference's
 *   cast_image (image_cast.cu:24-36) + GaussianGPUImagePyramid::build (image_pyramid.h:81-98,
 *   gaussian_scaling_kernel image_pyramid.cu:56-102) + GPUGradientPyramid::set
 *   (gradient_pyramid.cpp:83-118, conv_grad_x/y convolutions.cu:74-139).
 * `pyr` must describe width x height at level 0.  box3 = 1 applies the reference's box prefilter
 * first (GaussianGPUImagePyramid::build with blur_filter, CudaBoxPrefilter::prefilter,
 * box_prefilter.cpp:31-38): done on each tile inside the same kernel.
 * One launch builds every level (the last CTA of the levels 0-2 pass computes the deeper ones, with
 * one of the context's 64 completion counters, used in turn: at most 64 builds in flight per context). */
FE_API int fe_build_pyramid(fe_context* ctx, const uint8_t* image, int64_t image_pitch_bytes, int width, int height,
                     int box3, const fe_pyramid* pyr, fe_stream stream);
/* Same from an RGB8 frame (3 bytes per pixel, rows image_pitch_bytes apart): level 0 is the
 * reference's gray conversion (cast_image_rgb, image_cast.cu:52-70, as ImageContext::
 * build_gpu_image_pyramid does for RGB8 sources, image_context.cpp:215-240), box prefiltered when
 * box3 = 1, computed by one input kernel straight into level 0; then the FP32 stages. */
FE_API int fe_build_pyramid_rgb(fe_context* ctx, const uint8_t* image, int64_t image_pitch_bytes, int width,
                                int height, int box3, const fe_pyramid* pyr, fe_stream stream);
/* Same from an FP32 level-0 image (rows pitch_bytes apart): GaussianGPUImagePyramid::build of a
 * float GPUImageT (image_pyramid.h:81-98) + GPUGradientPyramid::set (gradient_pyramid.cpp:83-118). */
FE_API int fe_build_pyramid_f32(fe_context* ctx, const float* image, int64_t image_pitch_bytes, int width, int height,
                         const fe_pyramid* pyr, fe_stream stream);

/* ---------------------------------------------------------------------------------------- */
/* Selection                                                                                 */
/* ---------------------------------------------------------------------------------------- */

/* Shi-Tomasi response on level 0 of `pyr`, 3x3 non-maximum suppression, 9x9 suppression around
 * the n_alive alive features, one candidate per 8x8 cell above 1e-2 refined to sub-pixel, and the
 * per-bin (8x8 bins) quota apportioned by response strength; writes at most num_desired new
 * features (x, y pairs) to out_xy and their number to *out_count (both device memory).
 * Equals GPUSelection::computeGFTTAndSelectFeatures (selection_v2.cpp:27-184) with a total order
 * where the reference is nondeterministic: keypoints are ordered by strength, ties by cell raster
 * index, and each bin sum adds its 16x16 sub-tile sums row by row (left to right within a row,
 * then the row sums top to bottom).
 * mask (optional, device, width x height, non-zero = masked) and alive_xy (device, n_alive
 * x,y pairs) may be NULL.  Asynchronous; no host synchronisation.
 * One context runs one selection at a time: calls on different streams must use different contexts.
 * Limits: width, height <= 4096; num_desired <= 16384. */
FE_API int fe_select(fe_context* ctx, const fe_pyramid* pyr, int border_top, int border_bottom, int border_left,
              int border_right, const uint8_t* mask, int64_t mask_pitch_bytes, const float* alive_xy, int n_alive,
              int num_desired, float* out_xy, int32_t* out_count, fe_stream stream);

/* fe_select without a context and without allocating: for callers that cannot call cudaMalloc
 * while they run (a tracking loop with a per-frame deadline that reserves all memory at start-up,
 * where cudaMalloc's device synchronisation and unbounded latency would break the deadline, or a
 * process whose device memory all belongs to its own pool allocator).  No counterpart in the
 * reference: it has no allocation-free selection.
 * Scratch is a static device array of about 1.5 MB inside the library, held by every GPU that
 * loads it until the process exits.  Limits: width, height <= 2048 (FE_ERR_CAPACITY beyond), and
 * within that fe_select's own limits (num_desired <= 16384; at most 16384 kept candidates, i.e.
 * min(width/8 * height/8, n_alive + num_desired + 64) <= 16384).  Level-0 planes must be 16-byte
 * aligned, as fe_select requires.  The first call on a device sets up that device (looks up the
 * array's device address, sets kernel attributes) and must come before any stream capture on it:
 * a first call made while `stream` captures returns FE_ERR_INVALID_ARGUMENT and enqueues nothing.
 * All calls share the one array and each starts by clearing the part that must start at zero:
 * calls whose GPU work overlaps (other streams, other host threads) race and must be serialised by
 * the caller.  Results equal fe_select's bit for bit. */
FE_API int fe_select_noalloc(const fe_pyramid* pyr, int border_top, int border_bottom, int border_left,
                             int border_right, const uint8_t* mask, int64_t mask_pitch_bytes, const float* alive_xy,
                             int n_alive, int num_desired, float* out_xy, int32_t* out_count, fe_stream stream);

/* Diagnostic outputs of the last fe_select on this context (device pointers, valid until the
 * next fe_select): the response map (level-0 size, pitch = width*4) and the NMS map, the buffers
 * GPUSelection keeps as members (selection_v2.h:28-58). */
FE_API int fe_select_debug(fe_context* ctx, const float** response, const float** nms);

/* ---------------------------------------------------------------------------------------- */
/* Lucas-Kanade                                                                              */
/* ---------------------------------------------------------------------------------------- */

/* Pyramidal LK of n tracks from `prev` (image + gradients) to `cur` (image), updating `tracks`
 * in place (device memory).  One warp per track.  With FE_SAMPLE_TEXTURE the results agree with
 * the reference's lk_track_kernel (lk_tracker.cu:69-379, launched by
 * GPULKFeatureTracker::track_points, cuda_modules/lk_tracker.cpp:24-73) to well under 0.01 px;
 * horizontal != 0 selects lk_track_horizontal_kernel (lk_tracker.cu:381-665). */
FE_API int fe_track(fe_context* ctx, const fe_pyramid* prev, const fe_pyramid* cur, fe_track_data* tracks, int n,
             int horizontal, int sampling, fe_stream stream);

/* MonoSOFGPU::launch's two LK passes as MonoSOFGPU::collect merges them (sof_mono_gpu.cpp:34-104):
 * each track with its record's ncc_threshold (0.8 in the reference), and the tracks that pass lost
 * again from the same inputs with retrack_ncc (0.85); a record ends with the first pass's result if
 * it tracked, else the retrack's.  The records keep their own ncc_threshold. */
FE_API int fe_track_mono(fe_context* ctx, const fe_pyramid* prev, const fe_pyramid* cur, fe_track_data* tracks,
                         int n, float retrack_ncc, int sampling, fe_stream stream);

/* ---------------------------------------------------------------------------------------- */
/* Affine (Shi-Tomasi) tracker                                                               */
/* ---------------------------------------------------------------------------------------- */

/* cuvslam::cuda::PointCacheData<float, 9> (cuda_kernels.h:68-74), byte-for-byte: a track's
 * previous-frame 9x9 patches on up to FE_MAX_LEVELS levels (81 floats per level, row-major), their
 * sums, and the mask of the levels whose patch lies inside the image. */
typedef struct {
  float patch[81 * FE_MAX_LEVELS];
  float patch_sums[FE_MAX_LEVELS];
  uint32_t level_mask;
} fe_affine_cache;

/* st_track (st_tracker.cu:1397-1409, kernel st_track_kernel st_tracker.cu:320-814; host wrapper
 * GPUSTFeatureTracker::track_points, cuda_modules/st_tracker.cpp:24-78): affine tracking of n
 * tracks from `prev` (image) to `cur` (image + gradients), in place.  n_shift_iterations
 * translation-only Gauss-Newton steps, then n_full_iterations steps of the full 2x2 map + shift
 * (the reference's GPUSTFeatureTracker runs 0 and 20).  Uses the records' offset (predicted
 * motion), initial_guess_map (row-major 2x2; identity for a plain track), search_radius_px and
 * ncc_threshold; writes track, track_status, info and, when tracked, ncc.  Persistent warps take
 * tracks from a counter the context owns: affine tracking calls on one context must not overlap on
 * the GPU (use one stream per context). */
FE_API int fe_track_affine(fe_context* ctx, const fe_pyramid* prev, const fe_pyramid* cur, fe_track_data* tracks,
                           int n, int n_shift_iterations, int n_full_iterations, int sampling, fe_stream stream);

/* st_build_cache (st_tracker.cu:1386-1395, kernel st_tracker.cu:1298-1371): each track's
 * previous-frame patches from `prev` into cache[i] and cache_index = i.  cache holds n entries. */
FE_API int fe_affine_build_cache(fe_context* ctx, const fe_pyramid* prev, fe_track_data* tracks, int n,
                                 fe_affine_cache* cache, int sampling, fe_stream stream);

/* st_track_with_cache (st_tracker.cu:1373-1384, kernel st_tracker.cu:816-1296): as fe_track_affine
 * with the previous patches read from cache[tracks[i].cache_index] (-1: not tracked).  `cache`
 * holds n_cache entries; a track whose cache_index is outside [0, n_cache) is not tracked. */
FE_API int fe_track_affine_cached(fe_context* ctx, const fe_pyramid* cur, const fe_affine_cache* cache, int n_cache,
                                  fe_track_data* tracks, int n, int n_shift_iterations, int n_full_iterations,
                                  int sampling, fe_stream stream);

/* ---------------------------------------------------------------------------------------- */
/* Track filters after LK (MonoSOFGPU::finish, on the device)                                */
/* ---------------------------------------------------------------------------------------- */

/* Options of the filters MonoSOFGPU::finish applies after tracking (sof_mono_gpu.cpp:144-170).
 * Device pointers. */
typedef struct {
  float retrack_ncc;          /* batched step: > 0 runs the retrack pass of fe_track_mono */
  uint32_t* age;              /* n track ages (in/out; 0 = dead): required */
  const float* predicted;     /* n x 2 predicted positions (NaN x = none), or NULL (no predictor) */
  const uint8_t* mask;        /* nonzero = masked pixel, or NULL */
  int64_t mask_pitch_bytes;
  int32_t collapse;           /* 1: collapseTracks (the reference always applies it) */
  int32_t* alive_count;       /* out: tracks alive after the filters, or NULL */
} fe_track_finish;

/* One camera's tracks after LK. */
typedef struct {
  fe_track_data* tracks;      /* n records (in/out): dead tracks get track_status = 0 */
  int32_t n;
  int32_t width, height;      /* level-0 size */
  int32_t border[4];          /* top, bottom, left, right */
  fe_track_finish opts;       /* retrack_ncc is ignored here */
} fe_finish_camera;

/* The filters of MonoSOFGPU::finish for ncams (<= 64) cameras in one launch, in its order: collect
 * and age (an alive track whose record tracked ages by one, else dies; sof_mono_gpu.cpp:80-104,
 * sof_mono_base.cpp:111-118), the prediction-error filter (sof_mono_base.cpp:51-109: with at least 3
 * alive predicted tracks, those farther from their prediction than max(3, 2 x the median distance)
 * die), KillTracksOnBorder (selector_stereo.cpp:109-125), KillTracksWithinMask
 * (sof_mono_base.cpp:121-133) and collapseTracks (sof_mono_gpu.cpp:249-280: per 3x3-pixel cell the
 * first track with the cell's largest age survives).  Not on the device: the RANSAC filter (off by
 * default), keyframe selection and the track list's compaction.  Collapse scratch lives in the
 * context (grown on demand: make the first call at the largest size before capturing). */
FE_API int fe_finish_tracks(fe_context* ctx, const fe_finish_camera* cams, int ncams, fe_stream stream);

/* ---------------------------------------------------------------------------------------- */
/* Left-to-right (primary -> secondary camera) matching                                      */
/* ---------------------------------------------------------------------------------------- */

/* Precomputed epipolar candidate table of one camera pair (EpipolarCurves, epipolar_curves.h:26-64):
 * for each corner (u, v) of the primary pyramid's top level, 0 <= u < width = top_width + 1,
 * 0 <= v < height = top_height + 1, a curve of secondary base-level positions.  Device memory. */
typedef struct {
  int32_t width, height;  /* corners per row, corner rows */
  float inv_scale;        /* 1 / 2^top_level */
  const int32_t* offsets; /* width * height + 1: corner (u, v)'s curve is xy[offsets[v*width+u] ..
                             offsets[v*width+u+1]) (x, y pairs) */
  const float* xy;
  int32_t max_length;     /* longest curve (a bound on the candidates of any point) */
} fe_epipolar_curves;

/* One primary -> secondary pair of a left-to-right match. */
typedef struct {
  const fe_pyramid* primary;   /* host descriptor: primary frame's image + gradient pyramid */
  const fe_pyramid* secondary; /* host descriptor: secondary frame's image pyramid */
  const float* uv;             /* device, n x 2: primary positions (base-level pixels) */
  const uint8_t* valid;        /* device, n, or NULL: 0 = the point has no candidates (the caller could
                                  not project it; the reference then reports track (0, 0)) */
  int32_t n;
  /* candidates: an explicit list (cand_offsets != NULL) or the pair's epipolar table (curves) */
  const int32_t* cand_offsets; /* device, n + 1: point i's candidates are cand_xy[cand_offsets[i] ..
                                  cand_offsets[i+1]) (secondary base-level x, y pairs) */
  const float* cand_xy;
  int32_t max_candidates;      /* with cand_offsets: the longest list (longer lists are cut, and
                                  stats[3] gets bit 0) */
  const fe_epipolar_curves* curves; /* host descriptor, used when cand_offsets == NULL:
                                       candidates interpolated as EpipolarCurves::Candidates
                                       (epipolar_curves.cpp:64-101) */
  float search_radius;         /* search_radius_px of every attempt (CrossCamSearchRadius,
                                  sof_multicamera_base.cpp:31-37: 3 * 2^(top_level + 1)) */
  float ncc_threshold;         /* 0.8 in the reference */
  fe_track_data* out;          /* device, n records: the winning attempt's record; failed points
                                  get track = uv (or (0, 0) when not valid) and track_status = 0 */
  int32_t* winner;             /* device, n, or NULL: index of the winning candidate, -1 = none */
  int32_t* stats;              /* device, 4, or NULL: points matched, candidate rounds the
                                  reference would run, attempts tracked here, flags */
} fe_stereo_pair;

/* Left-to-right matching of npairs (<= 16) camera pairs in ONE launch: for each primary point, LK
 * from its position in the primary frame towards each of its candidates in turn, the first
 * candidate that tracks wins.  horizontal != 0: the 1-D tracker of rectified pairs
 * (lk_track_horizontal_kernel, lk_tracker.cu:381-665; lr_tracker = LKHorizontal); 0: the 2-D
 * tracker (lk_track_kernel, the default lr_tracker = LK; the primary pyramid needs grad_y).
 * Results equal MultiSOFGPU::LaunchTrackingPrimaryToSecondary (sof_multicamera_gpu.cpp:69-190),
 * which launches one tracking pass per candidate index k and synchronises after each, including
 * its early exit: after round k it stops once at least early_exit_fraction (kL2REarlyExitFraction
 * = 0.8, sof_multicamera_base.h:40) of the pair's points are matched, so points whose first
 * successful candidate comes after that round stay unmatched.  Here the (point, candidate)
 * attempts run in round order over persistent warps; an attempt is skipped once its point has an
 * earlier success or its round lies beyond a round that already met the early-exit count, so
 * the stop round and every result are those of the reference, whatever the scheduling.
 * Scratch (in the context) grows to the largest sum over pairs of n x max_candidates seen so far:
 * make the first call at the largest size before capturing a graph.  One call at a time per
 * context.  sampling as in fe_track. */
FE_API int fe_track_stereo(fe_context* ctx, const fe_stereo_pair* pairs, int npairs, float early_exit_fraction,
                           int horizontal, int sampling, fe_stream stream);

/* ---------------------------------------------------------------------------------------- */
/* Batched multi-camera frame step                                                           */
/* ---------------------------------------------------------------------------------------- */

/* One camera of a batched frame step.  All pointers are device memory except `prev`/`cur`,
 * which point to host descriptors. */
typedef struct {
  const uint8_t* image; /* current frame, uint8 grayscale */
  int64_t image_pitch_bytes;
  int32_t width, height;
  const fe_pyramid* prev; /* previous frame's pyramid (may be NULL on a first frame) */
  const fe_pyramid* cur;  /* pyramid to build from `image` */
  fe_track_data* tracks;  /* tracks to advance prev -> cur */
  int32_t n_tracks;
  int32_t num_desired;    /* tracks to maintain (num_desired_tracks): after LK, selection adds
                             max(0, num_desired - tracks LK kept) features (0 = no selection) */
  float* new_xy;          /* out: selected features, capacity num_desired */
  int32_t* new_count;     /* out */
  int32_t border[4];      /* top, bottom, left, right */
  const fe_track_finish* finish; /* host pointer, or NULL: MonoSOFGPU's retrack pass and finish
                                    filters between LK and selection (selection then keeps the
                                    survivors alive) */
} fe_camera_frame;

/* No counterpart in the reference, whose multi-camera rigs run one camera after another on
 * per-camera streams (MultiSOFBase::trackNextFrame, sof_multicamera_base.cpp:62-116).
 * Plans a batched frame step over ncams cameras: the pyramids of all cameras, LK of all tracks,
 * and selection on all cameras (alive features = tracks that LK kept), as a few launches over
 * flattened (camera, tile) and (camera, track) work lists, captured once into a CUDA graph.
 * The descriptors are copied; the device buffers they name must stay valid while the batch
 * lives.  sampling as in fe_track. */
FE_API int fe_batch_create(fe_context* ctx, const fe_camera_frame* cams, int ncams, int sampling, fe_batch** out);
/* Launches the planned step on `stream` (graph launch). */
FE_API int fe_batch_run(fe_batch* batch, fe_stream stream);

/* Parts of a batched step, for pipelining and measurement. */
typedef enum {
  FE_PART_PYRAMID = 0, /* pyramids of all cameras */
  FE_PART_TRACK = 1,   /* LK of all tracks (needs the pyramids) */
  FE_PART_SELECT = 2,  /* selection on all cameras (needs pyramids and LK) */
} fe_batch_part;
/* Enqueues one part of the planned step directly (no graph). */
FE_API int fe_batch_run_part(fe_batch* batch, int part, fe_stream stream);
/* Work counters of the batch's LK (no counterpart in the reference): runs the LK part once, from the
 * tracks as they are (they move as with fe_batch_run_part(FE_PART_TRACK)), with the kernel's own
 * per-track counting on, and adds to device_counts[0..2] (device memory, zeroed by the caller) the
 * number of pyramid levels at which a track was set up (previous patch and gradients sampled,
 * Hessian formed), of Gauss-Newton steps (current patch sampled, update solved) and of NCC
 * evaluations, over all tracks and both passes.  Timed steps never count.  Every sampling mode. */
FE_API int fe_batch_lk_work(fe_batch* batch, uint64_t* device_counts, fe_stream stream);
/* Number of kernel launches in one fe_batch_run (kernel nodes of the captured graph); -1 for a
 * NULL batch. */
FE_API int fe_batch_kernel_count(fe_batch* batch);
/* The same step as a plain per-camera sequence of fe_build_pyramid / fe_track / fe_select
 * (the drop-in launch pattern of MonoSOFGPU::track, sof_mono_gpu.cpp:106-137), for comparison. */
FE_API int fe_batch_run_plain(fe_batch* batch, fe_stream stream);
/* Autotuner: times the planned step (reps graph launches per candidate, after one warm-up) over
 *   the LK block shape (warps per block x minimum resident blocks: 8x4, 8x3, 4x8, 12x2),
 *   the response tiles after LK (0), on a second stream beside LK (1), beside the deeper
 *   pyramid stages and LK (2), before LK (3), or after LK with the LK survivors' burn applied in
 *   the tiles, which then need no pass over the burned cells (4),
 *   the generic pyramid stages' deepest-level tile (8 or 16) and the levels 0-2 kernel's register
 *   budget (2 or 3 CTAs per SM; stage_tile | 64 for 3),
 * one after the other (coordinate descent), keeps the fastest and re-captures the graph.  The
 * tracks are restored to their values before the call; the selection outputs hold the last run's.
 * Synchronises `stream`; allocates (call it before any capture of your own). */
FE_API int fe_batch_autotune(fe_batch* batch, int reps, fe_stream stream);
/* Sets the shapes directly (lk_shape 0..3 in the order above, overlap 0..4, stage_tile 8 or 16,
 * plus 64 for the three-CTA levels 0-2 kernel) and re-captures the graph. */
FE_API int fe_batch_set_tuning(fe_batch* batch, int lk_shape, int overlap, int stage_tile);
/* The shapes in use (defaults 0, 1, 8 until fe_batch_autotune runs). */
FE_API int fe_batch_tuning(const fe_batch* batch, int32_t* lk_shape, int32_t* overlap, int32_t* stage_tile);
FE_API int fe_batch_destroy(fe_batch* batch);

/* ---------------------------------------------------------------------------------------- */
/* Differentiable LK and its adjoint (no counterpart in the reference, which has no backward)  */
/* ---------------------------------------------------------------------------------------- */

/* The differentiable tracker is fe_track with FE_SAMPLE_EXACT and one of two iteration rules:
 *   FE_ADJOINT_IMPLICIT: the reference rule on every level (<= 11 steps, stop at |v| < 0.12 px,
 *     radius and NCC gates), then at level 0 up to `iterations` further steps c += v, stopping
 *     after the first with |v| < tolerance: the result is the fixed point e(c*) = 0 whose
 *     implicit-function-theorem derivative the adjoint takes.
 *   FE_ADJOINT_UNROLLED: exactly `iterations` (1..16) steps on every level, no early stop; a level
 *     is accepted when its last |v| < 0.12 px and the gates pass.  The adjoint differentiates every
 *     step, re-sampling the patches from the pyramids instead of storing them.
 * Pixel values are those of the pyramid (the reference tracker works at uint8 intensity scale:
 * its H carries +1 on the diagonal). */
typedef enum { FE_ADJOINT_IMPLICIT = 0, FE_ADJOINT_UNROLLED = 1 } fe_adjoint_mode;

/* One camera of a differentiable tracking step.  Pointers are device memory except prev/cur. */
typedef struct {
  const fe_pyramid* prev;          /* previous frame (image + gradients, e.g. fe_build_pyramid_f32) */
  const fe_pyramid* cur;           /* current frame, same level sizes */
  const fe_track_data* tracks_in;  /* forward input records (not modified) */
  fe_track_data* tracks_out;       /* forward output records; the implicit adjoint reads them */
  int32_t n_tracks;                /* <= 16384 */
  const float* grad_xy;            /* backward input, n x 2: dL/d(output track position) */
  float* grad_prev;                /* backward output: dL/d(level-0 previous image), written */
  int64_t grad_prev_pitch_bytes;
  float* grad_cur;                 /* backward output: dL/d(level-0 current image), written */
  int64_t grad_cur_pitch_bytes;
  float* grad_track;               /* n x 2 or NULL: dL/d(tracks_in position) */
  float* grad_offset;              /* n x 2 or NULL: dL/d(tracks_in offset); 0 in implicit mode */
  const float* prev_image;         /* optional level-0 FP32 frames that fe_adjoint_build_pyramids */
  const float* cur_image;          /*   turns into prev / cur, multiplied by image_scale on load */
  int64_t image_pitch_bytes;
  float image_scale;
} fe_adjoint_job;

typedef struct fe_adjoint fe_adjoint;

/* No counterpart in the reference (it has no backward).
 * Plans the differentiable step over njobs cameras (<= 64): allocates all scratch and copies the
 * descriptors once, so that forward and backward allocate nothing and can be captured into a CUDA
 * graph.  Failed tracks get zero gradients.  Deterministic: the per-pixel gradient sums run in a
 * fixed order (tracks in index order per 32x32 tile), no floating-point atomics. */
FE_API int fe_adjoint_create(fe_context* ctx, const fe_adjoint_job* jobs, int njobs, int mode, int iterations,
                             float tolerance, fe_adjoint** out);
/* Builds prev and cur of every job that names its frames (prev_image, cur_image) as
 * fe_build_pyramid_f32 would from image_scale * frame, all jobs in the same few launches. */
FE_API int fe_adjoint_build_pyramids(fe_adjoint* adj, fe_stream stream);
/* The differentiable tracker over all jobs: tracks_in -> tracks_out (one launch).  In unrolled
 * mode it also records every level's iterates for the backward. */
FE_API int fe_adjoint_forward(fe_adjoint* adj, fe_stream stream);
/* The vector-Jacobian product over all jobs: grad_xy -> grad_prev, grad_cur, grad_track,
 * grad_offset.  Reads the pyramids, so they must hold the forward's frames (rebuilt or kept).
 * Unrolled mode uses the iterates the plan's last forward recorded; before any forward it replays
 * the forward itself. */
FE_API int fe_adjoint_backward(fe_adjoint* adj, fe_stream stream);
/* Kernel launches of one forward (backward = 0), backward (1) or build_pyramids (2) call; -1 for a
 * NULL plan. */
FE_API int fe_adjoint_kernel_count(const fe_adjoint* adj, int backward);
/* Enqueues a copy, into the device int32 at `device_out`, of the number of tracks of the last
 * backward whose unrolled iterates on one level spread over more than 20 texels: those get NaN
 * position gradients and contribute nothing to the image gradients. */
FE_API int fe_adjoint_dropped(const fe_adjoint* adj, int32_t* device_out, fe_stream stream);
FE_API int fe_adjoint_destroy(fe_adjoint* adj);

/* One-camera conveniences (plan, run, synchronise the stream, free); no counterpart in the
 * reference. */
FE_API int fe_track_diff(fe_context* ctx, const fe_pyramid* prev, const fe_pyramid* cur,
                         const fe_track_data* tracks_in, fe_track_data* tracks_out, int n, int mode, int iterations,
                         float tolerance, fe_stream stream);
FE_API int fe_track_backward(fe_context* ctx, const fe_pyramid* prev, const fe_pyramid* cur,
                             const fe_track_data* tracks_in, const fe_track_data* tracks_out, int n, int mode,
                             int iterations, float tolerance, const float* grad_xy, float* grad_prev,
                             int64_t grad_prev_pitch_bytes, float* grad_cur, int64_t grad_cur_pitch_bytes,
                             float* grad_track, float* grad_offset, fe_stream stream);

#ifdef __cplusplus
}
#endif
#endif /* CUVSLAM_FE_H */
