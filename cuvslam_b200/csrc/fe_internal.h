// Host-visible job descriptors and launchers shared by the kernel files and the C ABI layer.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "fe_common.cuh"

namespace fe {

// ---------------------------------------------------------------- pyramid
struct alignas(64) StageJob {
  CUtensorMap tmap;         // uint8 frame (levels 0-2 stage, when use_tma)
  const void* src;          // level s: uint8 (s == 0) or float
  int64_t src_pitch_bytes;
  int src_w, src_h;
  int write_level0;         // also write level s (image cast + gradients): the uint8 stage
  int use_tma;              // frame meets TMA alignment (16-byte base and pitch)
  float scale;              // factor on the staged source (FP32 first stage; 1 otherwise)
  int box3;                 // levels 0-2 kernel: apply the box prefilter to the uint8 frame
  int tiles_x, tiles_y;
  int tile_begin;           // first CTA (queue position, when the launch has a queue) of this job's tiles
  Level out[3];             // out[k] = level s + k; out[0] describes level s
  // the levels after out[nl], computed by the job's last CTA from the complete out[nl]: at most two
  // small ones after a generic stage, all the remaining ones after the levels 0-2 kernel
  int tail_levels;
  int* done;                // the job's CTA counter (zero between launches; the last CTA resets it);
                            // levels 0-2 kernel: [0] tiles, [1] phase-3 bands, [2] phase-4 bands
  // levels 0-2 kernel: queue positions [q_deep, q_deep + deep_items) hold this job's deeper-level
  // items: deep_bands[p] band items of phase p (deep_band_rows[p] rows of tail[p + 1] each), then the
  // rest item from tail[deep_rest]
  int q_deep, deep_items, deep_rest;
  int deep_bands[2], deep_band_rows[2];
  Level tail[kMaxLevels - 3];
};

constexpr int kMaxStageJobs = 48;  // jobs per launch (the job table is a kernel parameter)

// Default iteration limit of the levels 0-2 kernel's bounded waits (a few hundred ms at most).
constexpr int kDefaultWaitLimit = 1 << 22;

struct StageBatch {
  int njobs;
  int wait_limit;           // iterations of a bounded wait before it gives up (0: at once)
  int* status;              // device flags: bit 0 = a TMA wait ran out (tile skipped), bit 1 = a
                            // deeper-level item's wait ran out (item skipped)
  int* queue;               // levels 0-2 kernel with deeper-level items: [0] next item, [1] CTAs
                            // finished (zero between launches), or nullptr: item = blockIdx.x
  StageJob job[kMaxStageJobs];
};
static_assert(sizeof(StageBatch) <= 32000, "stage job table exceeds the kernel parameter limit");

// kt: the generic stages' deepest-level tile (8 or 16), plus kL012Three to run the levels 0-2 kernel
// with registers for three CTAs per SM instead of two
constexpr int kL012Three = 64;
int stage_tile(bool u8, int nl, int kt);  // deepest-level core tile edge of a stage kind
constexpr int kTailFloats = 12 * 1024;  // shared-memory floats for a tail: the source level + one level
int l012_deep_floats();  // shared-memory floats a deeper-level item of the levels 0-2 kernel stages
// Encodes the uint8 frame's tensor map into job.tmap; returns false when the frame does not meet
// TMA alignment (the stage then stages its tile with ordinary loads).
bool encode_frame_tmap(StageJob& job);
// Encodes a 2-D FP32 plane's tensor map (w x h floats, rows pitch_floats apart) with a box of
// box_w x box_h floats; false when the driver entry point is missing or the plane does not meet TMA
// alignment (16-byte base and pitch).
bool encode_plane_tmap_f32(CUtensorMap* map, const float* base, int w, int h, int pitch_floats, int box_w, int box_h);
cudaError_t pyramid_init();  // kernel attributes; call once per device before capture
cudaError_t launch_pyramid_stage(const StageBatch& b, int tiles, bool u8, int nl, int kt, bool tail, cudaStream_t s);
// Level 0 of a pyramid from a uint8 mono (channels 1) or RGB8 (channels 3) frame: the reference's cast
// (gray = 0.299 r + 0.587 g + 0.114 b for RGB) and, with box3, its box prefilter; FP32 into dst.
cudaError_t launch_input_stage(const uint8_t* src, int64_t src_pitch, int channels, int box3, int w, int h,
                               float* dst, int64_t dst_pitch_floats, cudaStream_t s);

// ---------------------------------------------------------------- selection
struct SelectCam {
  // level-0 gradients
  const float* gx;
  const float* gy;
  int w, h, pitch;              // pitch in floats
  const uint8_t* mask;          // optional
  int64_t mask_pitch;
  const float* alive_xy;        // alive features as n_alive (x, y) pairs, or
  const fe_track_data* alive_tracks;  // n_alive tracks; alive = track_status != 0
  int n_alive;
  float* alive_out_xy;          // optional: compacted alive positions (capacity n_alive)
  int* stats;                   // [0] alive count, [1] quota total, [2] kept, [3] error flags,
                                // [4] new features wanted
  int num_desired;              // new features wanted, or
  int target_total;             // when > 0: wanted = max(0, target_total - alive count)
  int border[4];
  float* out_xy;
  int32_t* out_count;
  // scratch (device)
  float* resp;                  // w*h response map (batched path; single camera: debug only)
  float* nms;                   // w*h NMS map (burned pixels zeroed as the reference's)
  uint32_t* burn;               // ceil(w/32) * h bit mask of burned pixels
  uint32_t* touched;            // bit per 8x8 cell (ceil(w/8) x ceil(h/8)) reached by a burn window
  int touched_begin;            // first touched-mask word of this camera in the launch
  float* cell_m;                // (w/8)*(h/8) cell strength (0 = none)
  float2* cell_xy;              // refined position
  float* sub_sum;               // ceil(w/16)*ceil(h/16) sub-tile sums
  int* bin_want;                // 64 quotas + 64 counts
  uint64_t* q_keys;             // qualifying keys, capacity q_cap
  float2* q_xy;
  int q_cap;
  int tiles_x, tiles_y, tile_begin;  // 32x32 response tiles
  const CUtensorMap* grad_tmap;  // optional: [gx, gy] tensor maps (device memory, 64-byte aligned)
                                 // whose box is a response tile's gradient window: interior tiles
                                 // are then staged by TMA
};

struct SelectBatch {
  int ncams;
  int debug;
  int* status;     // device flags (bit 2: a response tile's TMA staging did not arrive; the tile
                   // is skipped), or null
  int wait_limit;  // iterations of that bounded wait
  SelectCam cam[kMaxCams];
};

constexpr int kMaxSelectKeys = 16384;  // shared-memory sort capacity of the selection kernels
// The [gx, gy] tensor maps of a camera's level-0 gradient planes with the response tile's gradient
// window as their box (SelectCam::grad_tmap); false when the planes do not meet TMA alignment.
bool encode_select_grad_tmaps(CUtensorMap* maps, const float* gx, const float* gy, int w, int h, int pitch_floats);
int select_tile_w();  // response tile (level-0 pixels)
int select_tile_h();
cudaError_t select_init();
// single-camera selection (burn before the response tiles; maps only when b.debug)
cudaError_t launch_select(const SelectBatch& b, int total_tiles, int bin_key_cap, int final_key_cap,
                          cudaStream_t s);
// batched selection in two parts: the response tiles (no dependency on tracking; writes the resp and
// nms maps) and, after tracking, the burn, the burned cells, quotas and order
cudaError_t launch_select_response(const SelectBatch& b, int total_tiles, cudaStream_t s);
cudaError_t launch_select_rest(const SelectBatch& b, int touched_words, int bin_key_cap, int final_key_cap,
                               cudaStream_t s);

// ---------------------------------------------------------------- LK
struct LkCam {
  Pyr prev;                     // image + gradients
  Pyr cur;                      // image
  fe_track_data* tracks;
  const fe_track_data* tracks_in;  // out-of-place input records, or nullptr (tracks in place)
  int n;
  int begin;                    // first track of this camera in the flattened list
  float retrack_ncc;            // > 0: tracks the first pass lost run again with this NCC threshold
};

// Iteration rule of a launch: the reference tracker, or the differentiable tracker (exact
// sampling) in one of its two adjoint modes.
constexpr int kLkReference = 0, kLkImplicit = 1, kLkUnrolled = 2;

namespace lk {
struct LkRecord;
}

// Texture objects of one camera's planes for FE_SAMPLE_HARDWARE (cudaTextureObject_t values).
struct LkTex {
  unsigned long long prev_img[kMaxLevels], prev_gx[kMaxLevels], prev_gy[kMaxLevels], cur_img[kMaxLevels];
};

struct LkLaunch {
  const LkCam* cams;            // device array (batched) or nullptr
  int* counter;                 // device track counter (persistent warps), or nullptr: one warp per track
  int ncams;
  int total;
  int horizontal;
  int sampling;
  int mode;                     // kLk*
  int iters;                    // implicit: refinement steps at level 0; unrolled: steps per level
  float tol2;                   // implicit: squared step below which the refinement stops
  int shape;                    // reference rule: block shape (kLkShapes), chosen by the batch autotuner
  lk::LkRecord* recs;           // unrolled: per-track records for the adjoint (may be null)
  LkCam single;                 // used when cams == nullptr
  const LkTex* texs;            // FE_SAMPLE_HARDWARE: device array parallel to cams, or nullptr
  LkTex single_tex;             // FE_SAMPLE_HARDWARE with cams == nullptr
  unsigned long long* counts;   // optional work counters (emulated sampling): [0] levels set up,
                                // [1] Gauss-Newton steps, [2] NCC evaluations, summed over tracks
};

cudaError_t launch_lk(const LkLaunch& p, cudaStream_t s);
// The reference rule with the texture unit's filtering (lk_hw.cu).
cudaError_t launch_lk_hw(const LkLaunch& p, cudaStream_t s);
constexpr int kLkShapes = 4;  // warps per block x minimum resident blocks: 8x4, 8x3, 4x8, 12x2

// ---------------------------------------------------------------- track filters after LK
struct FinishCam {
  fe_track_data* tracks;        // records after LK (status in, status 0 out for dead tracks)
  uint32_t* age;                // in/out, 0 = dead
  int n;
  const float* pred;            // n x 2 or nullptr; NaN x = no prediction
  int w, h;
  int border[4];                // top, bottom, left, right
  const uint8_t* mask;          // or nullptr
  int64_t mask_pitch;
  unsigned long long* cells;    // collapse: ceil(w/3) x ceil(h/3) keys, zero between launches; or nullptr
  int cw, ch;
  int* alive_count;             // optional
};

struct FinishBatch {
  int ncams;
  FinishCam cam[kMaxCams];
};

cudaError_t launch_finish(const FinishBatch& b, cudaStream_t s);

// ---------------------------------------------------------------- affine (Shi-Tomasi) tracker
struct StLaunch {
  Pyr prev;                     // image (track, build cache)
  Pyr cur;                      // image + gradients (track)
  fe_track_data* tracks;
  int n;
  int n_shift, n_full;          // translation-only, then full-map Gauss-Newton steps per level
  int sampling;
  const fe_affine_cache* cache; // cached tracking: entries indexed by cache_index
  int n_cache;
  fe_affine_cache* cache_out;   // build: n entries
  int* counter;                 // tracking: persistent warps' track counter (zeroed by the launch)
};

// kind 0: st_track, 1: st_track_with_cache, 2: st_build_cache
cudaError_t launch_st(const StLaunch& p, int kind, cudaStream_t s);

// ---------------------------------------------------------------- left-to-right matching
constexpr int kMaxStereoPairs = 16;

struct StereoPair {
  LkCam lk;                     // prev = primary (image + grad_x), cur = secondary (image)
  const float2* uv;
  const uint8_t* valid;         // optional
  int n;
  int begin;                    // first point of this pair in a round of the flattened list
  int maxc;                     // candidate rounds of this pair
  const int* cand_off;          // explicit candidates (n + 1 offsets), or nullptr: curves
  const float2* cand_xy;
  int cw, ch;                   // epipolar table: corners per row, corner rows
  float inv_scale;
  const int* c_off;
  const float2* c_xy;
  float radius, ncc_thr;
  float need;                   // early-exit count: frac * n
  fe_track_data* out;
  int* winner;                  // optional
  int* stats;                   // optional
  // scratch
  int* cnt;                     // [maxc]: points whose first success is at a round <= r (zeroed)
  int* attempts;                // attempts tracked (zeroed)
  unsigned* stop;               // earliest round known to meet the early-exit count (all ones)
  unsigned* best;               // [n]: lowest successful candidate index (all ones = none)
  float2* pos;                  // [n * maxc]: tracked position of each successful attempt
};

struct StereoLaunch {
  int npairs;
  int round;                    // points per round (sum of n)
  int rounds;                   // largest maxc
  int* counter;                 // attempt counter of the persistent warps (zeroed)
  int* done;                    // CTA counter (zeroed): the last CTA publishes the results
  int sampling;
  int horizontal;               // 1-D (x only) LK for rectified pairs
  StereoPair pair[kMaxStereoPairs];
};

cudaError_t launch_stereo(const StereoLaunch& p, cudaStream_t s);

// ---------------------------------------------------------------- LK adjoint
// Per-track gradient contributions are written as window records (slot = (plane q, level l, track g),
// q: 0 previous image, 1 previous grad_x, 2 previous grad_y, 3 current image), then summed per
// 32x32 tile of each plane in track order (a deterministic segmented reduction), then pushed through
// the gradient filters and the decimation, from the top level down.
struct AdjCam {
  LkCam lk;                          // pyramids, tracks_in (forward inputs), n, begin
  const fe_track_data* tracks_out;   // forward results (implicit mode reads position and status)
  const float* grad_xy;              // n x 2: dL/d(output position)
  float* grad_track;                 // n x 2 or null: dL/d(track position)
  float* grad_offset;                // n x 2 or null: dL/d(offset)
};

struct AdjLaunch {
  const AdjCam* cams;
  int ncams, total;
  int* counter;                      // persistent-warp track counter
  int mode, iters;                   // kLkImplicit / kLkUnrolled
  int L;                             // record levels (1 implicit; deepest pyramid unrolled)
  int cur_s;                         // current-image record edge: 12 implicit, 32 unrolled
  const lk::LkRecord* recs;          // unrolled: the forward's per-track records
  int4* hdr;                         // [4][L][total] {x0, y0, w, h}; w == 0: empty
  float* data_prev;                  // [3][L][total][12 * 12]
  float* data_cur;                   // [L][total][cur_s * cur_s]
  int* overflow;                     // tracks dropped because a level's iterates spread too far
};

struct AdjPlane {
  float* dst;                        // dense gradient plane (written whole)
  int pitch, w, h;                   // pitch in floats
  int tiles_x, tile_begin, ntiles;
};

struct AdjGather {
  const AdjPlane* planes;            // [(cam * 4 + q) * L + l]
  const AdjCam* cams;
  int nplanes, ncams, total_tiles, nslots, L, total, cur_s;
  const int4* hdr;
  const float* data_prev;
  const float* data_cur;
  int* count;                        // [total_tiles]
  int* off;                          // [total_tiles + 1]
  int* cursor;                       // [total_tiles]
  int* long_tiles;                   // tiles with more than 32 records ([total_tiles]), and their
  int* long_count;                   //   number
  int* list;
  int list_cap;                      // power of two >= the longest list (tracks of one camera)
};

struct AdjPyrJob {
  float* img;                        // in: summed records of the level; out: complete gradient
  const float* gx;                   // previous frame: gradient planes' adjoints (null: current frame)
  const float* gy;
  const float* up;                   // complete gradient of the next level (null at the top)
  int pitch, gpitch, up_pitch;
  int w, h, up_w, up_h;
  int px_begin;
};

struct AdjPyrLevel {
  int njobs, total_px;
  int max_blocks;                    // 128x8-pixel blocks of the largest job
  AdjPyrJob job[2 * kMaxCams];
};

cudaError_t adjoint_init();        // kernel attributes; call once per device before capture
int lk_max_unrolled();             // most steps per level the unrolled mode records
size_t lk_record_bytes();          // bytes of one track's unrolled-mode record
cudaError_t launch_lk_adjoint(const AdjLaunch& a, cudaStream_t s);
cudaError_t launch_adjoint_gather(const AdjGather& g, cudaStream_t s);
cudaError_t launch_pyramid_adjoint(const AdjPyrLevel& lv, cudaStream_t s);

}  // namespace fe
