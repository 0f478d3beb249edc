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
  int tiles_x, tiles_y;
  int tile_begin;           // first CTA of this job in the launch
  Level out[3];             // out[k] = level s + k; out[0] describes level s
};

struct StageBatch {
  int njobs;
  int* status;              // device flags: bit 0 = a TMA wait ran out (tile skipped)
  StageJob job[kMaxCams];
};

int stage_tile(bool u8, int nl);  // deepest-level core tile edge of a stage kind
// Encodes the uint8 frame's tensor map into job.tmap; returns false when the frame does not meet
// TMA alignment (the stage then stages its tile with ordinary loads).
bool encode_frame_tmap(StageJob& job);
cudaError_t pyramid_init();  // kernel attributes; call once per device before capture
cudaError_t launch_pyramid_stage(const StageBatch& b, int tiles, bool u8, int nl, cudaStream_t s);

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
};

struct SelectBatch {
  int ncams;
  int debug;
  SelectCam cam[kMaxCams];
};

constexpr int kMaxSelectKeys = 16384;  // shared-memory sort capacity of the selection kernels
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
  int n;
  int begin;                    // first track of this camera in the flattened list
};

struct LkLaunch {
  const LkCam* cams;            // device array (batched) or nullptr
  int* counter;                 // device track counter (persistent warps), or nullptr: one warp per track
  int ncams;
  int total;
  int horizontal;
  int sampling;
  LkCam single;                 // used when cams == nullptr
};

cudaError_t launch_lk(const LkLaunch& p, cudaStream_t s);

}  // namespace fe
