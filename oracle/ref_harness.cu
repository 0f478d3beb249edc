// Test-only harness around the reference's own CUDA kernels (cuVSLAM libs/cuda_modules/cuda_kernels).
//
// This file is oracle infrastructure: it is compiled together with the reference's unmodified
// kernel sources (image_pyramid.cu, convolutions.cu, gftt.cu, selection_v2.cu, sort.cu,
// lk_tracker.cu) by oracle/build_ref.sh into oracle/_ref/libcuvslam_ref.so.  Only tests and the
// golden-fixture script load it; the product never does.
//
// It restates, in plain host code, the launch sequences of the reference host wrappers so that the
// reference kernels run exactly as cuVSLAM's MonoSOFGPU drives them:
//   - GPUImage<float> pitched storage + point/linear texture objects   (cuda_helper.h:297-300,402-431)
//   - ImageCast::cast (u8 upload + cast_image)                          (image_cast.cpp:33-47)
//   - GaussianGPUImagePyramid::build / prepare_levels                   (image_pyramid.h:81-98,136-151)
//   - cast_image_rgb + CudaBoxPrefilter::prefilter (RGB8 input, box3)   (image_context.cpp:215-240,
//                                                                        box_prefilter.cpp:31-38)
//   - GPUGradientPyramid::set                                           (gradient_pyramid.cpp:83-118)
//   - GPUSelection::computeGFTTAndSelectFeatures incl. host quota loop  (selection_v2.cpp:27-184)
//   - GPULKFeatureTracker::track_points                                 (cuda_modules/lk_tracker.cpp:24-73)
//   - MultiSOFGPU::LaunchTrackingPrimaryToSecondary's candidate scan    (sof/sof_multicamera_gpu.cpp:118-190)
// Every entry point takes and returns HOST buffers and synchronises; it is a checker, not fast.

#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <vector>

#include "cuda_modules/cuda_kernels/cuda_kernels.h"

using namespace cuvslam::cuda;

namespace {

constexpr int kMaxLevels = 10;
constexpr int kMinDim = 15;

#define HCHECK(x)                         \
  do {                                    \
    cudaError_t e_ = (x);                 \
    if (e_ != cudaSuccess) return (int)e_; \
  } while (0)

struct DevImage {
  float* ptr = nullptr;
  size_t pitch = 0;
  int w = 0, h = 0;
  cudaTextureObject_t tex_point = 0, tex_linear = 0;

  cudaError_t alloc(int cols, int rows) {
    w = cols;
    h = rows;
    cudaError_t e = cudaMallocPitch((void**)&ptr, &pitch, (size_t)cols * sizeof(float), rows);
    if (e != cudaSuccess) return e;
    cudaResourceDesc rd;
    memset(&rd, 0, sizeof(rd));
    rd.resType = cudaResourceTypePitch2D;
    rd.res.pitch2D.devPtr = ptr;
    rd.res.pitch2D.width = cols;
    rd.res.pitch2D.height = rows;
    rd.res.pitch2D.pitchInBytes = pitch;
    rd.res.pitch2D.desc = cudaCreateChannelDesc(32, 0, 0, 0, cudaChannelFormatKindFloat);
    cudaTextureDesc td;
    memset(&td, 0, sizeof(td));
    // Same descriptors as the reference's GPUImage::prepare_texture.
    td.addressMode[0] = cudaAddressModeMirror;
    td.addressMode[1] = cudaAddressModeMirror;
    td.filterMode = cudaFilterModePoint;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 0;
    e = cudaCreateTextureObject(&tex_point, &rd, &td, nullptr);
    if (e != cudaSuccess) return e;
    td.addressMode[0] = cudaAddressModeWrap;
    td.addressMode[1] = cudaAddressModeWrap;
    td.filterMode = cudaFilterModeLinear;
    return cudaCreateTextureObject(&tex_linear, &rd, &td, nullptr);
  }
  ~DevImage() {
    if (tex_point) cudaDestroyTextureObject(tex_point);
    if (tex_linear) cudaDestroyTextureObject(tex_linear);
    if (ptr) cudaFree(ptr);
  }
  cudaError_t upload(const float* host) {
    return cudaMemcpy2D(ptr, pitch, host, (size_t)w * 4, (size_t)w * 4, h, cudaMemcpyHostToDevice);
  }
  cudaError_t download(float* host) const {
    return cudaMemcpy2D(host, (size_t)w * 4, ptr, pitch, (size_t)w * 4, h, cudaMemcpyDeviceToHost);
  }
};

int level_count(int w, int h, int max_levels) {
  int n = 0;
  while (n < max_levels) {
    ++n;
    h = (h + 1) / 2;
    w = (w + 1) / 2;
    if (h < kMinDim || w < kMinDim) break;
  }
  return n;
}

struct Pyr {
  int n = 0;
  std::unique_ptr<DevImage> img[kMaxLevels], gx[kMaxLevels], gy[kMaxLevels];
};

int init_tables() {
  HCHECK(init_scaler());
  HCHECK(init_conv_kernels());
  HCHECK(init_gauss_coeffs());
  HCHECK(init_gauss_square_kernel());
  return 0;
}

// ImageCast::cast + GaussianGPUImagePyramid::build + GPUGradientPyramid::set.
int build(const uint8_t* host_u8, int w, int h, int max_levels, Pyr& p, cudaStream_t s);

// The same with the input options of ImageContext::build_gpu_image_pyramid (image_context.cpp:215-240):
// an RGB8 frame (cast_image_rgb) and the box prefilter of GaussianGPUImagePyramid::build
// (CudaBoxPrefilter::prefilter: box_blur_x, box_blur_y, copy_border with border 1).
int build_ex(const uint8_t* host, int w, int h, int rgb, int box3, int max_levels, Pyr& p, cudaStream_t s) {
  p.n = level_count(w, h, max_levels);
  int lw = w, lh = h;
  for (int l = 0; l < p.n; ++l) {
    p.img[l].reset(new DevImage);
    p.gx[l].reset(new DevImage);
    p.gy[l].reset(new DevImage);
    HCHECK(p.img[l]->alloc(lw, lh));
    HCHECK(p.gx[l]->alloc(lw, lh));
    HCHECK(p.gy[l]->alloc(lw, lh));
    lw = (lw + 1) / 2;
    lh = (lh + 1) / 2;
  }
  const int bpp = rgb ? 3 : 1;
  uint8_t* d_u8 = nullptr;
  size_t u8_pitch = 0;
  HCHECK(cudaMallocPitch((void**)&d_u8, &u8_pitch, (size_t)w * bpp, h));
  HCHECK(cudaMemcpy2D(d_u8, u8_pitch, host, (size_t)w * bpp, (size_t)w * bpp, h, cudaMemcpyHostToDevice));
  DevImage cast, buffer;
  HCHECK(cast.alloc(w, h));
  if (rgb)
    HCHECK(cast_image_rgb(d_u8, u8_pitch, cast.ptr, cast.pitch, {(unsigned)w, (unsigned)h}, s));
  else
    HCHECK(cast_image(d_u8, u8_pitch, cast.ptr, cast.pitch, {(unsigned)w, (unsigned)h}, s));
  if (box3) {
    HCHECK(init_box_prefilter_kernels());
    HCHECK(buffer.alloc(w, h));
    HCHECK(box_blur_x(cast.tex_point, {(unsigned)w, (unsigned)h}, buffer.ptr, buffer.pitch, s));
    HCHECK(box_blur_y(buffer.tex_point, {(unsigned)w, (unsigned)h}, p.img[0]->ptr, p.img[0]->pitch, s));
    HCHECK(copy_border(cast.tex_point, {(unsigned)w, (unsigned)h}, p.img[0]->ptr, p.img[0]->pitch, 1, s));
  } else {
    HCHECK(cudaMemcpy2DAsync(p.img[0]->ptr, p.img[0]->pitch, cast.ptr, cast.pitch, (size_t)w * 4, h,
                             cudaMemcpyDeviceToDevice, s));
  }
  for (int l = 0; l + 1 < p.n; ++l) {
    const DevImage& a = *p.img[l];
    DevImage& b = *p.img[l + 1];
    HCHECK(gaussian_scaling(a.tex_point, {(unsigned)a.w, (unsigned)a.h}, b.ptr, b.pitch,
                            {(unsigned)b.w, (unsigned)b.h}, s));
  }
  for (int l = 0; l < p.n; ++l) {
    const DevImage& a = *p.img[l];
    HCHECK(conv_grad_x(a.tex_point, {(unsigned)a.w, (unsigned)a.h}, p.gx[l]->ptr, p.gx[l]->pitch, s));
    HCHECK(conv_grad_y(a.tex_point, {(unsigned)a.w, (unsigned)a.h}, p.gy[l]->ptr, p.gy[l]->pitch, s));
  }
  HCHECK(cudaStreamSynchronize(s));
  cudaFree(d_u8);
  return 0;
}

int build(const uint8_t* host_u8, int w, int h, int max_levels, Pyr& p, cudaStream_t s) {
  p.n = level_count(w, h, max_levels);
  int lw = w, lh = h;
  for (int l = 0; l < p.n; ++l) {
    p.img[l].reset(new DevImage);
    p.gx[l].reset(new DevImage);
    p.gy[l].reset(new DevImage);
    HCHECK(p.img[l]->alloc(lw, lh));
    HCHECK(p.gx[l]->alloc(lw, lh));
    HCHECK(p.gy[l]->alloc(lw, lh));
    lw = (lw + 1) / 2;
    lh = (lh + 1) / 2;
  }
  uint8_t* d_u8 = nullptr;
  size_t u8_pitch = 0;
  HCHECK(cudaMallocPitch((void**)&d_u8, &u8_pitch, w, h));
  HCHECK(cudaMemcpy2D(d_u8, u8_pitch, host_u8, w, w, h, cudaMemcpyHostToDevice));
  DevImage cast;
  HCHECK(cast.alloc(w, h));
  HCHECK(cast_image(d_u8, u8_pitch, cast.ptr, cast.pitch, {(unsigned)w, (unsigned)h}, s));
  HCHECK(cudaMemcpy2DAsync(p.img[0]->ptr, p.img[0]->pitch, cast.ptr, cast.pitch, (size_t)w * 4, h,
                           cudaMemcpyDeviceToDevice, s));
  for (int l = 0; l + 1 < p.n; ++l) {
    const DevImage& a = *p.img[l];
    DevImage& b = *p.img[l + 1];
    HCHECK(gaussian_scaling(a.tex_point, {(unsigned)a.w, (unsigned)a.h}, b.ptr, b.pitch,
                            {(unsigned)b.w, (unsigned)b.h}, s));
  }
  for (int l = 0; l < p.n; ++l) {
    const DevImage& a = *p.img[l];
    HCHECK(conv_grad_x(a.tex_point, {(unsigned)a.w, (unsigned)a.h}, p.gx[l]->ptr, p.gx[l]->pitch, s));
    HCHECK(conv_grad_y(a.tex_point, {(unsigned)a.w, (unsigned)a.h}, p.gy[l]->ptr, p.gy[l]->pitch, s));
  }
  HCHECK(cudaStreamSynchronize(s));
  cudaFree(d_u8);
  return 0;
}

Pyramid make_pyr(const Pyr& p, std::unique_ptr<DevImage> const* arr) {
  Pyramid out;
  memset(&out, 0, sizeof(out));
  out.levels = p.n;
  for (int l = 0; l < p.n; ++l) {
    out.level_tex[l] = arr[l]->tex_linear;
    out.level_sizes[l] = {arr[l]->w, arr[l]->h};
  }
  return out;
}

}  // namespace

extern "C" {

int ref_level_count(int w, int h, int max_levels) { return level_count(w, h, max_levels); }

// Pyramid + gradient pyramid of one u8 image.  Outputs are packed level after level
// (level l holds w_l*h_l floats, row-major, no padding).
int ref_pyramid(const uint8_t* img, int w, int h, int max_levels, int* nlev, float* levels, float* gx, float* gy) {
  int rc = init_tables();
  if (rc) return rc;
  Pyr p;
  rc = build(img, w, h, max_levels, p, 0);
  if (rc) return rc;
  *nlev = p.n;
  size_t off = 0;
  for (int l = 0; l < p.n; ++l) {
    HCHECK(p.img[l]->download(levels + off));
    HCHECK(p.gx[l]->download(gx + off));
    HCHECK(p.gy[l]->download(gy + off));
    off += (size_t)p.img[l]->w * p.img[l]->h;
  }
  return 0;
}

// GPUSelection::computeGFTTAndSelectFeatures on level 0 of the pyramid of `img`.
// Intermediate buffers are returned for stage-by-stage comparison:
//   gftt[w*h], nms[w*h] (after filter_maximums), cell_max[cw*ch], cell_idx[cw*ch*2] (x,y),
//   kp[cap*3] sorted keypoints (x,y,strength) with *n_kp entries, bins[64],
//   sel[num_desired*2] selected features with *n_sel entries.
int ref_select(const uint8_t* img, int w, int h, const float* alive_xy, int n_alive, int num_desired, int border_top,
               int border_bottom, int border_left, int border_right, float* gftt, float* nms, float* cell_max,
               uint32_t* cell_idx, float* kp_out, int* n_kp, float* bins_out, float* sel, int* n_sel) {
  int rc = init_tables();
  if (rc) return rc;
  Pyr p;
  rc = build(img, w, h, 1, p, 0);
  if (rc) return rc;
  cudaStream_t s = 0;
  const uint2 size = {(unsigned)w, (unsigned)h};
  const uint2 bin_size = {(unsigned)(w / 8), (unsigned)(h / 8)};
  const uint2 num_bins = {8, 8};
  const uint2 ds = {(unsigned)w / 8, (unsigned)h / 8};
  const int max_tracks = (int)(ds.x * ds.y);

  DevImage val, maxim, dsm;
  HCHECK(val.alloc(w, h));
  HCHECK(maxim.alloc(w, h));
  HCHECK(dsm.alloc((int)ds.x, (int)ds.y));
  uint2* idx = nullptr;
  size_t idx_pitch = 0;
  HCHECK(cudaMallocPitch((void**)&idx, &idx_pitch, ds.x * sizeof(uint2), ds.y));
  Keypoint* kp = nullptr;
  HCHECK(cudaMalloc((void**)&kp, sizeof(Keypoint) * (size_t)(max_tracks > 0 ? max_tracks : 1)));
  float* bins = nullptr;  // [0]=kpCount, [1]=kpIndex (as int), [2..65]=bins
  HCHECK(cudaMalloc((void**)&bins, sizeof(float) * 66));
  HCHECK(cudaMemset(bins, 0, sizeof(float) * 66));
  size_t tmp_bytes = sort_keypoints_get_temp_buffer_size((size_t)max_tracks);
  void* tmp = nullptr;
  HCHECK(cudaMalloc(&tmp, tmp_bytes > 0 ? tmp_bytes : 1));

  int n_old = n_alive < max_tracks ? n_alive : max_tracks;
  std::vector<Keypoint> host_kp((size_t)(max_tracks > 0 ? max_tracks : 1));
  for (int i = 0; i < n_old; ++i) host_kp[i] = {alive_xy[2 * i], alive_xy[2 * i + 1], 0.f};
  if (n_old > 0) HCHECK(cudaMemcpy(kp, host_kp.data(), sizeof(Keypoint) * n_old, cudaMemcpyHostToDevice));

  HCHECK(gftt_values(p.gx[0]->tex_point, p.gy[0]->tex_point, val.ptr, val.pitch, size, s));
  HCHECK(accumulateGFTT(val.tex_point, size, bin_size, num_bins, bins + 2, s));
  HCHECK(non_max_suppression(val.tex_point, size, maxim.ptr, maxim.pitch, s));
  if (n_old > 0) HCHECK(filter_maximums(maxim.ptr, size, maxim.pitch, kp, (size_t)n_old, s));
  int kp_count = 0;
  std::vector<float> hb(66, 0.f);
  if (max_tracks > 0) {
    HCHECK(downsample_gftt_x8(maxim.ptr, maxim.pitch, dsm.ptr, ds, dsm.pitch, idx, idx_pitch, s));
    HCHECK(select_features(val.ptr, size, val.pitch, dsm.ptr, ds, dsm.pitch, idx, idx_pitch, kp, (size_t)max_tracks,
                           (int*)bins, (int*)bins + 1, s));
  }
  HCHECK(cudaMemcpy(hb.data(), bins, sizeof(float) * 66, cudaMemcpyDeviceToHost));
  memcpy(&kp_count, hb.data(), sizeof(int));
  if (kp_count > 0) sort_keypoints(kp, (size_t)kp_count, tmp, tmp_bytes, s);
  HCHECK(cudaStreamSynchronize(s));
  HCHECK(cudaGetLastError());

  HCHECK(val.download(gftt));
  HCHECK(maxim.download(nms));
  if (max_tracks > 0) {
    HCHECK(dsm.download(cell_max));
    std::vector<uint2> hi((size_t)max_tracks);
    HCHECK(cudaMemcpy2D(hi.data(), ds.x * sizeof(uint2), idx, idx_pitch, ds.x * sizeof(uint2), ds.y,
                        cudaMemcpyDeviceToHost));
    for (int i = 0; i < max_tracks; ++i) {
      cell_idx[2 * i] = hi[i].x;
      cell_idx[2 * i + 1] = hi[i].y;
    }
  }
  if (kp_count > 0) HCHECK(cudaMemcpy(host_kp.data(), kp, sizeof(Keypoint) * kp_count, cudaMemcpyDeviceToHost));
  *n_kp = kp_count;
  for (int i = 0; i < kp_count; ++i) {
    kp_out[3 * i] = host_kp[i].x;
    kp_out[3 * i + 1] = host_kp[i].y;
    kp_out[3 * i + 2] = host_kp[i].strength;
  }
  for (int i = 0; i < 64; ++i) bins_out[i] = hb[i + 2];

  // Host quota loop of GPUSelection::computeGFTTAndSelectFeatures (selection_v2.cpp:108-183).
  float sum = 0.f;
  for (int i = 0; i < 64; ++i) sum += hb[i + 2];
  size_t prev_cnt[64] = {0}, want[64] = {0}, added[64] = {0};
  for (int i = 0; i < n_alive; ++i) {
    unsigned bx = (unsigned)(alive_xy[2 * i] / (float)bin_size.x);
    unsigned by = (unsigned)(alive_xy[2 * i + 1] / (float)bin_size.y);
    if (bx < 8 && by < 8) prev_cnt[by * 8 + bx]++;
  }
  const size_t expected = (size_t)n_alive + (size_t)num_desired;
  for (int i = 0; i < 64; ++i) {
    // A zero strength sum makes the reference's quota a NaN cast (undefined); no quota here.
    if (!(sum > 0.f)) break;
    size_t e = (size_t)std::round((float)expected * hb[i + 2] / sum);
    if (e > prev_cnt[i]) want[i] = e - prev_cnt[i];
  }
  int out_n = 0;
  for (int i = 0; i < kp_count; ++i) {
    float x = host_kp[i].x, y = host_kp[i].y;
    if (x < border_left || x > (float)(w - 1 - border_right) || y < border_top || y > (float)(h - 1 - border_bottom))
      continue;
    unsigned bx = (unsigned)(x / (float)bin_size.x), by = (unsigned)(y / (float)bin_size.y);
    if (bx < 8 && by < 8) {
      unsigned b = by * 8 + bx;
      if (added[b] < want[b]) {
        added[b]++;
        if (out_n < num_desired) {
          sel[2 * out_n] = x;
          sel[2 * out_n + 1] = y;
          ++out_n;
        } else {
          break;
        }
      }
    }
  }
  *n_sel = out_n;
  cudaFree(idx);
  cudaFree(kp);
  cudaFree(bins);
  cudaFree(tmp);
  return 0;
}

// Pyramid of a mono or RGB8 frame with or without the box prefilter (build_ex), all levels to host
// buffers laid out level after level (as ref_pyramid).
int ref_pyramid_ex(const uint8_t* img, int w, int h, int rgb, int box3, int max_levels, int* nlev, float* levels,
                   float* gx, float* gy) {
  int rc = init_tables();
  if (rc) return rc;
  Pyr p;
  rc = build_ex(img, w, h, rgb, box3, max_levels, p, 0);
  if (rc) return rc;
  size_t off = 0;
  for (int l = 0; l < p.n; ++l) {
    HCHECK(p.img[l]->download(levels + off));
    HCHECK(p.gx[l]->download(gx + off));
    HCHECK(p.gy[l]->download(gy + off));
    off += (size_t)p.img[l]->w * p.img[l]->h;
  }
  *nlev = p.n;
  return 0;
}

// GPULKFeatureTracker::track_points (or GPULKTrackerHorizontal) between the pyramids of two u8
// images.  `tracks` holds n reference TrackData records (80 bytes each), updated in place.
int ref_lk(const uint8_t* prev_img, const uint8_t* cur_img, int w, int h, int max_levels, void* tracks, int n,
           int horizontal) {
  int rc = init_tables();
  if (rc) return rc;
  if (sizeof(TrackData) != 80) return -1;
  Pyr pp, cp;
  rc = build(prev_img, w, h, max_levels, pp, 0);
  if (rc) return rc;
  rc = build(cur_img, w, h, max_levels, cp, 0);
  if (rc) return rc;
  TrackData* d = nullptr;
  HCHECK(cudaMalloc((void**)&d, sizeof(TrackData) * (size_t)(n > 0 ? n : 1)));
  HCHECK(cudaMemcpy(d, tracks, sizeof(TrackData) * (size_t)n, cudaMemcpyHostToDevice));
  Pyramid gx = make_pyr(pp, pp.gx), gy = make_pyr(pp, pp.gy), pi = make_pyr(pp, pp.img), ci = make_pyr(cp, cp.img);
  if (n > 0) {
    if (horizontal)
      HCHECK(lk_track_horizontal(gx, pi, ci, d, n, 0));
    else
      HCHECK(lk_track(gx, gy, pi, ci, d, n, 0));
  }
  HCHECK(cudaDeviceSynchronize());
  HCHECK(cudaMemcpy(tracks, d, sizeof(TrackData) * (size_t)n, cudaMemcpyDeviceToHost));
  cudaFree(d);
  return 0;
}

// GPUSTFeatureTracker::track_points (cached = 0) or GPUSTFeatureTrackerWithCache's
// build_points_cache + track_points (cached = 1) between the pyramids of two u8 images
// (cuda_modules/st_tracker.cpp:27-160): the current pyramid's image and gradients, the previous
// pyramid's image.  `tracks` (n TrackData records) is updated in place; with cached = 1 and
// cache_out != null the n PointCacheData entries (3284 bytes each) are copied out as well.
int ref_st_track(const uint8_t* prev_img, const uint8_t* cur_img, int w, int h, int max_levels, void* tracks, int n,
                 int n_shift, int n_full, int cached, void* cache_out) {
  int rc = init_tables();
  if (rc) return rc;
  HCHECK(init_st_tracker());
  if (sizeof(TrackData) != 80 || sizeof(PointCacheDataT) != 3284) return -1;
  Pyr pp, cp;
  rc = build(prev_img, w, h, max_levels, pp, 0);
  if (rc) return rc;
  rc = build(cur_img, w, h, max_levels, cp, 0);
  if (rc) return rc;
  TrackData* d = nullptr;
  PointCacheDataT* c = nullptr;
  HCHECK(cudaMalloc((void**)&d, sizeof(TrackData) * (size_t)(n > 0 ? n : 1)));
  HCHECK(cudaMalloc((void**)&c, sizeof(PointCacheDataT) * (size_t)(n > 0 ? n : 1)));
  HCHECK(cudaMemset(c, 0, sizeof(PointCacheDataT) * (size_t)(n > 0 ? n : 1)));
  HCHECK(cudaMemcpy(d, tracks, sizeof(TrackData) * (size_t)n, cudaMemcpyHostToDevice));
  Pyramid cgx = make_pyr(cp, cp.gx), cgy = make_pyr(cp, cp.gy), pi = make_pyr(pp, pp.img), ci = make_pyr(cp, cp.img);
  if (n > 0) {
    if (cached) {
      HCHECK(st_build_cache(pi, d, c, (size_t)n, 0));
      HCHECK(st_track_with_cache(cgx, cgy, ci, c, d, n, (unsigned)n_shift, (unsigned)n_full, 0));
    } else {
      HCHECK(st_track(cgx, cgy, pi, ci, d, n, (unsigned)n_shift, (unsigned)n_full, 0));
    }
  }
  HCHECK(cudaDeviceSynchronize());
  HCHECK(cudaMemcpy(tracks, d, sizeof(TrackData) * (size_t)n, cudaMemcpyDeviceToHost));
  if (cached && cache_out) HCHECK(cudaMemcpy(cache_out, c, sizeof(PointCacheDataT) * (size_t)n, cudaMemcpyDeviceToHost));
  cudaFree(d);
  cudaFree(c);
  return 0;
}

// Device time (CUDA events, mean over `reps` after 3 warm-up runs) of one reference GPU stage on
// the pyramids of two u8 images: which = 0 the current frame's pyramid (cast_image, gaussian_scaling
// per level, conv_grad_x/y per level, as build() enqueues them; allocations excluded); 1 lk_track;
// 2 st_track (n_shift, n_full); 3 st_track_with_cache after st_build_cache.  Tracks are reset from
// the caller's n records before every run (the copy is outside the timed interval).
int ref_time_stage(const uint8_t* prev_img, const uint8_t* cur_img, int w, int h, int max_levels, const void* tracks,
                   int n, int which, int n_shift, int n_full, int reps, float* ms_out) {
  int rc = init_tables();
  if (rc) return rc;
  HCHECK(init_st_tracker());
  Pyr pp, cp;
  rc = build(prev_img, w, h, max_levels, pp, 0);
  if (rc) return rc;
  rc = build(cur_img, w, h, max_levels, cp, 0);
  if (rc) return rc;
  TrackData *d = nullptr, *d0 = nullptr;
  PointCacheDataT* c = nullptr;
  const size_t nb = sizeof(TrackData) * (size_t)(n > 0 ? n : 1);
  HCHECK(cudaMalloc((void**)&d, nb));
  HCHECK(cudaMalloc((void**)&d0, nb));
  HCHECK(cudaMalloc((void**)&c, sizeof(PointCacheDataT) * (size_t)(n > 0 ? n : 1)));
  if (n > 0) HCHECK(cudaMemcpy(d0, tracks, sizeof(TrackData) * (size_t)n, cudaMemcpyHostToDevice));
  uint8_t* d_u8 = nullptr;
  size_t u8_pitch = 0;
  HCHECK(cudaMallocPitch((void**)&d_u8, &u8_pitch, w, h));
  HCHECK(cudaMemcpy2D(d_u8, u8_pitch, cur_img, w, w, h, cudaMemcpyHostToDevice));
  DevImage cast;
  HCHECK(cast.alloc(w, h));
  Pyramid pgx = make_pyr(pp, pp.gx), pgy = make_pyr(pp, pp.gy), pi = make_pyr(pp, pp.img);
  Pyramid cgx = make_pyr(cp, cp.gx), cgy = make_pyr(cp, cp.gy), ci = make_pyr(cp, cp.img);
  cudaStream_t s = 0;
  if (which == 3 && n > 0) {
    HCHECK(cudaMemcpy(d, d0, sizeof(TrackData) * (size_t)n, cudaMemcpyDeviceToDevice));
    HCHECK(st_build_cache(pi, d, c, (size_t)n, s));
    HCHECK(cudaMemcpy(d0, d, sizeof(TrackData) * (size_t)n, cudaMemcpyDeviceToDevice));  // cache_index set
  }
  auto run = [&]() -> int {
    if (which == 0) {
      HCHECK(cast_image(d_u8, u8_pitch, cast.ptr, cast.pitch, {(unsigned)w, (unsigned)h}, s));
      HCHECK(cudaMemcpy2DAsync(cp.img[0]->ptr, cp.img[0]->pitch, cast.ptr, cast.pitch, (size_t)w * 4, h,
                               cudaMemcpyDeviceToDevice, s));
      for (int l = 0; l + 1 < cp.n; ++l) {
        const DevImage& a = *cp.img[l];
        DevImage& b = *cp.img[l + 1];
        HCHECK(gaussian_scaling(a.tex_point, {(unsigned)a.w, (unsigned)a.h}, b.ptr, b.pitch,
                                {(unsigned)b.w, (unsigned)b.h}, s));
      }
      for (int l = 0; l < cp.n; ++l) {
        const DevImage& a = *cp.img[l];
        HCHECK(conv_grad_x(a.tex_point, {(unsigned)a.w, (unsigned)a.h}, cp.gx[l]->ptr, cp.gx[l]->pitch, s));
        HCHECK(conv_grad_y(a.tex_point, {(unsigned)a.w, (unsigned)a.h}, cp.gy[l]->ptr, cp.gy[l]->pitch, s));
      }
    } else if (which == 1) {
      HCHECK(lk_track(pgx, pgy, pi, ci, d, n, s));
    } else if (which == 2) {
      HCHECK(st_track(cgx, cgy, pi, ci, d, n, (unsigned)n_shift, (unsigned)n_full, s));
    } else {
      HCHECK(st_track_with_cache(cgx, cgy, ci, c, d, n, (unsigned)n_shift, (unsigned)n_full, s));
    }
    return 0;
  };
  cudaEvent_t e0, e1;
  HCHECK(cudaEventCreate(&e0));
  HCHECK(cudaEventCreate(&e1));
  float total = 0.f;
  for (int r = 0; r < reps + 3; ++r) {
    if (n > 0 && which != 0) HCHECK(cudaMemcpyAsync(d, d0, sizeof(TrackData) * (size_t)n, cudaMemcpyDeviceToDevice, s));
    HCHECK(cudaEventRecord(e0, s));
    rc = run();
    if (rc) return rc;
    HCHECK(cudaEventRecord(e1, s));
    HCHECK(cudaEventSynchronize(e1));
    float ms = 0.f;
    HCHECK(cudaEventElapsedTime(&ms, e0, e1));
    if (r >= 3) total += ms;
  }
  *ms_out = total / (float)(reps > 0 ? reps : 1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(d);
  cudaFree(d0);
  cudaFree(c);
  cudaFree(d_u8);
  return 0;
}

// Host wall-clock time (mean over `reps` after 2 warm-up runs) of one camera's frame through the
// reference's GPU path on one stream, as MonoSOFGPU runs it: the current frame's pyramid and
// gradients from a uint8 frame in device memory (cast_image, gaussian_scaling, conv_grad_x/y), LK of
// n tracks from the previous pyramid (lk_track; records reset before each run, outside the timed
// interval), then GPUSelection::computeGFTTAndSelectFeatures with the n track positions alive:
// gftt_values, accumulateGFTT, non_max_suppression, filter_maximums, downsample_gftt_x8,
// select_features, the count read back, sort_keypoints, the keypoints read back and the host quota
// loop for num_desired features (selection_v2.cpp:27-184).  Allocations happen before timing.
int ref_time_frame(const uint8_t* prev_img, const uint8_t* cur_img, int w, int h, int max_levels, const void* tracks,
                   int n, int num_desired, int reps, float* ms_out) {
  int rc = init_tables();
  if (rc) return rc;
  Pyr pp, cp;
  rc = build(prev_img, w, h, max_levels, pp, 0);
  if (rc) return rc;
  rc = build(cur_img, w, h, max_levels, cp, 0);
  if (rc) return rc;
  cudaStream_t s = 0;
  TrackData *d = nullptr, *d0 = nullptr;
  const size_t nb = sizeof(TrackData) * (size_t)(n > 0 ? n : 1);
  HCHECK(cudaMalloc((void**)&d, nb));
  HCHECK(cudaMalloc((void**)&d0, nb));
  if (n > 0) HCHECK(cudaMemcpy(d0, tracks, sizeof(TrackData) * (size_t)n, cudaMemcpyHostToDevice));
  std::vector<TrackData> host_td((size_t)(n > 0 ? n : 1));
  if (n > 0) memcpy(host_td.data(), tracks, sizeof(TrackData) * (size_t)n);
  uint8_t* d_u8 = nullptr;
  size_t u8_pitch = 0;
  HCHECK(cudaMallocPitch((void**)&d_u8, &u8_pitch, w, h));
  HCHECK(cudaMemcpy2D(d_u8, u8_pitch, cur_img, w, w, h, cudaMemcpyHostToDevice));
  DevImage cast, val, maxim, dsm;
  HCHECK(cast.alloc(w, h));
  const uint2 size = {(unsigned)w, (unsigned)h};
  const uint2 bin_size = {(unsigned)(w / 8), (unsigned)(h / 8)};
  const uint2 num_bins = {8, 8};
  const uint2 ds = {(unsigned)w / 8, (unsigned)h / 8};
  const int max_tracks = (int)(ds.x * ds.y);
  HCHECK(val.alloc(w, h));
  HCHECK(maxim.alloc(w, h));
  HCHECK(dsm.alloc((int)ds.x, (int)ds.y));
  uint2* idx = nullptr;
  size_t idx_pitch = 0;
  HCHECK(cudaMallocPitch((void**)&idx, &idx_pitch, ds.x * sizeof(uint2), ds.y));
  Keypoint* kp = nullptr;
  HCHECK(cudaMalloc((void**)&kp, sizeof(Keypoint) * (size_t)(max_tracks > 0 ? max_tracks : 1)));
  float* bins = nullptr;
  HCHECK(cudaMalloc((void**)&bins, sizeof(float) * 66));
  size_t tmp_bytes = sort_keypoints_get_temp_buffer_size((size_t)max_tracks);
  void* tmp = nullptr;
  HCHECK(cudaMalloc(&tmp, tmp_bytes > 0 ? tmp_bytes : 1));
  std::vector<Keypoint> alive((size_t)(max_tracks > 0 ? max_tracks : 1)), host_kp(alive.size());
  const int n_old = n < max_tracks ? n : max_tracks;
  for (int i = 0; i < n_old; ++i) alive[i] = {host_td[i].track.x, host_td[i].track.y, 0.f};
  Pyramid pgx = make_pyr(pp, pp.gx), pgy = make_pyr(pp, pp.gy), pi = make_pyr(pp, pp.img), ci = make_pyr(cp, cp.img);
  std::vector<float> sel((size_t)2 * (num_desired > 0 ? num_desired : 1));
  double total = 0.0;
  for (int r = 0; r < reps + 2; ++r) {
    if (n > 0) HCHECK(cudaMemcpy(d, d0, sizeof(TrackData) * (size_t)n, cudaMemcpyDeviceToDevice));
    HCHECK(cudaDeviceSynchronize());
    const auto t0 = std::chrono::steady_clock::now();
    // pyramid + gradients
    HCHECK(cast_image(d_u8, u8_pitch, cast.ptr, cast.pitch, size, s));
    HCHECK(cudaMemcpy2DAsync(cp.img[0]->ptr, cp.img[0]->pitch, cast.ptr, cast.pitch, (size_t)w * 4, h,
                             cudaMemcpyDeviceToDevice, s));
    for (int l = 0; l + 1 < cp.n; ++l) {
      const DevImage& a = *cp.img[l];
      DevImage& b = *cp.img[l + 1];
      HCHECK(gaussian_scaling(a.tex_point, {(unsigned)a.w, (unsigned)a.h}, b.ptr, b.pitch,
                              {(unsigned)b.w, (unsigned)b.h}, s));
    }
    for (int l = 0; l < cp.n; ++l) {
      const DevImage& a = *cp.img[l];
      HCHECK(conv_grad_x(a.tex_point, {(unsigned)a.w, (unsigned)a.h}, cp.gx[l]->ptr, cp.gx[l]->pitch, s));
      HCHECK(conv_grad_y(a.tex_point, {(unsigned)a.w, (unsigned)a.h}, cp.gy[l]->ptr, cp.gy[l]->pitch, s));
    }
    // LK
    if (n > 0) HCHECK(lk_track(pgx, pgy, pi, ci, d, n, s));
    // selection on the current frame with the tracks alive
    if (n_old > 0) HCHECK(cudaMemcpyAsync(kp, alive.data(), sizeof(Keypoint) * n_old, cudaMemcpyHostToDevice, s));
    HCHECK(cudaMemsetAsync(bins, 0, sizeof(float) * 66, s));
    HCHECK(gftt_values(cp.gx[0]->tex_point, cp.gy[0]->tex_point, val.ptr, val.pitch, size, s));
    HCHECK(accumulateGFTT(val.tex_point, size, bin_size, num_bins, bins + 2, s));
    HCHECK(non_max_suppression(val.tex_point, size, maxim.ptr, maxim.pitch, s));
    if (n_old > 0) HCHECK(filter_maximums(maxim.ptr, size, maxim.pitch, kp, (size_t)n_old, s));
    float hb[66];
    int kp_count = 0;
    if (max_tracks > 0) {
      HCHECK(downsample_gftt_x8(maxim.ptr, maxim.pitch, dsm.ptr, ds, dsm.pitch, idx, idx_pitch, s));
      HCHECK(select_features(val.ptr, size, val.pitch, dsm.ptr, ds, dsm.pitch, idx, idx_pitch, kp,
                             (size_t)max_tracks, (int*)bins, (int*)bins + 1, s));
    }
    HCHECK(cudaMemcpyAsync(hb, bins, sizeof(float) * 66, cudaMemcpyDeviceToHost, s));
    HCHECK(cudaStreamSynchronize(s));
    memcpy(&kp_count, hb, sizeof(int));
    if (kp_count > max_tracks) kp_count = max_tracks;
    if (kp_count > 0) sort_keypoints(kp, (size_t)kp_count, tmp, tmp_bytes, s);
    if (kp_count > 0) HCHECK(cudaMemcpyAsync(host_kp.data(), kp, sizeof(Keypoint) * kp_count, cudaMemcpyDeviceToHost, s));
    HCHECK(cudaStreamSynchronize(s));
    float sum = 0.f;
    for (int i = 0; i < 64; ++i) sum += hb[i + 2];
    size_t prev_cnt[64] = {0}, want[64] = {0}, added[64] = {0};
    for (int i = 0; i < n_old; ++i) {
      const unsigned bx = (unsigned)(alive[i].x / (float)bin_size.x), by = (unsigned)(alive[i].y / (float)bin_size.y);
      if (bx < 8 && by < 8) prev_cnt[by * 8 + bx]++;
    }
    for (int i = 0; i < 64 && sum > 0.f; ++i) {
      const size_t e = (size_t)std::round((float)((size_t)n + (size_t)num_desired) * hb[i + 2] / sum);
      if (e > prev_cnt[i]) want[i] = e - prev_cnt[i];
    }
    int out_n = 0;
    for (int i = 0; i < kp_count && out_n < num_desired; ++i) {
      const unsigned bx = (unsigned)(host_kp[i].x / (float)bin_size.x), by = (unsigned)(host_kp[i].y / (float)bin_size.y);
      if (bx < 8 && by < 8 && added[by * 8 + bx] < want[by * 8 + bx]) {
        added[by * 8 + bx]++;
        sel[2 * out_n] = host_kp[i].x;
        sel[2 * out_n + 1] = host_kp[i].y;
        ++out_n;
      }
    }
    const auto t1 = std::chrono::steady_clock::now();
    if (r >= 2) total += std::chrono::duration<double, std::milli>(t1 - t0).count();
  }
  *ms_out = (float)(total / (reps > 0 ? reps : 1));
  cudaFree(d);
  cudaFree(d0);
  cudaFree(d_u8);
  cudaFree(idx);
  cudaFree(kp);
  cudaFree(bins);
  cudaFree(tmp);
  return 0;
}

// MultiSOFGPU::LaunchTrackingPrimaryToSecondary's scan between the pyramids of a primary and a
// secondary u8 image: one lk_track_horizontal (or lk_track) launch per candidate index k over all n points, a copy
// back and a synchronisation, first success wins, early exit once matched >= frac * n.  Candidates
// of point i: cand_xy[cand_off[i] .. cand_off[i+1]); valid may be null.  out: n TrackData records as
// the reference publishes them; winner[i]: winning candidate or -1; stats: matched, rounds launched.
int ref_stereo_scan(const uint8_t* prim_img, const uint8_t* sec_img, int w, int h, int max_levels, const float* uv,
                    const uint8_t* valid, int n, const int* cand_off, const float* cand_xy, float radius,
                    float ncc_thr, float frac, int horizontal, void* out, int* winner, int* stats) {
  int rc = init_tables();
  if (rc) return rc;
  Pyr pp, sp;
  rc = build(prim_img, w, h, max_levels, pp, 0);
  if (rc) return rc;
  rc = build(sec_img, w, h, max_levels, sp, 0);
  if (rc) return rc;
  std::vector<TrackData> data((size_t)(n > 0 ? n : 1)), win((size_t)(n > 0 ? n : 1));
  std::vector<int> len((size_t)(n > 0 ? n : 1));
  int max_candidates = 0;
  for (int i = 0; i < n; ++i) {
    len[i] = (valid && !valid[i]) ? 0 : cand_off[i + 1] - cand_off[i];
    if (len[i] > max_candidates) max_candidates = len[i];
    win[i] = TrackData{};
    winner[i] = -1;
  }
  TrackData* d = nullptr;
  HCHECK(cudaMalloc((void**)&d, sizeof(TrackData) * data.size()));
  Pyramid gx = make_pyr(pp, pp.gx), gy = make_pyr(pp, pp.gy), pi = make_pyr(pp, pp.img), si = make_pyr(sp, sp.img);
  auto uv_of = [&](int i, int c) { return (valid && !valid[i]) ? 0.f : uv[2 * i + c]; };
  int tracked = 0, rounds = 0;
  for (int k = 0; k < max_candidates; ++k) {
    bool any_active = false;
    for (int i = 0; i < n; ++i) {
      TrackData& t = data[i];
      t.ncc_threshold = ncc_thr;
      t.track = {uv_of(i, 0), uv_of(i, 1)};
      t.track_status = false;
      t.search_radius_px = radius;
      for (int q = 0; q < 4; ++q) t.info[q] = 0.f;
      if (win[i].track_status || k >= len[i]) {
        t.offset = {0.f, 0.f};
      } else {
        const float* c = cand_xy + 2 * ((size_t)cand_off[i] + k);
        t.offset = {c[0] - uv_of(i, 0), c[1] - uv_of(i, 1)};
        any_active = true;
      }
    }
    if (!any_active) break;
    HCHECK(cudaMemcpy(d, data.data(), sizeof(TrackData) * (size_t)n, cudaMemcpyHostToDevice));
    if (horizontal)
      HCHECK(lk_track_horizontal(gx, pi, si, d, n, 0));
    else
      HCHECK(lk_track(gx, gy, pi, si, d, n, 0));
    HCHECK(cudaMemcpy(data.data(), d, sizeof(TrackData) * (size_t)n, cudaMemcpyDeviceToHost));
    HCHECK(cudaDeviceSynchronize());
    rounds = k + 1;
    for (int i = 0; i < n; ++i) {
      if (win[i].track_status || k >= len[i]) continue;
      if (data[i].track_status) {
        win[i] = data[i];
        winner[i] = k;
        ++tracked;
      }
    }
    if ((float)tracked >= frac * (float)n) break;
  }
  for (int i = 0; i < n; ++i) {
    if (win[i].track_status) {
      data[i] = win[i];
    } else {
      data[i].track_status = false;
      data[i].track = {uv_of(i, 0), uv_of(i, 1)};
    }
  }
  cudaFree(d);
  if (n > 0) memcpy(out, data.data(), sizeof(TrackData) * (size_t)n);
  stats[0] = tracked;
  stats[1] = rounds;
  return 0;
}

// Hardware bilinear texture sampling with the reference's linear texture descriptor
// (cudaFilterModeLinear, unnormalised coordinates).  Used to pin the oracle's emulation of
// the texture unit's 8-bit-fraction weights.
__global__ void tex_probe_kernel(cudaTextureObject_t t, const float2* xy, int n, float* out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = tex2D<float>(t, xy[i].x, xy[i].y);
}

int ref_tex_probe(const float* img, int w, int h, const float* xy, int n, float* out) {
  DevImage im;
  HCHECK(im.alloc(w, h));
  HCHECK(im.upload(img));
  float2* dxy = nullptr;
  float* dout = nullptr;
  HCHECK(cudaMalloc((void**)&dxy, sizeof(float2) * (size_t)n));
  HCHECK(cudaMalloc((void**)&dout, sizeof(float) * (size_t)n));
  HCHECK(cudaMemcpy(dxy, xy, sizeof(float2) * (size_t)n, cudaMemcpyHostToDevice));
  tex_probe_kernel<<<(n + 255) / 256, 256>>>(im.tex_linear, dxy, n, dout);
  HCHECK(cudaGetLastError());
  HCHECK(cudaDeviceSynchronize());
  HCHECK(cudaMemcpy(out, dout, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost));
  cudaFree(dxy);
  cudaFree(dout);
  return 0;
}

}  // extern "C"
