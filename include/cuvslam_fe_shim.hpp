/* cuvslam_fe_shim.hpp - cuVSLAM's four GPU wrapper classes restated on the C ABI of cuvslam_fe.h.
 *
 * MonoSOFGPU (libs/sof/sof_mono_gpu.cpp) and ImageContext (libs/sof/image_context.cpp) drive the
 * GPU front-end through four classes of libs/cuda_modules.  This header re-implements them with the
 * same names and method signatures on top of libcuvslam_fe.so, so that a cuVSLAM build can take this
 * header in place of their implementations and leave libs/sof and libs/odometry unchanged:
 *
 *   GaussianGPUImagePyramid::build        (image_pyramid.h:81-98)
 *   GPUGradientPyramid::set               (gradient_pyramid.h:45, gradient_pyramid.cpp:83-118)
 *   GPUSelection::computeGFTTAndSelectFeatures   (selection_v2.h:32-35, selection_v2.cpp:27-184)
 *   GPULKFeatureTracker::track_points     (lk_tracker.h:31-34, cuda_modules/lk_tracker.cpp:24-73)
 *   GPULKTrackerHorizontal::track_points  (lk_tracker.h:43-50, cuda_modules/lk_tracker.cpp:75-114)
 *
 * Differences a caller can see (all else follows the reference):
 *  - Gradients are computed by the pyramid build itself (one launch for the image pyramid and both
 *    gradient pyramids).  GPUGradientPyramid::set therefore does no work: it refers to the gradient
 *    planes of the image pyramid it is given, which must outlive it and not be rebuilt while its
 *    gradients are in use (ImageContext keeps both for the same frame).
 *  - ImageContext's cast + build (image_context.cpp:215-240) is one call, build_u8, from the uint8
 *    frame in device memory; build() from an FP32 frame has no box prefilter (blur_filter = true
 *    throws std::invalid_argument: prefilter uint8 frames with build_u8).
 *  - Errors throw std::runtime_error, as the reference's CUDA_CHECK does (cuda_helper.h:42-56).
 *
 * Inside cuVSLAM, define CUVSLAM_FE_SHIM_EXTERNAL_TYPES and include the reference's own
 * common/vector_2t.h, common/image_matrix.h and cuda_modules/cuda_helper.h first: the shim then uses
 * cuVSLAM's Vector2T, ImageMatrix, GPUImageT and GPUArrayPinned.  Otherwise it declares minimal
 * stand-ins with the members it uses (Vector2T(x, y), x(), y(); ImageMatrix rows()/cols()/data(),
 * row-major; GPUArrayPinned<T> with pinned host + device storage, ptr() = device pointer; GPUImageT
 * a pitched FP32 device image).
 */
#ifndef CUVSLAM_FE_SHIM_HPP
#define CUVSLAM_FE_SHIM_HPP

#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "cuvslam_fe.h"

namespace cuvslam {

#ifndef CUVSLAM_FE_SHIM_EXTERNAL_TYPES
/* Stand-in for Eigen::Matrix<float, 2, 1> (common/vector_2t.h:31). */
class Vector2T {
 public:
  Vector2T() = default;
  Vector2T(float x, float y) : v_{x, y} {}
  float x() const { return v_[0]; }
  float y() const { return v_[1]; }
  float& x() { return v_[0]; }
  float& y() { return v_[1]; }
  float operator[](int i) const { return v_[i]; }
  float& operator[](int i) { return v_[i]; }

 private:
  float v_[2] = {0.f, 0.f};
};

/* Stand-in for the row-major Eigen matrix of common/image_matrix.h:25 (host memory). */
template <class T>
class ImageMatrix {
 public:
  ImageMatrix() = default;
  ImageMatrix(size_t rows, size_t cols) : rows_(rows), cols_(cols), data_(rows * cols) {}
  size_t rows() const { return rows_; }
  size_t cols() const { return cols_; }
  T* data() { return data_.data(); }
  const T* data() const { return data_.data(); }
  T& operator()(size_t r, size_t c) { return data_[r * cols_ + c]; }
  const T& operator()(size_t r, size_t c) const { return data_[r * cols_ + c]; }

 private:
  size_t rows_ = 0, cols_ = 0;
  std::vector<T> data_;
};
#endif

namespace cuda {

inline void shim_throw(const std::string& what) { throw std::runtime_error(what); }

/* CUDA_CHECK's behaviour (cuda_helper.h:42-56) for both kinds of status. */
inline void shim_check_cuda(cudaError_t e, const char* what) {
  if (e != cudaSuccess) shim_throw(std::string(what) + ": " + cudaGetErrorString(e));
}
inline void shim_check_fe(int status, const char* what) {
  if (status != FE_OK) {
    std::string msg = std::string(what) + ": " + fe_status_string(status);
    if (status == FE_ERR_CUDA) msg += std::string(" (") + cudaGetErrorString((cudaError_t)fe_last_cuda_error()) + ")";
    if (status == FE_ERR_INVALID_ARGUMENT) throw std::invalid_argument(msg);
    shim_throw(msg);
  }
}

#ifndef CUVSLAM_FE_SHIM_EXTERNAL_TYPES
/* TrackData (cuda_kernels.h:76-87) is fe_track_data byte for byte. */
using TrackData = fe_track_data;

enum GPUCopyDirection { ToGPU, ToCPU };

/* Stand-in for GPUArrayPinned<T> (cuda_helper.h:135-230): a pinned host array and a device array of
 * the same size; ptr() is the device array. */
template <class T>
class GPUArrayPinned {
 public:
  explicit GPUArrayPinned(size_t size) { alloc(size); }
  GPUArrayPinned(const GPUArrayPinned&) = delete;
  GPUArrayPinned& operator=(const GPUArrayPinned&) = delete;
  ~GPUArrayPinned() { release(); }
  T& operator[](size_t i) { return host_[i]; }
  const T& operator[](size_t i) const { return host_[i]; }
  void copy(GPUCopyDirection direction, cudaStream_t s) const { copy_top_n(direction, size_, s); }
  void copy_top_n(GPUCopyDirection direction, size_t top_n, cudaStream_t s) const {
    if (top_n == 0) return;
    if (top_n > size_) throw std::out_of_range("copy_top_n exceeds GPUArrayPinned size");
    if (direction == ToGPU)
      shim_check_cuda(cudaMemcpyAsync(device_, host_, top_n * sizeof(T), cudaMemcpyHostToDevice, s), "copy_top_n");
    else
      shim_check_cuda(cudaMemcpyAsync(host_, device_, top_n * sizeof(T), cudaMemcpyDeviceToHost, s), "copy_top_n");
  }
  T* ptr() const { return device_; }
  size_t size() const { return size_; }
  void resize(size_t size) {
    if (size == size_) return;
    release();
    alloc(size);
  }

 private:
  void alloc(size_t size) {
    size_ = size;
    if (size == 0) return;
    shim_check_cuda(cudaMallocHost((void**)&host_, size * sizeof(T)), "GPUArrayPinned host");
    std::memset(static_cast<void*>(host_), 0, size * sizeof(T));
    shim_check_cuda(cudaMalloc((void**)&device_, size * sizeof(T)), "GPUArrayPinned device");
  }
  void release() {
    if (host_) cudaFreeHost(host_);
    if (device_) cudaFree(device_);
    host_ = nullptr;
    device_ = nullptr;
    size_ = 0;
  }
  T* host_ = nullptr;
  T* device_ = nullptr;
  size_t size_ = 0;
};

/* Stand-in for GPUImage<float> (cuda_helper.h:255-434): a pitched FP32 image in device memory. */
class GPUImageT {
 public:
  GPUImageT(size_t cols, size_t rows) : cols_(cols), rows_(rows) {
    shim_check_cuda(cudaMallocPitch((void**)&data_, &pitch_, cols * sizeof(float), rows), "GPUImage");
  }
  GPUImageT(const GPUImageT&) = delete;
  GPUImageT& operator=(const GPUImageT&) = delete;
  ~GPUImageT() {
    if (data_) cudaFree(data_);
  }
  float* ptr() const { return data_; }
  size_t pitch() const { return pitch_; }
  size_t cols() const { return cols_; }
  size_t rows() const { return rows_; }

 private:
  float* data_ = nullptr;
  size_t cols_ = 0, rows_ = 0, pitch_ = 0;
};
#endif

/* One fe_context per wrapper object, on the device current when the object first needs it: a
 * context runs one selection / one LK launch / 64 pyramid builds at a time, as each reference wrapper
 * object owns its own buffers and is used by one thread at a time. */
class ShimContext {
 public:
  fe_context* get() {
    if (!ctx_) {
      int dev = 0;
      shim_check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
      fe_context* c = nullptr;
      shim_check_fe(fe_create(dev, &c), "fe_create");
      ctx_.reset(c);
    }
    return ctx_.get();
  }

 private:
  struct Destroy {
    void operator()(fe_context* c) const { fe_destroy(c); }
  };
  std::unique_ptr<fe_context, Destroy> ctx_;
};

struct ShimDeviceFree {
  void operator()(void* p) const { cudaFree(p); }
};

/* GaussianGPUImagePyramid (image_pyramid.h:56-161, MAX_PYRAMID_LEVELS levels): the image pyramid and,
 * computed by the same build, its gradient pyramid, in one device allocation laid out by
 * fe_pyramid_init.  Level sizes follow GPUImagePyramid::prepare_levels (image_pyramid.h:136-151). */
class GaussianGPUImagePyramid {
 public:
  enum { MaxPyramidLevels = FE_MAX_LEVELS };

  GaussianGPUImagePyramid() = default;
  explicit GaussianGPUImagePyramid(size_t width, size_t height) { prepare_levels(width, height); }
  GaussianGPUImagePyramid(GaussianGPUImagePyramid&&) noexcept = default;
  GaussianGPUImagePyramid& operator=(GaussianGPUImagePyramid&&) noexcept = default;

  void init(size_t width, size_t height) {
    if (desc_.levels == 0) prepare_levels(width, height);
  }

  /* GPUImagePyramid::build (image_pyramid.h:81-98) from an FP32 frame in device memory: level 0 is
   * the frame, each further level the reference's 5x5 filter-and-decimate, and every level's
   * gradients as GPUGradientPyramid::set computes them.  Asynchronous on `stream`. */
  void build(const GPUImageT& image, bool blur_filter, cudaStream_t& stream) {
    if (blur_filter)
      throw std::invalid_argument("GaussianGPUImagePyramid::build: the box prefilter runs on uint8 frames (build_u8)");
    if (desc_.levels == 0) prepare_levels(image.cols(), image.rows());
    check_size(image.cols(), image.rows());
    shim_check_fe(fe_build_pyramid_f32(ctx_.get(), image.ptr(), (int64_t)image.pitch(), desc_.width[0], desc_.height[0],
                                       &desc_, stream),
                  "GaussianGPUImagePyramid::build");
  }

  /* ImageContext::build_gpu_image_pyramid's MONO8 path (image_context.cpp:215-240: ImageCast::cast,
   * then build with blur_filter) from the uint8 frame in device memory, in one launch. */
  void build_u8(const uint8_t* image, size_t pitch_bytes, size_t width, size_t height, bool blur_filter,
                cudaStream_t& stream) {
    if (desc_.levels == 0) prepare_levels(width, height);
    check_size(width, height);
    shim_check_fe(fe_build_pyramid(ctx_.get(), image, (int64_t)pitch_bytes, (int)width, (int)height, blur_filter ? 1 : 0,
                                   &desc_, stream),
                  "GaussianGPUImagePyramid::build_u8");
  }

  /* The same path for RGB8 frames (cast_image_rgb's gray conversion, image_cast.cu:52-70). */
  void build_rgb8(const uint8_t* image, size_t pitch_bytes, size_t width, size_t height, bool blur_filter,
                  cudaStream_t& stream) {
    if (desc_.levels == 0) prepare_levels(width, height);
    check_size(width, height);
    shim_check_fe(fe_build_pyramid_rgb(ctx_.get(), image, (int64_t)pitch_bytes, (int)width, (int)height,
                                       blur_filter ? 1 : 0, &desc_, stream),
                  "GaussianGPUImagePyramid::build_rgb8");
  }

  int getLevelsCount() const { return desc_.levels; }
  size_t cols(int level = 0) const { return (size_t)desc_.width[level]; }
  size_t rows(int level = 0) const { return (size_t)desc_.height[level]; }
  /* Device planes of every level (image, grad_x, grad_y), for the other entry points of the ABI. */
  const fe_pyramid& desc() const { return desc_; }

 private:
  void prepare_levels(size_t width, size_t height) {
    if (width == 0 || height == 0 || width > (size_t)INT32_MAX || height > (size_t)INT32_MAX)
      throw std::invalid_argument("GaussianGPUImagePyramid: bad frame size");
    const int64_t bytes = fe_pyramid_bytes((int)width, (int)height, FE_MAX_LEVELS);
    if (bytes <= 0) throw std::invalid_argument("GaussianGPUImagePyramid: bad frame size");
    void* mem = nullptr;
    shim_check_cuda(cudaMalloc(&mem, (size_t)bytes), "GaussianGPUImagePyramid allocation");
    mem_.reset(mem);
    shim_check_fe(fe_pyramid_init(mem, bytes, (int)width, (int)height, FE_MAX_LEVELS, &desc_), "fe_pyramid_init");
  }
  void check_size(size_t width, size_t height) const {
    if (width != (size_t)desc_.width[0] || height != (size_t)desc_.height[0])
      throw std::invalid_argument("GaussianGPUImagePyramid: frame size differs from the pyramid's");
  }

  ShimContext ctx_;
  std::unique_ptr<void, ShimDeviceFree> mem_;
  fe_pyramid desc_ = {};
};

/* GPUGradientPyramid (gradient_pyramid.h:30-59): the gradient planes of an image pyramid.  The
 * pyramid's build already computed them, so set() only refers to them. */
class GPUGradientPyramid {
 public:
  GPUGradientPyramid() = default;
  GPUGradientPyramid(size_t width, size_t height) : width_(width), height_(height) {}

  int getLevelsCount() const { return desc_.levels; }
  void init(size_t width, size_t height) {
    width_ = width;
    height_ = height;
  }

  /* GPUGradientPyramid::set (gradient_pyramid.cpp:83-118): the gradients of `image`, both
   * directions (horizontal = true: only grad_x is meant to be read, as the reference then skips y). */
  bool set(const GaussianGPUImagePyramid& image, cudaStream_t& stream, bool horizontal = false) {
    (void)stream;
    if (image.getLevelsCount() == 0) throw std::invalid_argument("GPUGradientPyramid::set: pyramid not built");
    if (width_ && (width_ != image.cols() || height_ != image.rows()))
      throw std::invalid_argument("GPUGradientPyramid::set: pyramid size differs");
    desc_ = image.desc();
    horizontal_ = horizontal;
    return true;
  }

  bool horizontal() const { return horizontal_; }
  const fe_pyramid& desc() const { return desc_; }

 private:
  size_t width_ = 0, height_ = 0;
  bool horizontal_ = false;
  fe_pyramid desc_ = {};
};

/* GPUSelection (selection_v2.h:28-58): Shi-Tomasi response, NMS, suppression around the alive
 * features, per-cell candidates and the per-bin quota, on level 0 of the gradient pyramid. */
class GPUSelection {
 public:
  GPUSelection() = default;
  GPUSelection(const GPUSelection&) = delete;
  GPUSelection& operator=(const GPUSelection&) = delete;
  ~GPUSelection() {
    if (host_) cudaFreeHost(host_);
  }

  /* GPUSelection::computeGFTTAndSelectFeatures (selection_v2.cpp:27-184).  Blocking, as the
   * reference (it synchronises `stream` before returning).  Appends the new features to
   * newSelectedFeatures, at most num_desired_new_features entries counting the ones already there,
   * in the reference's order (strength, then the cell raster index where the reference leaves ties
   * to its sort).  input_mask (host, rows x cols = height x width, non-zero = masked) may be null. */
  void computeGFTTAndSelectFeatures(const GPUGradientPyramid& gradientPyramid, int border_top, int border_bottom,
                                    int border_left, int border_right, const ImageMatrix<uint8_t>* input_mask,
                                    const std::vector<Vector2T>& AliveFeatures, size_t num_desired_new_features,
                                    std::vector<Vector2T>& newSelectedFeatures, cudaStream_t& stream) {
    const fe_pyramid& p = gradientPyramid.desc();
    if (p.levels == 0) throw std::invalid_argument("computeGFTTAndSelectFeatures: gradient pyramid not set");
    const int w = p.width[0], h = p.height[0];
    if (num_desired_new_features > 16384 || AliveFeatures.size() > (size_t)INT32_MAX)
      throw std::invalid_argument("computeGFTTAndSelectFeatures: more features than fe_select takes");
    const int n_alive = (int)AliveFeatures.size(), k = (int)num_desired_new_features;
    const bool masked = input_mask != nullptr;
    if (masked && (input_mask->rows() != (size_t)h || input_mask->cols() != (size_t)w))
      throw std::invalid_argument("computeGFTTAndSelectFeatures: mask size differs from the image");
    reserve(n_alive, k, masked ? (size_t)w * h : 0);
    float* h_alive = host_;
    for (int i = 0; i < n_alive; ++i) {
      h_alive[2 * i] = AliveFeatures[i].x();
      h_alive[2 * i + 1] = AliveFeatures[i].y();
    }
    char* d = static_cast<char*>(dev_.get());
    float* d_alive = reinterpret_cast<float*>(d + off_alive_);
    float* d_out = reinterpret_cast<float*>(d + off_out_);
    int32_t* d_count = reinterpret_cast<int32_t*>(d + off_count_);
    uint8_t* d_mask = masked ? reinterpret_cast<uint8_t*>(d + off_mask_) : nullptr;
    if (n_alive > 0)
      shim_check_cuda(cudaMemcpyAsync(d_alive, h_alive, sizeof(float) * 2 * n_alive, cudaMemcpyHostToDevice, stream),
                      "computeGFTTAndSelectFeatures upload");
    if (masked)
      shim_check_cuda(cudaMemcpyAsync(d_mask, input_mask->data(), (size_t)w * h, cudaMemcpyHostToDevice, stream),
                      "computeGFTTAndSelectFeatures mask upload");
    shim_check_fe(fe_select(ctx_.get(), &p, border_top, border_bottom, border_left, border_right, d_mask, w,
                            n_alive > 0 ? d_alive : nullptr, n_alive, k, k > 0 ? d_out : nullptr, d_count, stream),
                  "computeGFTTAndSelectFeatures");
    float* h_out = host_ + 2 * (size_t)cap_alive_;
    int32_t* h_count = reinterpret_cast<int32_t*>(h_out + 2 * (size_t)cap_out_);
    shim_check_cuda(cudaMemcpyAsync(h_count, d_count, sizeof(int32_t), cudaMemcpyDeviceToHost, stream),
                    "computeGFTTAndSelectFeatures count");
    if (k > 0)
      shim_check_cuda(cudaMemcpyAsync(h_out, d_out, sizeof(float) * 2 * k, cudaMemcpyDeviceToHost, stream),
                      "computeGFTTAndSelectFeatures download");
    shim_check_cuda(cudaStreamSynchronize(stream), "computeGFTTAndSelectFeatures");
    const size_t n = (size_t)std::max(0, std::min(*h_count, k));
    const size_t room = num_desired_new_features > newSelectedFeatures.size()
                            ? num_desired_new_features - newSelectedFeatures.size()
                            : 0;
    for (size_t i = 0; i < std::min(n, room); ++i) newSelectedFeatures.emplace_back(h_out[2 * i], h_out[2 * i + 1]);
  }

 private:
  static size_t up256(size_t v) { return (v + 255) / 256 * 256; }
  // device: alive | out | count | mask; pinned host: alive | out | count
  void reserve(int n_alive, int k, size_t mask_bytes) {
    if (dev_ && n_alive <= cap_alive_ && k <= cap_out_ && mask_bytes <= cap_mask_) return;
    cap_alive_ = std::max(cap_alive_, std::max(n_alive, 1024));
    cap_out_ = std::max(cap_out_, std::max(k, 1024));
    cap_mask_ = std::max(cap_mask_, mask_bytes);
    off_alive_ = 0;
    off_out_ = up256(sizeof(float) * 2 * (size_t)cap_alive_);
    off_count_ = off_out_ + up256(sizeof(float) * 2 * (size_t)cap_out_);
    off_mask_ = off_count_ + 256;
    void* d = nullptr;
    dev_.reset();
    shim_check_cuda(cudaMalloc(&d, off_mask_ + std::max<size_t>(cap_mask_, 1)), "GPUSelection buffers");
    dev_.reset(d);
    if (host_) cudaFreeHost(host_);
    host_ = nullptr;
    shim_check_cuda(cudaMallocHost((void**)&host_, sizeof(float) * 2 * ((size_t)cap_alive_ + cap_out_) + 16),
                    "GPUSelection pinned buffers");
  }

  ShimContext ctx_;
  std::unique_ptr<void, ShimDeviceFree> dev_;
  float* host_ = nullptr;
  int cap_alive_ = 0, cap_out_ = 0;
  size_t cap_mask_ = 0, off_alive_ = 0, off_out_ = 0, off_count_ = 0, off_mask_ = 0;
};

/* GPULKFeatureTracker (lk_tracker.h:27-37): pyramidal LK of TrackData records in device memory. */
class GPULKFeatureTracker {
 public:
  /* sampling: FE_SAMPLE_HARDWARE (the default: the texture unit's own filtering on texture objects
   * of the pyramid planes, as the reference's kernels sample) or another fe_sampling mode
   * (FE_SAMPLE_TEXTURE restates that filtering in FP32, bit for bit with the CPU restatement). */
  explicit GPULKFeatureTracker(int sampling = FE_SAMPLE_HARDWARE) : sampling_(sampling) {}
  virtual ~GPULKFeatureTracker() = default;

  /* GPULKFeatureTracker::track_points (cuda_modules/lk_tracker.cpp:24-73): tracks the first
   * num_tracks records of track_data's DEVICE array from the previous frame to the current one, in
   * place, asynchronously on `stream` (the caller copies the records up before and back after, as
   * MonoSOFGPU::launch does).  Levels: the previous gradients' level count, as the reference. */
  virtual bool track_points(const GPUGradientPyramid& previous_image_gradients,
                            const GPUGradientPyramid& current_image_gradients,
                            const GaussianGPUImagePyramid& previous_image, const GaussianGPUImagePyramid& current_image,
                            GPUArrayPinned<TrackData>& track_data, size_t num_tracks, cudaStream_t& stream) {
    return track(previous_image_gradients, current_image_gradients, previous_image, current_image,
                 reinterpret_cast<fe_track_data*>(track_data.ptr()), num_tracks, stream, false);
  }

 protected:
  bool track(const GPUGradientPyramid& prev_grad, const GPUGradientPyramid& cur_grad, const GaussianGPUImagePyramid& prev,
             const GaussianGPUImagePyramid& cur, fe_track_data* tracks, size_t n, cudaStream_t& stream, bool horizontal) {
    (void)cur_grad;
    if (n == 0) return true;
    if (n > (size_t)INT32_MAX) throw std::invalid_argument("track_points: too many tracks");
    const fe_pyramid& g = prev_grad.desc();
    if (g.levels == 0 || prev.getLevelsCount() < g.levels || cur.getLevelsCount() < g.levels)
      throw std::invalid_argument("track_points: pyramids not built / gradients not set");
    // previous frame: the image pyramid's planes with the gradient pyramid's gradient planes
    fe_pyramid p = prev.desc(), c = cur.desc();
    p.levels = g.levels;
    c.levels = g.levels;
    for (int l = 0; l < g.levels; ++l) {
      p.grad_x[l] = g.grad_x[l];
      p.grad_y[l] = g.grad_y[l];
    }
    shim_check_fe(fe_track(ctx_.get(), &p, &c, tracks, (int)n, horizontal ? 1 : 0, sampling_, stream), "track_points");
    return true;
  }

  ShimContext ctx_;
  int sampling_;
};

/* GPULKTrackerHorizontal (lk_tracker.h:43-50, cuda_modules/lk_tracker.cpp:75-114): the 1-D tracker
 * of rectified stereo pairs (lk_track_horizontal_kernel). */
class GPULKTrackerHorizontal : public GPULKFeatureTracker {
 public:
  using GPULKFeatureTracker::GPULKFeatureTracker;
  bool track_points(const GPUGradientPyramid& previous_image_gradients, const GPUGradientPyramid& current_image_gradients,
                    const GaussianGPUImagePyramid& previous_image, const GaussianGPUImagePyramid& current_image,
                    GPUArrayPinned<TrackData>& track_data, size_t num_tracks, cudaStream_t& stream) override {
    return track(previous_image_gradients, current_image_gradients, previous_image, current_image,
                 reinterpret_cast<fe_track_data*>(track_data.ptr()), num_tracks, stream, true);
  }
};

}  // namespace cuda
}  // namespace cuvslam

#endif /* CUVSLAM_FE_SHIM_HPP */
