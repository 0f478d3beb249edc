// fe_select_noalloc: feature selection whose scratch memory lives in a static device array, for
// callers that cannot allocate device memory.
//
// Some callers must not call cudaMalloc once they are running: a tracking loop with a per-frame
// deadline that reserves all of its memory at start-up (cudaMalloc can synchronise the device and
// its latency is unbounded), or a host process whose device memory is entirely owned by its own
// pool allocator.  fe_select needs a context whose scratch it allocates on first use; this entry
// point takes no context and allocates nothing.  Its scratch is the file-scope array below, which
// every GPU that loads the library holds until the process exits.
//
// The kernels are the ones fe_select launches (select.cu); only where their scratch lives differs.
// No counterpart in the reference (GPUSelection allocates its buffers, selection_v2.h:28-58).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>

#include "cuvslam_fe.h"
#include "fe_common.cuh"
#include "fe_internal.h"

namespace {

// Limits of the static scratch.
constexpr int kMaxW = 2048;
constexpr int kMaxH = 2048;
constexpr int kMaxKept = 16384;  // kept candidates: min(cells, n_alive + num_desired + 64), fe_select's limit

constexpr size_t align256(size_t v) { return (v + 255) / 256 * 256; }

struct Layout {
  size_t stats, burn, zero_end, cell_m, cell_xy, sub_sum, bin_want, q_keys, total;
};

constexpr Layout layout(int w, int h, int q_cap) {
  Layout L{};
  size_t o = 0;
  L.stats = o;
  o = align256(o + 16 * sizeof(int));
  L.burn = o;
  o = align256(o + (size_t)((w + 31) / 32) * h * 4);
  L.zero_end = o;  // [0, zero_end) must be zero before every call
  L.cell_m = o;
  o = align256(o + (size_t)(w / 8) * (h / 8) * 4 + 4);
  L.cell_xy = o;
  o = align256(o + (size_t)(w / 8) * (h / 8) * 8 + 8);
  L.sub_sum = o;
  o = align256(o + (size_t)((w + 15) / 16) * ((h + 15) / 16) * 4);
  L.bin_want = o;
  o = align256(o + 128 * 4);
  L.q_keys = o;
  o = align256(o + (size_t)q_cap * 8);
  L.total = o;
  return L;
}

constexpr size_t kScratchBytes = layout(kMaxW, kMaxH, kMaxKept).total;  // about 1.5 MB

// The scratch.  Host code must not pass `g_select_scratch` itself to a kernel: on the host that
// name is a stand-in, not a device address.  The device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_select_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_lock;
void* g_scratch_addr[kMaxDevices] = {};

// Once per device, with that device current: the scratch's device address and the selection
// kernels' shared-memory attributes.  That set-up cannot run inside a stream capture (the symbol
// lookup and attribute calls are not capturable): a first call on a device made while `stream`
// captures is refused with FE_ERR_INVALID_ARGUMENT before anything is enqueued.
int setup_current_device(cudaStream_t stream, void** addr) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return FE_ERR_CUDA;
  std::lock_guard<std::mutex> lock(g_setup_lock);
  if (!g_scratch_addr[dev]) {
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(stream, &cap) != cudaSuccess) return FE_ERR_CUDA;
    if (cap != cudaStreamCaptureStatusNone) return FE_ERR_INVALID_ARGUMENT;
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_select_scratch) != cudaSuccess || !p) return FE_ERR_CUDA;
    if (fe::select_init() != cudaSuccess) return FE_ERR_CUDA;
    g_scratch_addr[dev] = p;
  }
  *addr = g_scratch_addr[dev];
  return FE_OK;
}

int pow2_at_least(int v) {
  int p = 1;
  while (p < v) p <<= 1;
  return p;
}

}  // namespace

extern "C" FE_API int fe_select_noalloc(const fe_pyramid* pyr, int border_top, int border_bottom, int border_left,
                                        int border_right, const uint8_t* mask, int64_t mask_pitch_bytes,
                                        const float* alive_xy, int n_alive, int num_desired, float* out_xy,
                                        int32_t* out_count, fe_stream stream) {
  if (!pyr || pyr->levels <= 0 || !pyr->grad_x[0] || !pyr->grad_y[0] || !out_count || n_alive < 0 ||
      num_desired < 0)
    return FE_ERR_INVALID_ARGUMENT;
  if ((n_alive > 0 && !alive_xy) || (num_desired > 0 && !out_xy)) return FE_ERR_INVALID_ARGUMENT;
  const int w = pyr->width[0], h = pyr->height[0];
  // the same level-0 checks as fe_select's: the response tiles copy the gradient planes with 16-byte
  // asynchronous copies, which need 16-byte aligned sources and pitches
  if (w <= 0 || h <= 0 || pyr->pitch_bytes[0] % 16 != 0 || pyr->pitch_bytes[0] < (int64_t)w * 4)
    return FE_ERR_INVALID_ARGUMENT;
  if (((uintptr_t)pyr->grad_x[0] | (uintptr_t)pyr->grad_y[0]) % 16 != 0) return FE_ERR_INVALID_ARGUMENT;
  if (mask && mask_pitch_bytes < w) return FE_ERR_INVALID_ARGUMENT;
  // sizes beyond the static scratch are rejected, never truncated; within 2048x2048 the limits are
  // fe_select's own (num_desired <= 16384, at most 16384 kept candidates)
  if (w > kMaxW || h > kMaxH || num_desired > 16384) return FE_ERR_CAPACITY;
  const int cw = w / 8, ch = h / 8;  // 8x8 cells
  const int q_cap = (int)std::min<int64_t>(std::max(cw * ch, 1), (int64_t)n_alive + num_desired + 64);
  if (q_cap > kMaxKept) return FE_ERR_CAPACITY;

  void* base = nullptr;
  int rc = setup_current_device((cudaStream_t)stream, &base);
  if (rc) return rc;

  // shared-memory key capacities: the largest candidate-cell rectangle of a bin, the kept keys
  const int bw = w / 8, bh = h / 8;  // bin size in pixels (8x8 bins)
  int bin_cap = 1;
  if (bw > 0 && bh > 0) {
    int mx = 1, my = 1;
    for (int b = 0; b < 8; ++b) {
      mx = std::max(mx, std::min(((b + 1) * bw) / 8, cw - 1) - std::max((b * bw - 1) / 8, 0) + 1);
      my = std::max(my, std::min(((b + 1) * bh) / 8, ch - 1) - std::max((b * bh - 1) / 8, 0) + 1);
    }
    bin_cap = pow2_at_least(mx * my);
  }
  const int final_cap = pow2_at_least(q_cap);
  if (bin_cap > fe::kMaxSelectKeys || final_cap > fe::kMaxSelectKeys) return FE_ERR_CAPACITY;

  const Layout L = layout(w, h, q_cap);
  char* s = (char*)base;
  cudaStream_t st = (cudaStream_t)stream;
  // the array keeps the previous call's contents: clear the counters and the burn mask
  if (cudaMemsetAsync(s, 0, L.zero_end, st) != cudaSuccess) return FE_ERR_CUDA;

  static thread_local fe::SelectBatch b;
  memset(&b, 0, sizeof(b));
  b.ncams = 1;
  fe::SelectCam& c = b.cam[0];
  c.gx = pyr->grad_x[0];
  c.gy = pyr->grad_y[0];
  c.w = w;
  c.h = h;
  c.pitch = (int)(pyr->pitch_bytes[0] / 4);
  c.mask = mask;
  c.mask_pitch = mask_pitch_bytes;
  c.alive_xy = alive_xy;
  c.n_alive = n_alive;
  c.num_desired = num_desired;
  c.border[0] = border_top;
  c.border[1] = border_bottom;
  c.border[2] = border_left;
  c.border[3] = border_right;
  c.out_xy = out_xy;
  c.out_count = out_count;
  c.stats = (int*)(s + L.stats);
  c.burn = (uint32_t*)(s + L.burn);
  c.cell_m = (float*)(s + L.cell_m);
  c.cell_xy = (float2*)(s + L.cell_xy);
  c.sub_sum = (float*)(s + L.sub_sum);
  c.bin_want = (int*)(s + L.bin_want);
  c.q_keys = (uint64_t*)(s + L.q_keys);
  c.q_cap = q_cap;
  c.tiles_x = (w + fe::select_tile_w() - 1) / fe::select_tile_w();
  c.tiles_y = (h + fe::select_tile_h() - 1) / fe::select_tile_h();
  c.tile_begin = 0;
  if (fe::launch_select(b, c.tiles_x * c.tiles_y, bin_cap, final_cap, st) != cudaSuccess) return FE_ERR_CUDA;
  return FE_OK;
}
