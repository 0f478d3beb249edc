// C ABI of the front-end (include/cuvslam_fe.h): argument checking, scratch management, launch
// planning for single cameras and batches, and CUDA-graph capture of batched frame steps.  It takes
// the place of the reference's host wrappers: GaussianGPUImagePyramid::build (image_pyramid.h:81-98),
// GPUGradientPyramid::set (gradient_pyramid.cpp:83-118), GPUSelection::computeGFTTAndSelectFeatures
// (selection_v2.cpp:27-184) and GPULKFeatureTracker::track_points (cuda_modules/lk_tracker.cpp:24-73).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "cuvslam_fe.h"
#include "fe_common.cuh"
#include "fe_internal.h"

static_assert(sizeof(fe_track_data) == 80, "fe_track_data must match cuvslam::cuda::TrackData");
static_assert(offsetof(fe_track_data, track_status) == 32, "TrackData layout");
static_assert(offsetof(fe_track_data, initial_guess_map) == 48, "TrackData layout");
static_assert(offsetof(fe_track_data, search_radius_px) == 64, "TrackData layout");
static_assert(offsetof(fe_track_data, ncc) == 72, "TrackData layout");

namespace {

thread_local int g_last_cuda_error = 0;

// Every device allocation of the library (one place to count or instrument them).
cudaError_t dev_alloc(void** p, size_t bytes) { return cudaMalloc(p, bytes); }

int cuda_fail(cudaError_t e) {
  g_last_cuda_error = (int)e;
  return e == cudaErrorMemoryAllocation ? FE_ERR_OUT_OF_MEMORY : FE_ERR_CUDA;
}

#define FE_CUDA(x)                                  \
  do {                                              \
    cudaError_t e_ = (x);                           \
    if (e_ != cudaSuccess) return cuda_fail(e_);    \
  } while (0)

constexpr int64_t kAlign = 256;
constexpr int64_t kPlaneAlign = 512;  // pyramid planes: the texture base alignment (FE_SAMPLE_HARDWARE)
constexpr int kMaxContextTextures = 4096;  // FE_SAMPLE_HARDWARE texture objects one context keeps
int64_t align_up(int64_t v, int64_t a) { return (v + a - 1) / a * a; }
int next_pow2(int v) {
  int p = 1;
  while (p < v) p <<= 1;
  return p;
}

int level_sizes(int w, int h, int max_levels, int* ws, int* hs) {
  if (w <= 0 || h <= 0 || max_levels <= 0) return 0;
  max_levels = std::min(max_levels, FE_MAX_LEVELS);
  int n = 0;
  while (n < max_levels) {
    ws[n] = w;
    hs[n] = h;
    ++n;
    w = (w + 1) / 2;
    h = (h + 1) / 2;
    if (w < fe::kMinLevelDim || h < fe::kMinLevelDim) break;
  }
  return n;
}

bool valid_pyramid(const fe_pyramid* p) {
  if (!p || p->levels <= 0 || p->levels > FE_MAX_LEVELS) return false;
  for (int l = 0; l < p->levels; ++l) {
    if (!p->image[l] || !p->grad_x[l] || p->width[l] <= 0 || p->height[l] <= 0) return false;
    // 16-byte aligned planes (vector loads/stores)
    if (((uintptr_t)p->image[l] | (uintptr_t)p->grad_x[l] | (uintptr_t)p->grad_y[l]) % 16 != 0) return false;
    if (p->pitch_bytes[l] % 16 != 0 || p->pitch_bytes[l] < (int64_t)p->width[l] * 4) return false;
    if (l > 0 && (p->width[l] != (p->width[l - 1] + 1) / 2 || p->height[l] != (p->height[l - 1] + 1) / 2)) return false;
  }
  return true;
}

fe::Pyr to_pyr(const fe_pyramid& p) {
  fe::Pyr r;
  memset(&r, 0, sizeof(r));
  r.levels = p.levels;
  for (int l = 0; l < p.levels; ++l) {
    r.lv[l].img = p.image[l];
    r.lv[l].gx = p.grad_x[l];
    r.lv[l].gy = p.grad_y[l];
    r.lv[l].w = p.width[l];
    r.lv[l].h = p.height[l];
    r.lv[l].pitch = (int)(p.pitch_bytes[l] / 4);
  }
  return r;
}

// ------------------------------------------------------------------ pyramid planning
// The deeper-level items of a levels 0-2 job (levels 3 .. of `pyr`): the rest item starts at the
// first level r (level 3, 4 or 5) from which every remaining level fits in the kernel's shared
// memory together; each level before it is a banded phase (its gradients and the next level's
// image, a band of rows per item).  False when no such split exists (the job then keeps the
// generic stages).
bool plan_deep_items(const fe::Pyr& pyr, fe::StageJob& job) {
  const int n = pyr.levels - 3, cap = fe::l012_deep_floats();
  if (n <= 0) return false;
  int r = -1;
  for (int k = 0; k < std::min(n, 3) && r < 0; ++k) {
    int64_t need = (int64_t)((pyr.lv[3 + k].w + 3) & ~3) * pyr.lv[3 + k].h;
    for (int m = k + 1; m < n; ++m) need += (int64_t)pyr.lv[3 + m].w * pyr.lv[3 + m].h;
    if (need <= cap) r = k;
  }
  if (r < 0) return false;
  job.deep_rest = r;
  job.deep_bands[0] = job.deep_bands[1] = 0;
  job.deep_band_rows[0] = job.deep_band_rows[1] = 0;
  job.deep_items = 1;
  for (int p = 0; p < r; ++p) {
    const int ws = (pyr.lv[3 + p].w + 3) & ~3;
    const int rows = (cap / ws - 6) / 2;  // level 3+p+1 rows per band: 2 rows + 6 halo rows staged each
    if (rows < 1) return false;
    job.deep_band_rows[p] = rows;
    job.deep_bands[p] = (pyr.lv[4 + p].h + rows - 1) / rows;
    job.deep_items += job.deep_bands[p];
  }
  job.tail_levels = n;
  for (int k = 0; k < n; ++k) job.tail[k] = pyr.lv[3 + k];
  return true;
}

// Launches of one stage index that share the source kind and the number of produced levels.
struct StageGroup {
  bool u8;
  int nl;
  bool tail;  // jobs whose last CTA computes the remaining levels (more shared memory)
  int kt;  // deepest-level tile of the generic stages (8 or 16)
  int tiles;
  fe::StageBatch batch;
};
using StagePlan = std::vector<std::vector<StageGroup>>;  // [stage index][group]

// Appends the stages of one camera's pyramid build: stage 0 reads the frame (uint8 or FP32) and
// writes levels 0..2; each later stage reads the deepest level of the previous one and writes up
// to two more.
// `counters` (device, zeroed, one int per job, *ncounters used so far of counter_cap): when given, a
// generic stage after which at most two small levels remain computes them in its last CTA (one
// launch fewer per remaining stage).
int plan_pyramid(const void* src, int64_t src_pitch, bool u8, const fe_pyramid& p, StagePlan& plan,
                 float scale = 1.f, int kt = 8, int* counters = nullptr, int* ncounters = nullptr,
                 int counter_cap = 0, bool box3 = false) {
  const fe::Pyr pyr = to_pyr(p);
  int s = 0;
  for (int stage = 0;; ++stage) {
    const int nl = std::min(2, pyr.levels - 1 - s);
    if (stage > 0 && nl <= 0) break;
    fe::StageJob job;
    memset(&job, 0, sizeof(job));
    job.src = stage == 0 ? src : (const void*)pyr.lv[s].img;
    job.src_pitch_bytes = stage == 0 ? src_pitch : (int64_t)pyr.lv[s].pitch * 4;
    job.write_level0 = stage == 0 ? 1 : 0;
    job.box3 = stage == 0 && u8 && box3 ? 1 : 0;
    job.scale = stage == 0 && !u8 ? scale : 1.f;
    job.src_w = pyr.lv[s].w;
    job.src_h = pyr.lv[s].h;
    for (int k = 0; k <= nl; ++k) job.out[k] = pyr.lv[s + k];
    const bool kind_u8 = stage == 0 && u8;
    const int T = fe::stage_tile(kind_u8, nl, kt);
    const fe::Level& deep = pyr.lv[s + nl];
    job.tiles_x = (deep.w + T - 1) / T;
    job.tiles_y = (deep.h + T - 1) / T;
    if (kind_u8 && nl == 2) fe::encode_frame_tmap(job);
    const int rem = pyr.levels - 1 - (s + std::max(nl, 0));
    if (kind_u8 && nl == 2 && rem > 0 && counters && *ncounters + 4 <= counter_cap && plan_deep_items(pyr, job)) {
      // the levels 0-2 launch also computes every deeper level (work items after the tiles)
      job.done = counters + *ncounters;
      *ncounters += 4;
    } else if (!(kind_u8 && nl == 2) && nl > 0 && rem > 0 && rem <= 2 && counters && *ncounters < counter_cap) {
      const fe::Level& deepest = pyr.lv[s + nl];
      const fe::Level& next = pyr.lv[s + nl + 1];
      if ((int64_t)deepest.w * deepest.h + (int64_t)next.w * next.h <= fe::kTailFloats) {
        job.tail_levels = rem;
        for (int k = 0; k < rem; ++k) job.tail[k] = pyr.lv[s + nl + 1 + k];
        job.done = counters + (*ncounters)++;
      }
    }
    if ((int)plan.size() <= stage) plan.resize(stage + 1);
    StageGroup* g = nullptr;
    const bool has_tail = job.tail_levels > 0;
    for (auto& gg : plan[stage])
      if (gg.u8 == kind_u8 && gg.nl == nl && gg.tail == has_tail && gg.batch.njobs < fe::kMaxStageJobs) g = &gg;
    if (!g) {
      plan[stage].emplace_back();
      g = &plan[stage].back();
      memset(&g->batch, 0, sizeof(g->batch));
      g->u8 = kind_u8;
      g->nl = nl;
      g->tail = has_tail;
      g->kt = kt;
      g->tiles = 0;
    }
    job.tile_begin = g->tiles;
    g->batch.job[g->batch.njobs++] = job;
    g->tiles += job.tiles_x * job.tiles_y;
    if (nl <= 0 || job.tail_levels > 0) break;
    s += nl;
  }
  return FE_OK;
}

// The launches of stages [first, last) of a plan.
int run_stages(const StagePlan& plan, size_t first, size_t last, cudaStream_t st) {
  for (size_t k = first; k < std::min(last, plan.size()); ++k)
    for (const auto& g : plan[k]) FE_CUDA(fe::launch_pyramid_stage(g.batch, g.tiles, g.u8, g.nl, g.kt, g.tail, st));
  return FE_OK;
}

// Lays out the work queue of each levels 0-2 launch whose jobs compute their deeper levels: jobs by
// frame size, largest first (their deeper levels are the most work), each job's tiles, and each
// job's deeper-level items after the next job's tiles (by then its tiles are usually done).
// `queues`: two zeroed ints per such launch (*nqueues used so far of queue_cap).
int finish_l012_plan(StagePlan& plan, int* queues, int* nqueues, int queue_cap) {
  if (plan.empty()) return FE_OK;
  for (auto& g : plan[0]) {
    if (!(g.u8 && g.nl == 2 && g.tail)) continue;
    fe::StageJob* J = g.batch.job;
    const int n = g.batch.njobs;
    std::stable_sort(J, J + n, [](const fe::StageJob& a, const fe::StageJob& b) {
      return (int64_t)a.src_w * a.src_h > (int64_t)b.src_w * b.src_h;
    });
    int q = 0;
    for (int i = 0; i < n; ++i) {
      J[i].tile_begin = q;
      q += J[i].tiles_x * J[i].tiles_y;
      if (i > 0) {
        J[i - 1].q_deep = q;
        q += J[i - 1].deep_items;
      }
    }
    J[n - 1].q_deep = q;
    q += J[n - 1].deep_items;
    if (*nqueues + 2 > queue_cap) return FE_ERR_CAPACITY;
    g.batch.queue = queues + *nqueues;
    *nqueues += 2;
    g.tiles = q;
  }
  return FE_OK;
}

int run_plan(const StagePlan& plan, cudaStream_t st) {
  for (const auto& stage : plan)
    for (const auto& g : stage) FE_CUDA(fe::launch_pyramid_stage(g.batch, g.tiles, g.u8, g.nl, g.kt, g.tail, st));
  return FE_OK;
}

}  // namespace

// ------------------------------------------------------------------ context
struct SelectScratch {
  int w = 0, h = 0, n_alive_cap = 0, q_cap = 0;
  void* mem = nullptr;
  size_t bytes = 0;
  float* resp = nullptr;  // debug maps, allocated on demand
  float* nms = nullptr;
  uint32_t* burn = nullptr;
  float* cell_m = nullptr;
  float2* cell_xy = nullptr;
  float* sub_sum = nullptr;
  int* bin_want = nullptr;
  int* stats = nullptr;
  uint64_t* q_keys = nullptr;
  float* alive_xy = nullptr;
  size_t burn_bytes = 0, zero_bytes = 0;  // bytes to clear per run (burn + stats)
};

struct fe_context {
  int device = 0;
  SelectScratch sel;
  int* lk_counter = nullptr;  // persistent LK warps' track counter
  int* stage_done = nullptr;  // fe_build_pyramid's CTA counters (the levels 0-2 kernel's last CTA per
                              // frame computes the deeper levels): 64, used in turn
  unsigned stage_slot = 0;
  unsigned long long* finish_cells = nullptr;  // fe_finish_tracks' collapse cells (zero between calls)
  size_t finish_cap = 0;
  void* stereo_mem = nullptr;  // left-to-right matching scratch (grown on demand)
  size_t stereo_bytes = 0;
  bool debug = false;
  int* dev_status = nullptr;  // device flags the kernels set (fe_device_status reads and clears them)
  int wait_limit = fe::kDefaultWaitLimit;  // bounded waits' iteration limit (fe_set_wait_limit)
  // FE_SAMPLE_HARDWARE: texture objects of the planes tracked on, created on first use
  struct Tex {
    const void* ptr;
    int w, h;
    int64_t pitch;
    cudaTextureObject_t t;
  };
  std::vector<Tex> tex;
};

namespace {

// Points every pyramid launch of a plan at the context's device status word and gives it the
// context's wait limit.
void stamp_plan(StagePlan& plan, const fe_context* ctx) {
  for (auto& stage : plan)
    for (auto& g : stage) {
      g.batch.status = ctx->dev_status;
      g.batch.wait_limit = ctx->wait_limit;
    }
}

// The texture object (linear filtering, clamped, unnormalised coordinates: the reference's sampling
// of its pyramid planes) of one plane, from the context's cache or created now.
int plane_texture(fe_context* ctx, const float* ptr, int w, int h, int64_t pitch, unsigned long long* out) {
  for (const auto& t : ctx->tex)
    if (t.ptr == ptr && t.w == w && t.h == h && t.pitch == pitch) {
      *out = (unsigned long long)t.t;
      return FE_OK;
    }
  int base_align = 0, pitch_align = 0;
  if (cudaDeviceGetAttribute(&base_align, cudaDevAttrTextureAlignment, ctx->device) != cudaSuccess || base_align <= 0)
    base_align = 512;
  if (cudaDeviceGetAttribute(&pitch_align, cudaDevAttrTexturePitchAlignment, ctx->device) != cudaSuccess ||
      pitch_align <= 0)
    pitch_align = 32;
  if ((uintptr_t)ptr % (uintptr_t)base_align != 0 || pitch % pitch_align != 0) return FE_ERR_INVALID_ARGUMENT;
  // kept until fe_destroy (a kernel in flight may still read one): a bounded number per context
  if (ctx->tex.size() >= (size_t)kMaxContextTextures) return FE_ERR_CAPACITY;
  cudaResourceDesc rd;
  memset(&rd, 0, sizeof(rd));
  rd.resType = cudaResourceTypePitch2D;
  rd.res.pitch2D.devPtr = const_cast<float*>(ptr);
  rd.res.pitch2D.width = (size_t)w;
  rd.res.pitch2D.height = (size_t)h;
  rd.res.pitch2D.pitchInBytes = (size_t)pitch;
  rd.res.pitch2D.desc = cudaCreateChannelDesc(32, 0, 0, 0, cudaChannelFormatKindFloat);
  cudaTextureDesc td;
  memset(&td, 0, sizeof(td));
  td.addressMode[0] = cudaAddressModeClamp;
  td.addressMode[1] = cudaAddressModeClamp;
  td.filterMode = cudaFilterModeLinear;
  td.readMode = cudaReadModeElementType;
  td.normalizedCoords = 0;
  cudaTextureObject_t t = 0;
  if (cudaCreateTextureObject(&t, &rd, &td, nullptr) != cudaSuccess) {
    cudaGetLastError();
    return FE_ERR_INVALID_ARGUMENT;
  }
  ctx->tex.push_back({ptr, w, h, pitch, t});
  *out = (unsigned long long)t;
  return FE_OK;
}

// The texture objects LK with FE_SAMPLE_HARDWARE reads: previous image and gradients, current image.
int lk_textures(fe_context* ctx, const fe_pyramid& prev, const fe_pyramid& cur, bool horizontal, fe::LkTex& out) {
  memset(&out, 0, sizeof(out));
  for (int l = 0; l < prev.levels; ++l) {
    int rc = plane_texture(ctx, prev.image[l], prev.width[l], prev.height[l], prev.pitch_bytes[l], &out.prev_img[l]);
    if (!rc) rc = plane_texture(ctx, prev.grad_x[l], prev.width[l], prev.height[l], prev.pitch_bytes[l], &out.prev_gx[l]);
    if (!rc && !horizontal)
      rc = plane_texture(ctx, prev.grad_y[l], prev.width[l], prev.height[l], prev.pitch_bytes[l], &out.prev_gy[l]);
    if (!rc) rc = plane_texture(ctx, cur.image[l], cur.width[l], cur.height[l], cur.pitch_bytes[l], &out.cur_img[l]);
    if (rc) return rc;
  }
  return FE_OK;
}

}  // namespace

namespace {

struct ScratchLayout {
  size_t burn, cell_m, cell_xy, sub_sum, bin_want, stats, q_keys, alive, total, burn_bytes;
};

ScratchLayout scratch_layout(int w, int h, int n_alive_cap, int q_cap) {
  ScratchLayout L;
  size_t o = 0;
  auto take = [&](size_t bytes) {
    size_t at = o;
    o = (size_t)align_up((int64_t)(o + bytes), kAlign);
    return at;
  };
  const size_t words = (size_t)((w + 31) / 32) * h;
  const size_t cells = (size_t)(w / 8) * (h / 8);
  const size_t subs = (size_t)((w + 15) / 16) * ((h + 15) / 16);
  L.stats = take(16 * sizeof(int));  // first so one memset clears stats + burn
  L.burn = take(words * 4);
  L.burn_bytes = L.burn + words * 4;
  L.cell_m = take(std::max<size_t>(cells, 1) * 4);
  L.cell_xy = take(std::max<size_t>(cells, 1) * 8);
  L.sub_sum = take(subs * 4);
  L.bin_want = take(128 * 4);
  L.q_keys = take((size_t)std::max(q_cap, 1) * 8);
  L.alive = take((size_t)std::max(n_alive_cap, 1) * 8);
  L.total = o;
  return L;
}

// Shared-memory key capacities of bin_kernel (largest candidate-cell rectangle of a bin) and
// final_kernel (kept candidates), and the kept-candidate buffer size.
int sel_caps(int w, int h, int n_alive, int num_desired, int* bin_key_cap, int* final_key_cap, int* q_cap) {
  const int cw = w / 8, ch = h / 8, bw = w / 8, bh = h / 8;
  int mx = 1;
  if (bw > 0 && bh > 0) {
    int mxx = 1, mxy = 1;
    for (int b = 0; b < 8; ++b) {
      mxx = std::max(mxx, std::min(((b + 1) * bw) / 8, cw - 1) - std::max((b * bw - 1) / 8, 0) + 1);
      mxy = std::max(mxy, std::min(((b + 1) * bh) / 8, ch - 1) - std::max((b * bh - 1) / 8, 0) + 1);
    }
    mx = mxx * mxy;
  }
  *bin_key_cap = next_pow2(mx);
  const int cells = std::max(cw * ch, 1);
  *q_cap = (int)std::min<int64_t>(cells, (int64_t)std::max(n_alive, 0) + num_desired + 64);
  *final_key_cap = next_pow2(*q_cap);
  if (*bin_key_cap > 16384 || *final_key_cap > 16384) return FE_ERR_CAPACITY;
  return FE_OK;
}

int ensure_select_scratch(fe_context* ctx, int w, int h, int n_alive_cap, int q_cap) {
  SelectScratch& s = ctx->sel;
  if (s.mem && s.w == w && s.h == h && s.n_alive_cap >= n_alive_cap && s.q_cap >= q_cap) return FE_OK;
  const int na = std::max(n_alive_cap, s.w == w && s.h == h ? s.n_alive_cap : 0);
  const int qc = std::max(q_cap, s.w == w && s.h == h ? s.q_cap : 0);
  ScratchLayout L = scratch_layout(w, h, na, qc);
  if (s.mem) cudaFree(s.mem);
  s.mem = nullptr;
  FE_CUDA(dev_alloc((void**)&s.mem, L.total));
  char* base = (char*)s.mem;
  s.w = w;
  s.h = h;
  s.n_alive_cap = na;
  s.q_cap = qc;
  s.bytes = L.total;
  s.stats = (int*)(base + L.stats);
  s.burn = (uint32_t*)(base + L.burn);
  s.cell_m = (float*)(base + L.cell_m);
  s.cell_xy = (float2*)(base + L.cell_xy);
  s.sub_sum = (float*)(base + L.sub_sum);
  s.bin_want = (int*)(base + L.bin_want);
  s.q_keys = (uint64_t*)(base + L.q_keys);
  s.alive_xy = (float*)(base + L.alive);
  s.zero_bytes = L.burn_bytes;
  if (s.resp) cudaFree(s.resp);
  if (s.nms) cudaFree(s.nms);
  s.resp = s.nms = nullptr;
  return FE_OK;
}

void fill_select_cam(fe::SelectCam& c, const SelectScratch& s, const fe_pyramid& p, int q_cap) {
  memset(&c, 0, sizeof(c));
  c.gx = p.grad_x[0];
  c.gy = p.grad_y[0];
  c.w = p.width[0];
  c.h = p.height[0];
  c.pitch = (int)(p.pitch_bytes[0] / 4);
  c.resp = s.resp;
  c.nms = s.nms;
  c.burn = s.burn;
  c.cell_m = s.cell_m;
  c.cell_xy = s.cell_xy;
  c.sub_sum = s.sub_sum;
  c.bin_want = s.bin_want;
  c.stats = s.stats;
  c.q_keys = s.q_keys;
  c.q_cap = q_cap;
  c.tiles_x = (c.w + fe::select_tile_w() - 1) / fe::select_tile_w();
  c.tiles_y = (c.h + fe::select_tile_h() - 1) / fe::select_tile_h();
}

}  // namespace

extern "C" {

int fe_abi_version(void) { return FE_ABI_VERSION; }

const char* fe_status_string(int status) {
  switch (status) {
    case FE_OK: return "ok";
    case FE_ERR_INVALID_ARGUMENT: return "invalid argument";
    case FE_ERR_CUDA: return "CUDA error";
    case FE_ERR_OUT_OF_MEMORY: return "out of device memory";
    case FE_ERR_CAPACITY: return "size limit exceeded";
    case FE_ERR_DEVICE_FAULT: return "device-side error flag";
    default: return "unknown status";
  }
}

int fe_last_cuda_error(void) { return g_last_cuda_error; }

int fe_create(int device, fe_context** out) {
  if (!out) return FE_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int n = 0;
  FE_CUDA(cudaGetDeviceCount(&n));
  if (device < 0 || device >= n) return FE_ERR_INVALID_ARGUMENT;
  FE_CUDA(cudaSetDevice(device));
  FE_CUDA(fe::pyramid_init());
  FE_CUDA(fe::select_init());
  FE_CUDA(fe::adjoint_init());
  fe_context* c = new (std::nothrow) fe_context;
  if (!c) return FE_ERR_OUT_OF_MEMORY;
  c->device = device;
  c->debug = getenv("CUVSLAM_FE_DEBUG_MAPS") != nullptr;
  cudaError_t e = dev_alloc((void**)&c->lk_counter, 256);
  if (e == cudaSuccess) e = dev_alloc((void**)&c->stage_done, 64 * 8 * sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(c->stage_done, 0, 64 * 8 * sizeof(int));
  if (e == cudaSuccess) e = dev_alloc((void**)&c->dev_status, 4 * sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(c->dev_status, 0, 4 * sizeof(int));
  if (e != cudaSuccess) {
    if (c->lk_counter) cudaFree(c->lk_counter);
    if (c->stage_done) cudaFree(c->stage_done);
    if (c->dev_status) cudaFree(c->dev_status);
    delete c;
    return cuda_fail(e);
  }
  *out = c;
  return FE_OK;
}

int fe_destroy(fe_context* ctx) {
  if (!ctx) return FE_ERR_INVALID_ARGUMENT;
  for (const auto& t : ctx->tex) cudaDestroyTextureObject(t.t);
  if (ctx->sel.mem) cudaFree(ctx->sel.mem);
  if (ctx->lk_counter) cudaFree(ctx->lk_counter);
  if (ctx->stage_done) cudaFree(ctx->stage_done);
  if (ctx->dev_status) cudaFree(ctx->dev_status);
  if (ctx->stereo_mem) cudaFree(ctx->stereo_mem);
  if (ctx->finish_cells) cudaFree(ctx->finish_cells);
  if (ctx->sel.resp) cudaFree(ctx->sel.resp);
  if (ctx->sel.nms) cudaFree(ctx->sel.nms);
  delete ctx;
  return FE_OK;
}

int fe_pyramid_levels(int width, int height, int max_levels) {
  int ws[FE_MAX_LEVELS], hs[FE_MAX_LEVELS];
  return level_sizes(width, height, max_levels, ws, hs);
}

int64_t fe_pyramid_bytes(int width, int height, int max_levels) {
  int ws[FE_MAX_LEVELS], hs[FE_MAX_LEVELS];
  const int n = level_sizes(width, height, max_levels, ws, hs);
  int64_t total = 0;
  for (int l = 0; l < n; ++l) total += 3 * align_up(align_up((int64_t)ws[l] * 4, kAlign) * hs[l], kPlaneAlign);
  return total;
}

int fe_pyramid_init(void* device_memory, int64_t bytes, int width, int height, int max_levels, fe_pyramid* out) {
  if (!device_memory || !out || ((uintptr_t)device_memory % kAlign) != 0) return FE_ERR_INVALID_ARGUMENT;
  int ws[FE_MAX_LEVELS], hs[FE_MAX_LEVELS];
  const int n = level_sizes(width, height, max_levels, ws, hs);
  if (n == 0) return FE_ERR_INVALID_ARGUMENT;
  if (bytes < fe_pyramid_bytes(width, height, max_levels)) return FE_ERR_INVALID_ARGUMENT;
  memset(out, 0, sizeof(*out));
  out->levels = n;
  char* p = (char*)device_memory;
  for (int l = 0; l < n; ++l) {
    const int64_t pitch = align_up((int64_t)ws[l] * 4, kAlign);
    const int64_t plane = align_up(pitch * hs[l], kPlaneAlign);
    out->width[l] = ws[l];
    out->height[l] = hs[l];
    out->pitch_bytes[l] = pitch;
    out->image[l] = (float*)p;
    out->grad_x[l] = (float*)(p + plane);
    out->grad_y[l] = (float*)(p + 2 * plane);
    p += 3 * plane;
  }
  return FE_OK;
}

// The pyramid of a level 0 already in pyr->image[0] (the input stage wrote it): the FP32 plan, whose
// first stage rewrites level 0 with the same values while it computes the gradients.
int build_from_level0(fe_context* ctx, const fe_pyramid* pyr, cudaStream_t s) {
  StagePlan plan;
  int rc = plan_pyramid(pyr->image[0], pyr->pitch_bytes[0], false, *pyr, plan);
  if (rc) return rc;
  stamp_plan(plan, ctx);
  return run_plan(plan, s);
}

int fe_build_pyramid(fe_context* ctx, const uint8_t* image, int64_t image_pitch_bytes, int width, int height,
                     int box3, const fe_pyramid* pyr, fe_stream stream) {
  if (!ctx || !image || !valid_pyramid(pyr) || (box3 != 0 && box3 != 1)) return FE_ERR_INVALID_ARGUMENT;
  if (pyr->width[0] != width || pyr->height[0] != height || image_pitch_bytes < width) return FE_ERR_INVALID_ARGUMENT;
  if (!pyr->grad_y[0]) return FE_ERR_INVALID_ARGUMENT;
  if (box3 && pyr->levels < 3) {
    // frames too small for the levels 0-2 kernel: the prefilter as its own input stage
    FE_CUDA(fe::launch_input_stage(image, image_pitch_bytes, 1, 1, width, height, pyr->image[0],
                                   pyr->pitch_bytes[0] / 4, (cudaStream_t)stream));
    return build_from_level0(ctx, pyr, (cudaStream_t)stream);
  }
  StagePlan plan;
  // one of the context's 64 counter sets per call, in turn (at most 64 builds in flight per context)
  int used = 0, nq = 0;
  int* done = ctx->stage_done + 8 * (ctx->stage_slot++ & 63);
  int rc = plan_pyramid(image, image_pitch_bytes, true, *pyr, plan, 1.f, 8, done, &used, 4, box3 != 0);
  if (!rc) rc = finish_l012_plan(plan, done + 4, &nq, 2);
  if (rc) return rc;
  stamp_plan(plan, ctx);
  return run_plan(plan, (cudaStream_t)stream);
}

int fe_build_pyramid_rgb(fe_context* ctx, const uint8_t* image, int64_t image_pitch_bytes, int width, int height,
                         int box3, const fe_pyramid* pyr, fe_stream stream) {
  if (!ctx || !image || !valid_pyramid(pyr) || (box3 != 0 && box3 != 1)) return FE_ERR_INVALID_ARGUMENT;
  if (pyr->width[0] != width || pyr->height[0] != height || image_pitch_bytes < 3 * (int64_t)width)
    return FE_ERR_INVALID_ARGUMENT;
  if (!pyr->grad_y[0]) return FE_ERR_INVALID_ARGUMENT;
  FE_CUDA(fe::launch_input_stage(image, image_pitch_bytes, 3, box3, width, height, pyr->image[0],
                                 pyr->pitch_bytes[0] / 4, (cudaStream_t)stream));
  return build_from_level0(ctx, pyr, (cudaStream_t)stream);
}

int fe_build_pyramid_f32(fe_context* ctx, const float* image, int64_t image_pitch_bytes, int width, int height,
                         const fe_pyramid* pyr, fe_stream stream) {
  if (!ctx || !image || !valid_pyramid(pyr)) return FE_ERR_INVALID_ARGUMENT;
  if (pyr->width[0] != width || pyr->height[0] != height || image_pitch_bytes < (int64_t)width * 4 ||
      image_pitch_bytes % 4 != 0)
    return FE_ERR_INVALID_ARGUMENT;
  StagePlan plan;
  int rc = plan_pyramid(image, image_pitch_bytes, false, *pyr, plan);
  if (rc) return rc;
  stamp_plan(plan, ctx);
  return run_plan(plan, (cudaStream_t)stream);
}

int fe_select(fe_context* ctx, const fe_pyramid* pyr, int border_top, int border_bottom, int border_left,
              int border_right, const uint8_t* mask, int64_t mask_pitch_bytes, const float* alive_xy, int n_alive,
              int num_desired, float* out_xy, int32_t* out_count, fe_stream stream) {
  if (!ctx || !valid_pyramid(pyr) || !pyr->grad_y[0] || !out_count || n_alive < 0 || num_desired < 0)
    return FE_ERR_INVALID_ARGUMENT;
  if ((n_alive > 0 && !alive_xy) || (num_desired > 0 && !out_xy)) return FE_ERR_INVALID_ARGUMENT;
  const int w = pyr->width[0], h = pyr->height[0];
  if (w > 4096 || h > 4096 || num_desired > 16384) return FE_ERR_CAPACITY;
  if (mask && mask_pitch_bytes < w) return FE_ERR_INVALID_ARGUMENT;
  int bin_cap, final_cap, q_cap;
  int rc = sel_caps(w, h, n_alive, num_desired, &bin_cap, &final_cap, &q_cap);
  if (rc) return rc;
  rc = ensure_select_scratch(ctx, w, h, 0, q_cap);
  if (rc) return rc;
  SelectScratch& s = ctx->sel;
  if (ctx->debug && !s.resp) {
    FE_CUDA(dev_alloc((void**)&s.resp, (size_t)w * h * 4));
    FE_CUDA(dev_alloc((void**)&s.nms, (size_t)w * h * 4));
  }
  cudaStream_t st = (cudaStream_t)stream;
  FE_CUDA(cudaMemsetAsync(s.mem, 0, s.zero_bytes, st));
  static thread_local fe::SelectBatch b;  // large: keep off the stack
  memset(&b, 0, sizeof(b));
  b.ncams = 1;
  b.debug = ctx->debug ? 1 : 0;
  fe::SelectCam& c = b.cam[0];
  fill_select_cam(c, s, *pyr, q_cap);
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
  c.tile_begin = 0;
  FE_CUDA(fe::launch_select(b, c.tiles_x * c.tiles_y, bin_cap, final_cap, st));
  return FE_OK;
}

int fe_device_status(fe_context* ctx, fe_stream stream, int32_t* flags) {
  if (!ctx) return FE_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  int h[4] = {0, 0, 0, 0};
  FE_CUDA(cudaStreamSynchronize(st));
  FE_CUDA(cudaMemcpy(h, ctx->dev_status, sizeof(h), cudaMemcpyDeviceToHost));
  FE_CUDA(cudaMemset(ctx->dev_status, 0, sizeof(h)));
  if (flags) *flags = h[0];
  return h[0] ? FE_ERR_DEVICE_FAULT : FE_OK;
}

int fe_set_wait_limit(fe_context* ctx, int iterations) {
  if (!ctx || iterations < 0) return FE_ERR_INVALID_ARGUMENT;
  ctx->wait_limit = iterations;
  return FE_OK;
}

int fe_select_debug(fe_context* ctx, const float** response, const float** nms) {
  if (!ctx || !response || !nms) return FE_ERR_INVALID_ARGUMENT;
  *response = ctx->sel.resp;
  *nms = ctx->sel.nms;
  return ctx->debug ? FE_OK : FE_ERR_INVALID_ARGUMENT;
}

int fe_track(fe_context* ctx, const fe_pyramid* prev, const fe_pyramid* cur, fe_track_data* tracks, int n,
             int horizontal, int sampling, fe_stream stream) {
  if (!ctx || !valid_pyramid(prev) || !valid_pyramid(cur) || n < 0 || (n > 0 && !tracks)) return FE_ERR_INVALID_ARGUMENT;
  if (cur->levels < prev->levels) return FE_ERR_INVALID_ARGUMENT;
  if (sampling < FE_SAMPLE_TEXTURE || sampling > FE_SAMPLE_HARDWARE) return FE_ERR_INVALID_ARGUMENT;
  if (!horizontal)
    for (int l = 0; l < prev->levels; ++l)
      if (!prev->grad_y[l]) return FE_ERR_INVALID_ARGUMENT;
  if ((uintptr_t)tracks % 16 != 0) return FE_ERR_INVALID_ARGUMENT;
  if (n == 0) return FE_OK;
  fe::LkLaunch p;
  memset(&p, 0, sizeof(p));
  p.cams = nullptr;
  p.counter = ctx->lk_counter;
  p.ncams = 1;
  p.total = n;
  p.horizontal = horizontal ? 1 : 0;
  p.sampling = sampling;
  p.single.prev = to_pyr(*prev);
  p.single.cur = to_pyr(*cur);
  p.single.tracks = tracks;
  p.single.n = n;
  p.single.begin = 0;
  if (sampling == FE_SAMPLE_HARDWARE) {
    const int rc = lk_textures(ctx, *prev, *cur, horizontal != 0, p.single_tex);
    if (rc) return rc;
  }
  FE_CUDA(fe::launch_lk(p, (cudaStream_t)stream));
  return FE_OK;
}

int fe_track_mono(fe_context* ctx, const fe_pyramid* prev, const fe_pyramid* cur, fe_track_data* tracks, int n,
                  float retrack_ncc, int sampling, fe_stream stream) {
  if (!(retrack_ncc == retrack_ncc)) return FE_ERR_INVALID_ARGUMENT;
  if (!ctx || !valid_pyramid(prev) || !valid_pyramid(cur) || n < 0 || (n > 0 && !tracks)) return FE_ERR_INVALID_ARGUMENT;
  if (cur->levels < prev->levels) return FE_ERR_INVALID_ARGUMENT;
  if (sampling < FE_SAMPLE_TEXTURE || sampling > FE_SAMPLE_HARDWARE) return FE_ERR_INVALID_ARGUMENT;
  for (int l = 0; l < prev->levels; ++l)
    if (!prev->grad_y[l]) return FE_ERR_INVALID_ARGUMENT;
  if ((uintptr_t)tracks % 16 != 0) return FE_ERR_INVALID_ARGUMENT;
  if (n == 0) return FE_OK;
  fe::LkLaunch p;
  memset(&p, 0, sizeof(p));
  p.counter = ctx->lk_counter;
  p.ncams = 1;
  p.total = n;
  p.sampling = sampling;
  p.single.prev = to_pyr(*prev);
  p.single.cur = to_pyr(*cur);
  p.single.tracks = tracks;
  p.single.n = n;
  p.single.retrack_ncc = retrack_ncc > 0.f ? retrack_ncc : 0.f;
  if (sampling == FE_SAMPLE_HARDWARE) {
    const int rc = lk_textures(ctx, *prev, *cur, false, p.single_tex);
    if (rc) return rc;
  }
  FE_CUDA(fe::launch_lk(p, (cudaStream_t)stream));
  return FE_OK;
}

namespace {

int affine_args(fe_context* ctx, const fe_pyramid* cur, fe_track_data* tracks, int n, int n_shift, int n_full,
                int sampling) {
  if (!ctx || !valid_pyramid(cur) || n < 0 || (n > 0 && !tracks)) return FE_ERR_INVALID_ARGUMENT;
  if (n_shift < 0 || n_full < 0 || n_shift > 1000 || n_full > 1000) return FE_ERR_INVALID_ARGUMENT;
  if (sampling < FE_SAMPLE_TEXTURE || sampling > FE_SAMPLE_TEXTURE_WIDE) return FE_ERR_INVALID_ARGUMENT;
  for (int l = 0; l < cur->levels; ++l)
    if (!cur->grad_y[l]) return FE_ERR_INVALID_ARGUMENT;
  if ((uintptr_t)tracks % 16 != 0) return FE_ERR_INVALID_ARGUMENT;
  return FE_OK;
}

}  // namespace

int fe_track_affine(fe_context* ctx, const fe_pyramid* prev, const fe_pyramid* cur, fe_track_data* tracks, int n,
                    int n_shift_iterations, int n_full_iterations, int sampling, fe_stream stream) {
  const int rc = affine_args(ctx, cur, tracks, n, n_shift_iterations, n_full_iterations, sampling);
  if (rc) return rc;
  if (!valid_pyramid(prev) || prev->levels < cur->levels) return FE_ERR_INVALID_ARGUMENT;
  for (int l = 0; l < cur->levels; ++l)
    if (prev->width[l] != cur->width[l] || prev->height[l] != cur->height[l]) return FE_ERR_INVALID_ARGUMENT;
  if (n == 0) return FE_OK;
  fe::StLaunch p;
  memset(&p, 0, sizeof(p));
  p.prev = to_pyr(*prev);
  p.cur = to_pyr(*cur);
  p.tracks = tracks;
  p.n = n;
  p.n_shift = n_shift_iterations;
  p.n_full = n_full_iterations;
  p.sampling = sampling;
  p.counter = ctx->lk_counter + 32;
  FE_CUDA(fe::launch_st(p, 0, (cudaStream_t)stream));
  return FE_OK;
}

int fe_affine_build_cache(fe_context* ctx, const fe_pyramid* prev, fe_track_data* tracks, int n,
                          fe_affine_cache* cache, int sampling, fe_stream stream) {
  if (!ctx || !valid_pyramid(prev) || n < 0 || (n > 0 && (!tracks || !cache))) return FE_ERR_INVALID_ARGUMENT;
  if (sampling < FE_SAMPLE_TEXTURE || sampling > FE_SAMPLE_TEXTURE_WIDE) return FE_ERR_INVALID_ARGUMENT;
  if ((uintptr_t)tracks % 16 != 0 || (uintptr_t)cache % 4 != 0) return FE_ERR_INVALID_ARGUMENT;
  if (n == 0) return FE_OK;
  fe::StLaunch p;
  memset(&p, 0, sizeof(p));
  p.prev = to_pyr(*prev);
  p.tracks = tracks;
  p.n = n;
  p.sampling = sampling;
  p.cache_out = cache;
  FE_CUDA(fe::launch_st(p, 2, (cudaStream_t)stream));
  return FE_OK;
}

int fe_track_affine_cached(fe_context* ctx, const fe_pyramid* cur, const fe_affine_cache* cache, int n_cache,
                           fe_track_data* tracks, int n, int n_shift_iterations, int n_full_iterations, int sampling,
                           fe_stream stream) {
  const int rc = affine_args(ctx, cur, tracks, n, n_shift_iterations, n_full_iterations, sampling);
  if (rc) return rc;
  if (n_cache < 0 || (n_cache > 0 && !cache) || (uintptr_t)cache % 4 != 0) return FE_ERR_INVALID_ARGUMENT;
  if (n == 0) return FE_OK;
  fe::StLaunch p;
  memset(&p, 0, sizeof(p));
  p.cur = to_pyr(*cur);
  p.tracks = tracks;
  p.n = n;
  p.n_shift = n_shift_iterations;
  p.n_full = n_full_iterations;
  p.sampling = sampling;
  p.cache = cache;
  p.n_cache = n_cache;
  p.counter = ctx->lk_counter + 32;
  FE_CUDA(fe::launch_st(p, 1, (cudaStream_t)stream));
  return FE_OK;
}

int fe_finish_tracks(fe_context* ctx, const fe_finish_camera* cams, int ncams, fe_stream stream) {
  if (!ctx || !cams || ncams <= 0) return FE_ERR_INVALID_ARGUMENT;
  if (ncams > fe::kMaxCams) return FE_ERR_CAPACITY;
  fe::FinishBatch fb;
  memset(&fb, 0, sizeof(fb));
  size_t ncells = 0;
  for (int i = 0; i < ncams; ++i) {
    const fe_finish_camera& c = cams[i];
    if (c.n < 0 || (c.n > 0 && (!c.tracks || !c.opts.age)) || c.width <= 0 || c.height <= 0)
      return FE_ERR_INVALID_ARGUMENT;
    if ((uintptr_t)c.tracks % 16 != 0 || (uintptr_t)c.opts.predicted % 8 != 0) return FE_ERR_INVALID_ARGUMENT;
    if (c.opts.mask && c.opts.mask_pitch_bytes < c.width) return FE_ERR_INVALID_ARGUMENT;
    if (c.opts.collapse) ncells += (size_t)((c.width + 2) / 3) * ((c.height + 2) / 3);
  }
  if (ncells > ctx->finish_cap) {
    if (ctx->finish_cells) cudaFree(ctx->finish_cells);
    ctx->finish_cells = nullptr;
    ctx->finish_cap = 0;
    FE_CUDA(dev_alloc((void**)&ctx->finish_cells, ncells * sizeof(unsigned long long)));
    FE_CUDA(cudaMemset(ctx->finish_cells, 0, ncells * sizeof(unsigned long long)));
    ctx->finish_cap = ncells;
  }
  size_t o = 0;
  for (int i = 0; i < ncams; ++i) {
    const fe_finish_camera& c = cams[i];
    fe::FinishCam& f = fb.cam[fb.ncams++];
    f.tracks = c.tracks;
    f.age = c.opts.age;
    f.n = c.n;
    f.pred = c.opts.predicted;
    f.w = c.width;
    f.h = c.height;
    for (int k = 0; k < 4; ++k) f.border[k] = c.border[k];
    f.mask = c.opts.mask;
    f.mask_pitch = c.opts.mask_pitch_bytes;
    f.alive_count = c.opts.alive_count;
    if (c.opts.collapse) {
      f.cw = (c.width + 2) / 3;
      f.ch = (c.height + 2) / 3;
      f.cells = ctx->finish_cells + o;
      o += (size_t)f.cw * f.ch;
    }
  }
  FE_CUDA(fe::launch_finish(fb, (cudaStream_t)stream));
  return FE_OK;
}

int fe_track_stereo(fe_context* ctx, const fe_stereo_pair* pairs, int npairs, float early_exit_fraction,
                    int horizontal, int sampling, fe_stream stream) {
  if (!ctx || !pairs || npairs <= 0) return FE_ERR_INVALID_ARGUMENT;
  if (npairs > fe::kMaxStereoPairs) return FE_ERR_CAPACITY;
  if (sampling < FE_SAMPLE_TEXTURE || sampling > FE_SAMPLE_TEXTURE_WIDE) return FE_ERR_INVALID_ARGUMENT;
  if (!(early_exit_fraction == early_exit_fraction)) return FE_ERR_INVALID_ARGUMENT;
  cudaStream_t s = (cudaStream_t)stream;
  // scratch layout: [counter, done, per pair: attempts, cnt[maxc]] zeroed; [per pair: stop, best[n]]
  // set to all ones; [per pair: pos[n * maxc]] uninitialised
  int64_t zero_words = 2, ones_words = 0, pos_elems = 0, round = 0;
  int rounds = 0;
  for (int q = 0; q < npairs; ++q) {
    const fe_stereo_pair& P = pairs[q];
    if (!valid_pyramid(P.primary) || !valid_pyramid(P.secondary)) return FE_ERR_INVALID_ARGUMENT;
    if (P.secondary->levels < P.primary->levels) return FE_ERR_INVALID_ARGUMENT;
    if (!horizontal)
      for (int l = 0; l < P.primary->levels; ++l)
        if (!P.primary->grad_y[l]) return FE_ERR_INVALID_ARGUMENT;
    if (P.n < 0 || (P.n > 0 && (!P.uv || !P.out))) return FE_ERR_INVALID_ARGUMENT;
    if ((uintptr_t)P.out % 16 != 0 || (uintptr_t)P.uv % 8 != 0) return FE_ERR_INVALID_ARGUMENT;
    int maxc = 0;
    if (P.cand_offsets) {
      if (P.max_candidates < 0 || (P.max_candidates > 0 && !P.cand_xy) || (uintptr_t)P.cand_xy % 8 != 0)
        return FE_ERR_INVALID_ARGUMENT;
      maxc = P.max_candidates;
    } else {
      const fe_epipolar_curves* c = P.curves;
      if (!c || c->width < 1 || c->height < 1 || !c->offsets || c->max_length < 0 || !(c->inv_scale > 0.f) ||
          (c->max_length > 0 && !c->xy) || (uintptr_t)c->xy % 8 != 0)
        return FE_ERR_INVALID_ARGUMENT;
      maxc = c->max_length;
    }
    if (P.n > 0 && maxc > (INT32_MAX / 4) / P.n) return FE_ERR_CAPACITY;
    zero_words += 1 + maxc;
    ones_words += 1 + P.n;
    pos_elems += (int64_t)P.n * maxc;
    round += P.n;
    rounds = std::max(rounds, maxc);
  }
  if (round == 0) {
    for (int q = 0; q < npairs; ++q)
      if (pairs[q].stats) FE_CUDA(cudaMemsetAsync(pairs[q].stats, 0, 4 * sizeof(int32_t), s));
    return FE_OK;
  }
  if ((int64_t)rounds * round > (int64_t)INT32_MAX - (1 << 24)) return FE_ERR_CAPACITY;
  const int64_t zero_bytes = align_up(zero_words * 4, kAlign), ones_bytes = align_up(ones_words * 4, kAlign);
  const int64_t need = zero_bytes + ones_bytes + pos_elems * 8;
  if ((size_t)need > ctx->stereo_bytes) {
    if (ctx->stereo_mem) cudaFree(ctx->stereo_mem);
    ctx->stereo_mem = nullptr;
    ctx->stereo_bytes = 0;
    FE_CUDA(dev_alloc((void**)&ctx->stereo_mem, (size_t)need));
    ctx->stereo_bytes = (size_t)need;
  }
  char* base = (char*)ctx->stereo_mem;
  int* zw = (int*)base;
  unsigned* ow = (unsigned*)(base + zero_bytes);
  float2* pw = (float2*)(base + zero_bytes + ones_bytes);
  fe::StereoLaunch L;
  memset(&L, 0, sizeof(L));
  L.npairs = npairs;
  L.round = (int)round;
  L.rounds = rounds;
  L.counter = zw;
  L.done = zw + 1;
  L.sampling = sampling;
  L.horizontal = horizontal ? 1 : 0;
  zw += 2;
  int begin = 0;
  for (int q = 0; q < npairs; ++q) {
    const fe_stereo_pair& P = pairs[q];
    fe::StereoPair& D = L.pair[q];
    D.lk.prev = to_pyr(*P.primary);
    D.lk.cur = to_pyr(*P.secondary);
    D.uv = (const float2*)P.uv;
    D.valid = P.valid;
    D.n = P.n;
    D.begin = begin;
    begin += P.n;
    if (P.cand_offsets) {
      D.maxc = P.max_candidates;
      D.cand_off = P.cand_offsets;
      D.cand_xy = (const float2*)P.cand_xy;
    } else {
      D.maxc = P.curves->max_length;
      D.cw = P.curves->width;
      D.ch = P.curves->height;
      D.inv_scale = P.curves->inv_scale;
      D.c_off = P.curves->offsets;
      D.c_xy = (const float2*)P.curves->xy;
    }
    D.radius = P.search_radius;
    D.ncc_thr = P.ncc_threshold;
    D.need = early_exit_fraction * (float)P.n;  // kL2REarlyExitFraction * n, as the reference computes it
    D.out = P.out;
    D.winner = P.winner;
    D.stats = P.stats;
    D.attempts = zw;
    D.cnt = zw + 1;
    zw += 1 + D.maxc;
    D.stop = ow;
    D.best = ow + 1;
    ow += 1 + P.n;
    D.pos = pw;
    pw += (size_t)P.n * D.maxc;
  }
  FE_CUDA(cudaMemsetAsync(base, 0, (size_t)zero_words * 4, s));
  FE_CUDA(cudaMemsetAsync(base + zero_bytes, 0xff, (size_t)ones_words * 4, s));
  FE_CUDA(fe::launch_stereo(L, s));
  return FE_OK;
}

}  // extern "C"

// ------------------------------------------------------------------ batched frame step
struct fe_batch {
  fe_context* ctx = nullptr;
  int ncams = 0;
  int sampling = FE_SAMPLE_TEXTURE;
  std::vector<fe_camera_frame> cams;
  std::vector<fe_pyramid> prev, cur;
  std::vector<char> has_prev;
  StagePlan plan;
  fe::LkCam* d_lk = nullptr;
  fe::LkTex* d_tex = nullptr;  // FE_SAMPLE_HARDWARE: texture objects per LK camera
  CUtensorMap* d_grad_tmaps = nullptr;  // selection cameras' [gx, gy] level-0 tensor maps
  int* lk_counter = nullptr;
  fe::LkLaunch lk;
  fe::SelectBatch* sel = nullptr;  // heap: large
  fe::SelectBatch* sel_burned = nullptr;  // the same cameras without touched-cell marks (placement 4)
  int sel_tiles = 0, bin_cap = 1, final_cap = 1, touched_words = 0;
  void* sel_mem = nullptr;
  size_t zero_bytes = 0;
  bool any_select = false;
  cudaStream_t cap_stream = nullptr;
  cudaStream_t side_stream = nullptr;   // second branch of the captured step
  cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  // shapes chosen by fe_batch_autotune (defaults until it runs)
  int* stage_done = nullptr;  // pyramid counters: four per camera, then the levels 0-2 launches' queues
  int lk_shape = 0;      // LK block shape (fe::kLkShapes)
  int overlap = 1;       // response tiles on a second stream beside LK
  int stage_tile = 8;    // deepest-level tile of the generic pyramid stages
  fe::FinishBatch* finish = nullptr;      // cameras with finish filters (heap), or nullptr
  unsigned long long* finish_cells = nullptr;
};

namespace {

// One frame step: the pyramids, LK (and the finish filters), the selection's response tiles (which
// do not depend on tracking), then the rest of the selection (burn of the LK survivors, burned
// cells, quotas, order).  Where the response tiles run (`overlap`):
//   0: after LK on `st` (LK reads the pyramids the pyramid launch has just left in L2);
//   1: on `side`, forked after the whole pyramid, beside LK; joined before the rest;
//   2: on `side`, forked after the levels 0-2 stage, beside the deeper pyramid stages and LK;
//   3: before LK on `st`;
//   4: after LK on `st`, after the burn of the LK survivors (alive_kernel), which the tiles then
//      apply themselves, as the single-camera selection does: no burned-cell pass, no response map.
int enqueue_batch(fe_batch* b, cudaStream_t st, cudaStream_t side, int overlap) {
  const bool fork = b->any_select && side && (overlap == 1 || overlap == 2);
  const size_t split = (fork && overlap == 2) ? 1 : b->plan.size();
  int rc = run_stages(b->plan, 0, split, st);
  if (rc) return rc;
  if (b->any_select) FE_CUDA(cudaMemsetAsync(b->sel_mem, 0, b->zero_bytes, st));
  if (fork) {
    FE_CUDA(cudaEventRecord(b->fork_ev, st));
    FE_CUDA(cudaStreamWaitEvent(side, b->fork_ev, 0));
    FE_CUDA(fe::launch_select_response(*b->sel, b->sel_tiles, side));
  }
  rc = run_stages(b->plan, split, b->plan.size(), st);
  if (rc) return rc;
  if (b->any_select && !fork && overlap == 3) FE_CUDA(fe::launch_select_response(*b->sel, b->sel_tiles, st));
  if (b->lk.total > 0) FE_CUDA(fe::launch_lk(b->lk, st));
  if (b->finish) FE_CUDA(fe::launch_finish(*b->finish, st));
  if (fork) {
    FE_CUDA(cudaEventRecord(b->join_ev, side));
    FE_CUDA(cudaStreamWaitEvent(st, b->join_ev, 0));
  } else if (b->any_select && overlap == 4) {
    FE_CUDA(fe::launch_select(*b->sel_burned, b->sel_tiles, b->bin_cap, b->final_cap, st));
    return FE_OK;
  } else if (b->any_select && overlap != 3) {
    FE_CUDA(fe::launch_select_response(*b->sel, b->sel_tiles, st));
  }
  if (b->any_select)
    FE_CUDA(fe::launch_select_rest(*b->sel, b->touched_words, b->bin_cap, b->final_cap, st));
  return FE_OK;
}

// (Re)captures the step with the batch's current shapes into its graph.
int capture_batch(fe_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
  b->lk.shape = b->lk_shape;
  cudaError_t e = cudaStreamBeginCapture(b->cap_stream, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return cuda_fail(e);
  int rc = enqueue_batch(b, b->cap_stream, b->side_stream, b->overlap);
  cudaGraph_t g = nullptr;
  e = cudaStreamEndCapture(b->cap_stream, &g);
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) return cuda_fail(e);
  b->graph = g;
  e = cudaGraphInstantiate(&b->exec, g, 0);
  return e == cudaSuccess ? FE_OK : cuda_fail(e);
}

// Re-plans the pyramid stages with the generic stages' tile `kt`.
int replan_pyramids(fe_batch* b, int kt) {
  StagePlan plan;
  int used = 0;
  for (int i = 0; i < b->ncams; ++i) {
    int rc = plan_pyramid(b->cams[i].image, b->cams[i].image_pitch_bytes, true, b->cur[i], plan, 1.f, kt,
                          b->stage_done, &used, 4 * b->ncams);
    if (rc) return rc;
  }
  int nq = 0;
  int rc = finish_l012_plan(plan, b->stage_done + 4 * b->ncams, &nq, 8);
  if (rc) return rc;
  stamp_plan(plan, b->ctx);
  b->plan = std::move(plan);
  b->stage_tile = kt;
  return FE_OK;
}

}  // namespace

extern "C" {

int fe_batch_autotune(fe_batch* b, int reps, fe_stream stream) {
  if (!b || reps <= 0) return FE_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  // the step moves the tracks: keep the originals and restore them before every timed step and at the end
  size_t bytes = 0;
  for (int i = 0; i < b->ncams; ++i)
    if (b->has_prev[i]) bytes += (size_t)b->cams[i].n_tracks * sizeof(fe_track_data);
  void* saved = nullptr;
  if (bytes) FE_CUDA(dev_alloc((void**)&saved, bytes));
  auto copy_tracks = [&](bool save) -> cudaError_t {
    size_t o = 0;
    for (int i = 0; i < b->ncams; ++i) {
      if (!b->has_prev[i] || b->cams[i].n_tracks <= 0) continue;
      const size_t n = (size_t)b->cams[i].n_tracks * sizeof(fe_track_data);
      cudaError_t e = save ? cudaMemcpyAsync((char*)saved + o, b->cams[i].tracks, n, cudaMemcpyDeviceToDevice, st)
                           : cudaMemcpyAsync(b->cams[i].tracks, (char*)saved + o, n, cudaMemcpyDeviceToDevice, st);
      if (e != cudaSuccess) return e;
      o += n;
    }
    return cudaSuccess;
  };
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = FE_OK;
  auto measure = [&](float* ms) -> int {
    int r = capture_batch(b);
    if (r) return r;
    *ms = 0.f;
    for (int k = 0; k < reps + 1; ++k) {  // the first step warms up
      cudaError_t e = copy_tracks(false);
      if (e == cudaSuccess) e = cudaEventRecord(e0, st);
      if (e == cudaSuccess) e = cudaGraphLaunch(b->exec, st);
      if (e == cudaSuccess) e = cudaEventRecord(e1, st);
      if (e == cudaSuccess) e = cudaEventSynchronize(e1);
      float t = 0.f;
      if (e == cudaSuccess) e = cudaEventElapsedTime(&t, e0, e1);
      if (e != cudaSuccess) return cuda_fail(e);
      if (k > 0) *ms += t;
    }
    return FE_OK;
  };
  cudaError_t ce = cudaEventCreate(&e0);
  if (ce == cudaSuccess) ce = cudaEventCreate(&e1);
  if (ce == cudaSuccess) ce = copy_tracks(true);
  if (ce != cudaSuccess) rc = cuda_fail(ce);
  // coordinate descent over the three shapes, each candidate timed as whole graph launches
  float best = 0.f;
  if (!rc) rc = measure(&best);
  for (int shape = 0; !rc && shape < fe::kLkShapes; ++shape) {
    if (shape == b->lk_shape) continue;
    const int keep = b->lk_shape;
    b->lk_shape = shape;
    float t = 0.f;
    rc = measure(&t);
    if (!rc && t < best) best = t;
    else b->lk_shape = keep;
  }
  for (int ov = 0; !rc && b->any_select && ov < 5; ++ov) {
    if (ov == b->overlap) continue;
    const int keep = b->overlap;
    b->overlap = ov;
    float t = 0.f;
    rc = measure(&t);
    if (!rc && t < best) best = t;
    else b->overlap = keep;
  }
  const int tiles[4] = {8, 16, 8 | fe::kL012Three, 16 | fe::kL012Three};
  for (int k = 0; !rc && k < 4; ++k) {
    if (tiles[k] == b->stage_tile) continue;
    const int keep = b->stage_tile;
    rc = replan_pyramids(b, tiles[k]);
    float t = 0.f;
    if (!rc) rc = measure(&t);
    if (!rc && t < best) best = t;
    else if (!rc) rc = replan_pyramids(b, keep);
  }
  if (!rc) rc = capture_batch(b);
  if (!rc && bytes) {
    ce = copy_tracks(false);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
    if (ce != cudaSuccess) rc = cuda_fail(ce);
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (saved) cudaFree(saved);
  return rc;
}

int fe_batch_set_tuning(fe_batch* b, int lk_shape, int overlap, int stage_tile) {
  const int tile = stage_tile & ~fe::kL012Three;
  if (!b || lk_shape < 0 || lk_shape >= fe::kLkShapes || (tile != 8 && tile != 16) || overlap < 0 || overlap > 4)
    return FE_ERR_INVALID_ARGUMENT;
  b->lk_shape = lk_shape;
  b->overlap = overlap;
  if (stage_tile != b->stage_tile) {
    int rc = replan_pyramids(b, stage_tile);
    if (rc) return rc;
  }
  return capture_batch(b);
}

int fe_batch_tuning(const fe_batch* b, int32_t* lk_shape, int32_t* overlap, int32_t* stage_tile) {
  if (!b) return FE_ERR_INVALID_ARGUMENT;
  if (lk_shape) *lk_shape = b->lk_shape;
  if (overlap) *overlap = b->overlap;
  if (stage_tile) *stage_tile = b->stage_tile;
  return FE_OK;
}

int fe_batch_create(fe_context* ctx, const fe_camera_frame* cams, int ncams, int sampling, fe_batch** out) {
  if (!ctx || !cams || !out || ncams <= 0) return FE_ERR_INVALID_ARGUMENT;
  if (ncams > fe::kMaxCams) return FE_ERR_CAPACITY;
  if (sampling < FE_SAMPLE_TEXTURE || sampling > FE_SAMPLE_HARDWARE) return FE_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  fe_batch* b = new (std::nothrow) fe_batch;
  if (!b) return FE_ERR_OUT_OF_MEMORY;
  b->ctx = ctx;
  b->ncams = ncams;
  b->sampling = sampling;
  b->cams.assign(cams, cams + ncams);
  b->prev.resize(ncams);
  b->cur.resize(ncams);
  b->has_prev.assign(ncams, 0);
  b->sel = new (std::nothrow) fe::SelectBatch;
  if (!b->sel) {
    delete b;
    return FE_ERR_OUT_OF_MEMORY;
  }
  memset(b->sel, 0, sizeof(*b->sel));
  auto fail = [&](int rc) {
    fe_batch_destroy(b);
    return rc;
  };
  // validate and copy descriptors; plan the pyramid stages
  std::vector<fe::LkCam> lk;
  std::vector<fe::LkTex> lk_tex;
  int total = 0;
  for (int i = 0; i < ncams; ++i) {
    const fe_camera_frame& c = cams[i];
    if (!c.image || !valid_pyramid(c.cur) || !c.cur->grad_y[0] || c.cur->width[0] != c.width ||
        c.cur->height[0] != c.height || c.image_pitch_bytes < c.width || c.n_tracks < 0 || c.num_desired < 0)
      return fail(FE_ERR_INVALID_ARGUMENT);
    b->cur[i] = *c.cur;
    int rc = plan_pyramid(c.image, c.image_pitch_bytes, true, b->cur[i], b->plan);
    if (rc) return fail(rc);
    if (c.prev && c.n_tracks > 0) {
      if (!valid_pyramid(c.prev) || !c.tracks || c.cur->levels < c.prev->levels || (uintptr_t)c.tracks % 16)
        return fail(FE_ERR_INVALID_ARGUMENT);
      b->prev[i] = *c.prev;
      b->has_prev[i] = 1;
      fe::LkCam lc;
      memset(&lc, 0, sizeof(lc));
      lc.prev = to_pyr(b->prev[i]);
      lc.cur = to_pyr(b->cur[i]);
      lc.tracks = c.tracks;
      lc.n = c.n_tracks;
      lc.begin = total;
      lc.retrack_ncc = c.finish ? c.finish->retrack_ncc : 0.f;
      total += c.n_tracks;
      lk.push_back(lc);
      if (sampling == FE_SAMPLE_HARDWARE) {
        fe::LkTex t;
        rc = lk_textures(ctx, b->prev[i], b->cur[i], false, t);
        if (rc) return fail(rc);
        lk_tex.push_back(t);
      }
    }
  }
  memset(&b->lk, 0, sizeof(b->lk));
  if (!lk.empty()) {
    cudaError_t e = dev_alloc((void**)&b->d_lk, sizeof(fe::LkCam) * lk.size());
    if (e != cudaSuccess) return fail(cuda_fail(e));
    e = cudaMemcpy(b->d_lk, lk.data(), sizeof(fe::LkCam) * lk.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return fail(cuda_fail(e));
    e = dev_alloc((void**)&b->lk_counter, 256);
    if (e != cudaSuccess) return fail(cuda_fail(e));
    b->lk.cams = b->d_lk;
    b->lk.counter = b->lk_counter;
    b->lk.ncams = (int)lk.size();
    b->lk.total = total;
    b->lk.horizontal = 0;
    b->lk.sampling = sampling;
    if (sampling == FE_SAMPLE_HARDWARE) {
      e = dev_alloc((void**)&b->d_tex, sizeof(fe::LkTex) * lk_tex.size());
      if (e != cudaSuccess) return fail(cuda_fail(e));
      e = cudaMemcpy(b->d_tex, lk_tex.data(), sizeof(fe::LkTex) * lk_tex.size(), cudaMemcpyHostToDevice);
      if (e != cudaSuccess) return fail(cuda_fail(e));
      b->lk.texs = b->d_tex;
    }
  }
  // finish filters (cameras with tracks and options): one CTA per camera, collapse cells zeroed once
  {
    fe::FinishBatch fb;
    memset(&fb, 0, sizeof(fb));
    size_t ncells = 0;
    for (int i = 0; i < ncams; ++i) {
      const fe_camera_frame& c = cams[i];
      if (!c.finish || !b->has_prev[i]) continue;
      if (!c.finish->age) return fail(FE_ERR_INVALID_ARGUMENT);
      fe::FinishCam& f = fb.cam[fb.ncams++];
      f.tracks = c.tracks;
      f.age = c.finish->age;
      f.n = c.n_tracks;
      f.pred = c.finish->predicted;
      f.w = c.width;
      f.h = c.height;
      for (int k = 0; k < 4; ++k) f.border[k] = c.border[k];
      f.mask = c.finish->mask;
      f.mask_pitch = c.finish->mask_pitch_bytes;
      f.alive_count = c.finish->alive_count;
      if (c.finish->collapse) {
        f.cw = (c.width + 2) / 3;
        f.ch = (c.height + 2) / 3;
        ncells += (size_t)f.cw * f.ch;
      }
    }
    if (fb.ncams > 0) {
      if (ncells) {
        cudaError_t e = dev_alloc((void**)&b->finish_cells, ncells * sizeof(unsigned long long));
        if (e == cudaSuccess) e = cudaMemset(b->finish_cells, 0, ncells * sizeof(unsigned long long));
        if (e != cudaSuccess) return fail(cuda_fail(e));
      }
      size_t o = 0;
      for (int k = 0; k < fb.ncams; ++k)
        if (fb.cam[k].cw) {
          fb.cam[k].cells = b->finish_cells + o;
          o += (size_t)fb.cam[k].cw * fb.cam[k].ch;
        }
      b->finish = new (std::nothrow) fe::FinishBatch(fb);
      if (!b->finish) return fail(FE_ERR_OUT_OF_MEMORY);
    }
  }
  // selection scratch: every camera's [stats | burn | touched] first (one memset per step), then
  // each camera's cells, sub-tile sums, quotas, kept keys and response/NMS maps
  struct BatchSel {
    size_t stats, burn, touched, zero, cell_m, cell_xy, sub_sum, bin_want, q_keys, resp, rest;
    int touched_words;
  };
  std::vector<BatchSel> lay(ncams);
  size_t zero = 0, rest = 0;
  std::vector<int> qcaps(ncams);
  for (int i = 0; i < ncams; ++i) {
    const fe_camera_frame& c = cams[i];
    if (c.num_desired <= 0) continue;
    if (!c.new_xy || !c.new_count) return fail(FE_ERR_INVALID_ARGUMENT);
    if (c.width > 4096 || c.height > 4096 || c.num_desired > 16384) return fail(FE_ERR_CAPACITY);
    int bc, fc, qc;
    const int n_alive = b->has_prev[i] ? c.n_tracks : 0;
    int rc = sel_caps(c.width, c.height, n_alive, c.num_desired, &bc, &fc, &qc);
    if (rc) return fail(rc);
    b->bin_cap = std::max(b->bin_cap, bc);
    b->final_cap = std::max(b->final_cap, fc);
    qcaps[i] = qc;
    const int w = c.width, h = c.height;
    const size_t cells = std::max<size_t>((size_t)(w / 8) * (h / 8), 1);
    const int vcells = ((w + 7) / 8) * ((h + 7) / 8);
    BatchSel& L = lay[i];
    L.touched_words = (vcells + 31) / 32;
    size_t o = 0;
    auto take = [&](size_t bytes) {
      size_t at = o;
      o = (size_t)align_up((int64_t)(o + bytes), kAlign);
      return at;
    };
    L.stats = take(16 * sizeof(int));
    L.burn = take((size_t)((w + 31) / 32) * h * 4);
    L.touched = take((size_t)L.touched_words * 4);
    L.zero = o;
    o = 0;
    L.cell_m = take(cells * 4);
    L.cell_xy = take(cells * 8);
    L.sub_sum = take((size_t)((w + 15) / 16) * ((h + 15) / 16) * 4);
    L.bin_want = take(128 * 4);
    L.q_keys = take((size_t)std::max(qc, 1) * 8);
    L.resp = take((size_t)w * h * 4);  // the response map that cells_kernel reads
    L.rest = o;
    zero += L.zero;
    rest += L.rest;
    b->any_select = true;
  }
  if (b->any_select) {
    cudaError_t e = dev_alloc((void**)&b->sel_mem, zero + rest);
    if (e != cudaSuccess) return fail(cuda_fail(e));
    b->zero_bytes = zero;
    char* zp = (char*)b->sel_mem;
    char* rp = (char*)b->sel_mem + zero;
    fe::SelectBatch& sb = *b->sel;
    sb.ncams = 0;
    sb.debug = 0;
    for (int i = 0; i < ncams; ++i) {
      const fe_camera_frame& c = cams[i];
      if (c.num_desired <= 0) continue;
      const BatchSel& L = lay[i];
      SelectScratch s;
      s.stats = (int*)(zp + L.stats);
      s.burn = (uint32_t*)(zp + L.burn);
      uint32_t* touched = (uint32_t*)(zp + L.touched);
      zp += L.zero;
      s.cell_m = (float*)(rp + L.cell_m);
      s.cell_xy = (float2*)(rp + L.cell_xy);
      s.sub_sum = (float*)(rp + L.sub_sum);
      s.bin_want = (int*)(rp + L.bin_want);
      s.q_keys = (uint64_t*)(rp + L.q_keys);
      s.resp = (float*)(rp + L.resp);
      s.nms = nullptr;
      rp += L.rest;
      fe::SelectCam& sc = sb.cam[sb.ncams++];
      fill_select_cam(sc, s, b->cur[i], qcaps[i]);
      sc.touched = touched;
      sc.touched_begin = b->touched_words;
      b->touched_words += L.touched_words;
      sc.alive_tracks = b->has_prev[i] ? c.tracks : nullptr;
      sc.n_alive = b->has_prev[i] ? c.n_tracks : 0;
      sc.num_desired = c.num_desired;
      sc.target_total = c.num_desired;
      for (int k = 0; k < 4; ++k) sc.border[k] = c.border[k];
      sc.out_xy = c.new_xy;
      sc.out_count = c.new_count;
      sc.tile_begin = b->sel_tiles;
      b->sel_tiles += sc.tiles_x * sc.tiles_y;
    }
    // the response tiles of cameras whose level-0 gradient planes meet TMA alignment stage their
    // interior windows by TMA (the others with asynchronous 16-byte copies)
    sb.status = ctx->dev_status;
    sb.wait_limit = ctx->wait_limit;
    if (sb.ncams > 0) {
      std::vector<CUtensorMap> maps((size_t)2 * sb.ncams);
      std::vector<char> ok(sb.ncams, 0);
      bool any = false;
      for (int k = 0; k < sb.ncams; ++k) {
        const fe::SelectCam& sc = sb.cam[k];
        ok[k] = fe::encode_select_grad_tmaps(&maps[2 * k], sc.gx, sc.gy, sc.w, sc.h, sc.pitch) ? 1 : 0;
        any = any || ok[k];
      }
      if (any) {
        cudaError_t e = dev_alloc((void**)&b->d_grad_tmaps, sizeof(CUtensorMap) * maps.size());
        if (e == cudaSuccess)
          e = cudaMemcpy(b->d_grad_tmaps, maps.data(), sizeof(CUtensorMap) * maps.size(), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return fail(cuda_fail(e));
        for (int k = 0; k < sb.ncams; ++k)
          if (ok[k]) sb.cam[k].grad_tmap = b->d_grad_tmaps + 2 * k;
      }
    }
    b->sel_burned = new (std::nothrow) fe::SelectBatch;
    if (!b->sel_burned) return fail(FE_ERR_OUT_OF_MEMORY);
    *b->sel_burned = sb;
    for (int k = 0; k < sb.ncams; ++k) b->sel_burned->cam[k].touched = nullptr;
  }
  // capture the step into a graph
  cudaError_t e = cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->side_stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->fork_ev, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->join_ev, cudaEventDisableTiming);
  if (e != cudaSuccess) return fail(cuda_fail(e));
  // pyramid stages with tails: the deep levels' counters, then the final plan
  e = dev_alloc((void**)&b->stage_done, sizeof(int) * (4 * ncams + 8));
  if (e == cudaSuccess) e = cudaMemset(b->stage_done, 0, sizeof(int) * (4 * ncams + 8));
  if (e != cudaSuccess) return fail(cuda_fail(e));
  int rc = replan_pyramids(b, b->stage_tile);
  if (!rc) rc = capture_batch(b);
  if (rc) return fail(rc);
  *out = b;
  return FE_OK;
}

int fe_batch_run(fe_batch* b, fe_stream stream) {
  if (!b || !b->exec) return FE_ERR_INVALID_ARGUMENT;
  FE_CUDA(cudaGraphLaunch(b->exec, (cudaStream_t)stream));
  return FE_OK;
}

int fe_batch_run_part(fe_batch* b, int part, fe_stream stream) {
  if (!b) return FE_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  switch (part) {
    case FE_PART_PYRAMID:
      return run_plan(b->plan, st);
    case FE_PART_TRACK:
      if (b->lk.total > 0) FE_CUDA(fe::launch_lk(b->lk, st));
      return FE_OK;
    case FE_PART_SELECT:
      if (b->any_select) {
        FE_CUDA(cudaMemsetAsync(b->sel_mem, 0, b->zero_bytes, st));
        if (b->overlap == 4) {  // as the step runs it: burn, then tiles that apply it
          FE_CUDA(fe::launch_select(*b->sel_burned, b->sel_tiles, b->bin_cap, b->final_cap, st));
        } else {
          FE_CUDA(fe::launch_select_response(*b->sel, b->sel_tiles, st));
          FE_CUDA(fe::launch_select_rest(*b->sel, b->touched_words, b->bin_cap, b->final_cap, st));
        }
      }
      return FE_OK;
    default:
      return FE_ERR_INVALID_ARGUMENT;
  }
}

int fe_batch_lk_work(fe_batch* b, uint64_t* device_counts, fe_stream stream) {
  if (!b || !device_counts) return FE_ERR_INVALID_ARGUMENT;
  if (b->lk.total <= 0) return FE_OK;
  fe::LkLaunch counted = b->lk;
  counted.counts = reinterpret_cast<unsigned long long*>(device_counts);
  FE_CUDA(fe::launch_lk(counted, (cudaStream_t)stream));
  return FE_OK;
}

int fe_batch_kernel_count(fe_batch* b) {
  if (!b || !b->graph) return -1;
  size_t n = 0;
  if (cudaGraphGetNodes(b->graph, nullptr, &n) != cudaSuccess) return -1;
  std::vector<cudaGraphNode_t> nodes(n);
  if (n && cudaGraphGetNodes(b->graph, nodes.data(), &n) != cudaSuccess) return -1;
  int k = 0;
  for (auto nd : nodes) {
    cudaGraphNodeType t;
    if (cudaGraphNodeGetType(nd, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ++k;
  }
  return k;
}

int fe_batch_run_plain(fe_batch* b, fe_stream stream) {
  if (!b) return FE_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  fe_context* ctx = b->ctx;
  for (int i = 0; i < b->ncams; ++i) {
    const fe_camera_frame& c = b->cams[i];
    int rc = fe_build_pyramid(ctx, c.image, c.image_pitch_bytes, c.width, c.height, 0, &b->cur[i], stream);
    if (rc) return rc;
    if (b->has_prev[i]) {
      if (c.finish) {
        rc = fe_track_mono(ctx, &b->prev[i], &b->cur[i], c.tracks, c.n_tracks, c.finish->retrack_ncc, b->sampling,
                           stream);
        if (rc) return rc;
        fe_finish_camera fc;
        memset(&fc, 0, sizeof(fc));
        fc.tracks = c.tracks;
        fc.n = c.n_tracks;
        fc.width = c.width;
        fc.height = c.height;
        for (int k = 0; k < 4; ++k) fc.border[k] = c.border[k];
        fc.opts = *c.finish;
        rc = fe_finish_tracks(ctx, &fc, 1, stream);
      } else {
        rc = fe_track(ctx, &b->prev[i], &b->cur[i], c.tracks, c.n_tracks, 0, b->sampling, stream);
      }
      if (rc) return rc;
    }
    if (c.num_desired > 0) {
      // same selection as the batch, one camera at a time on the context's scratch
      int bc, fc, qc;
      const int n_alive = b->has_prev[i] ? c.n_tracks : 0;
      rc = sel_caps(c.width, c.height, n_alive, c.num_desired, &bc, &fc, &qc);
      if (rc) return rc;
      rc = ensure_select_scratch(ctx, c.width, c.height, 0, qc);
      if (rc) return rc;
      SelectScratch& s = ctx->sel;
      FE_CUDA(cudaMemsetAsync(s.mem, 0, s.zero_bytes, st));
      static thread_local fe::SelectBatch sb;
      memset(&sb, 0, sizeof(sb));
      sb.ncams = 1;
      fe::SelectCam& sc = sb.cam[0];
      fill_select_cam(sc, s, b->cur[i], qc);
      sc.alive_tracks = b->has_prev[i] ? c.tracks : nullptr;
      sc.n_alive = n_alive;
      sc.num_desired = c.num_desired;
      sc.target_total = c.num_desired;
      for (int k = 0; k < 4; ++k) sc.border[k] = c.border[k];
      sc.out_xy = c.new_xy;
      sc.out_count = c.new_count;
      FE_CUDA(fe::launch_select(sb, sc.tiles_x * sc.tiles_y, bc, fc, st));
    }
  }
  return FE_OK;
}

int fe_batch_destroy(fe_batch* b) {
  if (!b) return FE_ERR_INVALID_ARGUMENT;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->cap_stream) cudaStreamDestroy(b->cap_stream);
  if (b->side_stream) cudaStreamDestroy(b->side_stream);
  if (b->d_grad_tmaps) cudaFree(b->d_grad_tmaps);
  if (b->fork_ev) cudaEventDestroy(b->fork_ev);
  if (b->join_ev) cudaEventDestroy(b->join_ev);
  if (b->d_lk) cudaFree(b->d_lk);
  if (b->lk_counter) cudaFree(b->lk_counter);
  if (b->d_tex) cudaFree(b->d_tex);
  if (b->sel_mem) cudaFree(b->sel_mem);
  if (b->stage_done) cudaFree(b->stage_done);
  if (b->finish_cells) cudaFree(b->finish_cells);
  delete b->finish;
  delete b->sel;
  delete b->sel_burned;
  delete b;
  return FE_OK;
}

}  // extern "C"

// ------------------------------------------------------------------ differentiable LK + adjoint
struct fe_adjoint {
  fe_context* ctx = nullptr;
  int mode = FE_ADJOINT_IMPLICIT, iters = 0;
  int L = 1, total = 0, nplanes = 0, total_tiles = 0;
  fe::LkLaunch lk;
  fe::LkLaunch lk_replay;            // unrolled backward before any forward: records into scratch tracks
  fe::AdjLaunch adj;
  fe::AdjGather gat;
  std::vector<fe::AdjPyrLevel> pyr;  // [level]
  StagePlan build;                   // pyramid builds of the jobs that name their frames
  bool forward_ran = false;          // the unrolled backward can use the forward's records
  fe::lk::LkRecord* recs = nullptr;
  void* mem = nullptr;               // every device buffer of the plan
  int* counters = nullptr;           // [0] forward track counter, [1] adjoint counter, [2] dropped
};

namespace {

constexpr int kAdjMaxTracks = 16384;  // per camera: the gather's shared-memory sort capacity

}  // namespace

extern "C" {

int fe_adjoint_destroy(fe_adjoint* a) {
  if (!a) return FE_ERR_INVALID_ARGUMENT;
  if (a->mem) cudaFree(a->mem);
  delete a;
  return FE_OK;
}

int fe_adjoint_create(fe_context* ctx, const fe_adjoint_job* jobs, int njobs, int mode, int iterations,
                      float tolerance, fe_adjoint** out) {
  if (!out) return FE_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (!ctx || !jobs || njobs <= 0 || njobs > fe::kMaxCams) return FE_ERR_INVALID_ARGUMENT;
  if (mode != FE_ADJOINT_IMPLICIT && mode != FE_ADJOINT_UNROLLED) return FE_ERR_INVALID_ARGUMENT;
  if (mode == FE_ADJOINT_UNROLLED && (iterations < 1 || iterations > fe::lk_max_unrolled())) return FE_ERR_INVALID_ARGUMENT;
  if (mode == FE_ADJOINT_IMPLICIT && (iterations < 0 || !(tolerance >= 0.f))) return FE_ERR_INVALID_ARGUMENT;
  int L = 1, total = 0;
  for (int j = 0; j < njobs; ++j) {
    const fe_adjoint_job& J = jobs[j];
    if (!valid_pyramid(J.prev) || !valid_pyramid(J.cur) || J.prev->levels != J.cur->levels) return FE_ERR_INVALID_ARGUMENT;
    for (int l = 0; l < J.prev->levels; ++l)
      if (!J.prev->grad_y[l] || J.prev->width[l] != J.cur->width[l] || J.prev->height[l] != J.cur->height[l])
        return FE_ERR_INVALID_ARGUMENT;
    if (J.n_tracks < 0) return FE_ERR_INVALID_ARGUMENT;
    if (J.n_tracks > kAdjMaxTracks) return FE_ERR_CAPACITY;
    if (J.n_tracks > 0 && (!J.tracks_in || !J.tracks_out || !J.grad_xy)) return FE_ERR_INVALID_ARGUMENT;
    if ((uintptr_t)J.tracks_in % 16 || (uintptr_t)J.tracks_out % 16 || (uintptr_t)J.grad_xy % 8) return FE_ERR_INVALID_ARGUMENT;
    if ((uintptr_t)J.grad_track % 8 || (uintptr_t)J.grad_offset % 8) return FE_ERR_INVALID_ARGUMENT;
    const int w = J.prev->width[0], h = J.prev->height[0];
    if (!J.grad_prev || !J.grad_cur || J.grad_prev_pitch_bytes < (int64_t)w * 4 || J.grad_cur_pitch_bytes < (int64_t)w * 4 ||
        J.grad_prev_pitch_bytes % 4 || J.grad_cur_pitch_bytes % 4 || (uintptr_t)J.grad_prev % 4 || (uintptr_t)J.grad_cur % 4)
      return FE_ERR_INVALID_ARGUMENT;
    (void)h;
    if ((J.prev_image || J.cur_image) &&
        (!J.prev_image || !J.cur_image || J.image_pitch_bytes < (int64_t)w * 4 || J.image_pitch_bytes % 4 ||
         !(J.image_scale > 0.f)))
      return FE_ERR_INVALID_ARGUMENT;
    if (mode == FE_ADJOINT_UNROLLED) L = std::max(L, J.prev->levels);
    total += J.n_tracks;
  }
  fe_adjoint* a = new (std::nothrow) fe_adjoint;
  if (!a) return FE_ERR_OUT_OF_MEMORY;
  auto fail = [&](int rc) {
    fe_adjoint_destroy(a);
    return rc;
  };
  a->ctx = ctx;
  a->mode = mode;
  a->iters = iterations;
  a->L = L;
  a->total = total;
  const int cur_s = mode == FE_ADJOINT_UNROLLED ? 32 : 12;

  // planes: (camera, q, level); level-0 image planes are the caller's gradient buffers
  struct PlaneSpec {
    int w, h, pitch;
    float* user;        // caller's buffer, or null: scratch at `off`
    size_t off;
  };
  std::vector<PlaneSpec> spec((size_t)njobs * 4 * L);
  std::vector<fe::AdjPlane> planes(spec.size());
  size_t scratch = 0;
  int tiles = 0;
  for (int j = 0; j < njobs; ++j)
    for (int q = 0; q < 4; ++q)
      for (int l = 0; l < L; ++l) {
        const size_t k = ((size_t)j * 4 + q) * L + l;
        PlaneSpec& s = spec[k];
        fe::AdjPlane& P = planes[k];
        memset(&P, 0, sizeof(P));
        s = PlaneSpec{0, 0, 0, nullptr, 0};
        P.tile_begin = tiles;
        if (l >= jobs[j].prev->levels) continue;
        s.w = jobs[j].prev->width[l];
        s.h = jobs[j].prev->height[l];
        if (l == 0 && q == 0) {
          s.user = jobs[j].grad_prev;
          s.pitch = (int)(jobs[j].grad_prev_pitch_bytes / 4);
        } else if (l == 0 && q == 3) {
          s.user = jobs[j].grad_cur;
          s.pitch = (int)(jobs[j].grad_cur_pitch_bytes / 4);
        } else {
          s.pitch = (int)(align_up((int64_t)s.w * 4, kAlign) / 4);
          s.off = scratch;
          scratch += (size_t)s.pitch * s.h * 4;
        }
        P.w = s.w;
        P.h = s.h;
        P.pitch = s.pitch;
        P.tiles_x = (s.w + 31) / 32;
        P.ntiles = P.tiles_x * ((s.h + 31) / 32);
        tiles += P.ntiles;
      }
  a->nplanes = (int)planes.size();
  a->total_tiles = tiles;

  // one allocation: scratch planes, records, tile lists, descriptors, counters
  const size_t nslots = (size_t)4 * L * total;
  size_t o = 0;
  auto take = [&](size_t bytes) {
    const size_t at = o;
    o = (size_t)align_up((int64_t)(o + bytes), kAlign);
    return at;
  };
  const size_t o_planes = take(scratch);
  const size_t o_hdr = take(std::max<size_t>(nslots, 1) * sizeof(int4));
  const size_t o_dprev = take(std::max<size_t>((size_t)3 * L * total * 144 * 4, 4));
  const size_t o_dcur = take(std::max<size_t>((size_t)L * total * cur_s * cur_s * 4, 4));
  const size_t o_count = take(((size_t)tiles + 1) * 4);
  const size_t o_off = take(((size_t)tiles + 1) * 4);
  const size_t o_cursor = take(((size_t)tiles + 1) * 4);
  const size_t o_long = take(((size_t)tiles + 2) * 4);
  const size_t o_list = take(std::max<size_t>(nslots * 4, 1) * 4);  // a record covers <= 4 tiles
  const size_t o_pl = take(planes.size() * sizeof(fe::AdjPlane));
  const size_t o_cams = take((size_t)njobs * sizeof(fe::AdjCam));
  const size_t o_lk = take((size_t)njobs * sizeof(fe::LkCam));
  const size_t o_lk2 = take(mode == FE_ADJOINT_UNROLLED ? (size_t)njobs * sizeof(fe::LkCam) : 0);
  const size_t o_rtr = take(mode == FE_ADJOINT_UNROLLED ? (size_t)std::max(total, 1) * sizeof(fe_track_data) : 0);
  const size_t o_recs = take(mode == FE_ADJOINT_UNROLLED ? std::max(total, 1) * fe::lk_record_bytes() : 0);
  const size_t o_done = take(sizeof(int) * 2 * njobs);
  const size_t o_ctr = take(256);
  cudaError_t e = dev_alloc((void**)&a->mem, o);
  if (e != cudaSuccess) return fail(cuda_fail(e));
  char* base = (char*)a->mem;
  a->counters = (int*)(base + o_ctr);
  for (size_t k = 0; k < planes.size(); ++k)
    if (planes[k].ntiles > 0) planes[k].dst = spec[k].user ? spec[k].user : (float*)(base + o_planes + spec[k].off);

  std::vector<fe::AdjCam> cams(njobs);
  std::vector<fe::LkCam> lks(njobs);
  int begin = 0, max_n = 1;
  for (int j = 0; j < njobs; ++j) {
    const fe_adjoint_job& J = jobs[j];
    fe::LkCam& lc = lks[j];
    memset(&lc, 0, sizeof(lc));
    lc.prev = to_pyr(*J.prev);
    lc.cur = to_pyr(*J.cur);
    lc.tracks = J.tracks_out;
    lc.tracks_in = J.tracks_in;
    lc.n = J.n_tracks;
    lc.begin = begin;
    fe::AdjCam& ac = cams[j];
    memset(&ac, 0, sizeof(ac));
    ac.lk = lc;
    ac.tracks_out = J.tracks_out;
    ac.grad_xy = J.grad_xy;
    ac.grad_track = J.grad_track;
    ac.grad_offset = J.grad_offset;
    begin += J.n_tracks;
    max_n = std::max(max_n, J.n_tracks);
  }
  e = cudaMemcpy(base + o_pl, planes.data(), planes.size() * sizeof(fe::AdjPlane), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(base + o_cams, cams.data(), cams.size() * sizeof(fe::AdjCam), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(base + o_lk, lks.data(), lks.size() * sizeof(fe::LkCam), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && mode == FE_ADJOINT_UNROLLED) {
    std::vector<fe::LkCam> rl = lks;
    for (auto& c : rl) c.tracks = (fe_track_data*)(base + o_rtr) + c.begin;
    e = cudaMemcpy(base + o_lk2, rl.data(), rl.size() * sizeof(fe::LkCam), cudaMemcpyHostToDevice);
  }
  if (e != cudaSuccess) return fail(cuda_fail(e));

  memset(&a->lk, 0, sizeof(a->lk));
  a->lk.cams = (const fe::LkCam*)(base + o_lk);
  a->lk.counter = a->counters;
  a->lk.ncams = njobs;
  a->lk.total = total;
  a->lk.sampling = FE_SAMPLE_EXACT;
  a->lk.mode = mode == FE_ADJOINT_UNROLLED ? fe::kLkUnrolled : fe::kLkImplicit;
  a->lk.iters = iterations;
  a->lk.tol2 = tolerance * tolerance;
  a->lk_replay = a->lk;
  if (mode == FE_ADJOINT_UNROLLED) {
    a->recs = (fe::lk::LkRecord*)(base + o_recs);
    a->lk.recs = a->recs;
    a->lk_replay.cams = (const fe::LkCam*)(base + o_lk2);
    a->lk_replay.recs = a->recs;
  }
  e = cudaMemset(base + o_done, 0, sizeof(int) * 2 * njobs);
  if (e != cudaSuccess) return fail(cuda_fail(e));
  int used = 0;
  for (int j = 0; j < njobs; ++j) {
    const fe_adjoint_job& J = jobs[j];
    if (!J.prev_image) continue;
    int* done = (int*)(base + o_done);
    int rc = plan_pyramid(J.prev_image, J.image_pitch_bytes, false, *J.prev, a->build, J.image_scale, 8, done, &used,
                          2 * njobs);
    if (!rc)
      rc = plan_pyramid(J.cur_image, J.image_pitch_bytes, false, *J.cur, a->build, J.image_scale, 8, done, &used,
                        2 * njobs);
    if (rc) return fail(rc);
  }
  stamp_plan(a->build, ctx);

  memset(&a->adj, 0, sizeof(a->adj));
  a->adj.cams = (const fe::AdjCam*)(base + o_cams);
  a->adj.ncams = njobs;
  a->adj.total = total;
  a->adj.counter = a->counters + 1;
  a->adj.mode = a->lk.mode;
  a->adj.iters = iterations;
  a->adj.L = L;
  a->adj.cur_s = cur_s;
  a->adj.hdr = (int4*)(base + o_hdr);
  a->adj.data_prev = (float*)(base + o_dprev);
  a->adj.data_cur = (float*)(base + o_dcur);
  a->adj.overflow = a->counters + 2;

  memset(&a->gat, 0, sizeof(a->gat));
  a->gat.planes = (const fe::AdjPlane*)(base + o_pl);
  a->gat.cams = a->adj.cams;
  a->gat.nplanes = a->nplanes;
  a->gat.ncams = njobs;
  a->gat.total_tiles = tiles;
  a->gat.nslots = (int)nslots;
  a->gat.L = L;
  a->gat.total = total;
  a->gat.cur_s = cur_s;
  a->gat.hdr = a->adj.hdr;
  a->gat.data_prev = a->adj.data_prev;
  a->gat.data_cur = a->adj.data_cur;
  a->gat.count = (int*)(base + o_count);
  a->gat.off = (int*)(base + o_off);
  a->gat.cursor = (int*)(base + o_cursor);
  a->gat.long_count = (int*)(base + o_long);
  a->gat.long_tiles = (int*)(base + o_long) + 1;
  a->gat.list = (int*)(base + o_list);
  a->gat.list_cap = next_pow2(max_n);

  // pyramid adjoint, one launch per level (top level first)
  a->pyr.resize(L);
  for (int l = 0; l < L; ++l) {
    fe::AdjPyrLevel& lv = a->pyr[l];
    memset(&lv, 0, sizeof(lv));
    int px = 0;
    for (int j = 0; j < njobs; ++j) {
      if (l >= jobs[j].prev->levels) continue;
      for (int side = 0; side < 2; ++side) {
        const int q = side ? 3 : 0;
        const fe::AdjPlane& P = planes[((size_t)j * 4 + q) * L + l];
        fe::AdjPyrJob& J = lv.job[lv.njobs++];
        memset(&J, 0, sizeof(J));
        J.img = P.dst;
        J.pitch = P.pitch;
        J.w = P.w;
        J.h = P.h;
        if (!side) {
          J.gx = planes[((size_t)j * 4 + 1) * L + l].dst;
          J.gy = planes[((size_t)j * 4 + 2) * L + l].dst;
          J.gpitch = planes[((size_t)j * 4 + 1) * L + l].pitch;
        }
        if (l + 1 < L && l + 1 < jobs[j].prev->levels) {
          const fe::AdjPlane& U = planes[((size_t)j * 4 + q) * L + l + 1];
          J.up = U.dst;
          J.up_pitch = U.pitch;
          J.up_w = U.w;
          J.up_h = U.h;
        }
        J.px_begin = px;
        px += P.w * P.h;
        lv.max_blocks = std::max(lv.max_blocks, ((P.w + 127) / 128) * ((P.h + 7) / 8));
      }
    }
    lv.total_px = px;
  }
  *out = a;
  return FE_OK;
}

int fe_adjoint_build_pyramids(fe_adjoint* a, fe_stream stream) {
  if (!a) return FE_ERR_INVALID_ARGUMENT;
  return run_plan(a->build, (cudaStream_t)stream);
}

int fe_adjoint_forward(fe_adjoint* a, fe_stream stream) {
  if (!a) return FE_ERR_INVALID_ARGUMENT;
  FE_CUDA(fe::launch_lk(a->lk, (cudaStream_t)stream));
  a->forward_ran = true;
  return FE_OK;
}

int fe_adjoint_backward(fe_adjoint* a, fe_stream stream) {
  if (!a) return FE_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  a->adj.recs = a->recs;
  // the unrolled adjoint replays the recorded steps: without a forward of this plan, record them now
  // (the tracks of this replay go to scratch)
  if (a->mode == FE_ADJOINT_UNROLLED && !a->forward_ran) FE_CUDA(fe::launch_lk(a->lk_replay, st));
  FE_CUDA(cudaMemsetAsync(a->adj.overflow, 0, sizeof(int), st));
  FE_CUDA(fe::launch_lk_adjoint(a->adj, st));
  FE_CUDA(fe::launch_adjoint_gather(a->gat, st));
  for (int l = a->L - 1; l >= 0; --l) FE_CUDA(fe::launch_pyramid_adjoint(a->pyr[l], st));
  return FE_OK;
}

int fe_adjoint_kernel_count(const fe_adjoint* a, int backward) {
  if (!a) return -1;
  if (backward == 2) {  // pyramid builds
    int n = 0;
    for (const auto& stage : a->build) n += (int)stage.size();
    return n;
  }
  if (!backward) return a->total > 0 ? 1 : 0;
  int n = a->total > 0 ? 1 : 0;              // adjoint
  if (a->total > 0 && a->mode == FE_ADJOINT_UNROLLED && !a->forward_ran) ++n;  // the replayed forward
  if (a->total_tiles > 0) n += a->gat.nslots > 0 ? 5 : 3;  // count, scan, fill, short and long gathers
  for (int l = 0; l < a->L; ++l) n += a->pyr[l].total_px > 0 ? 1 : 0;
  return n;
}

int fe_adjoint_dropped(const fe_adjoint* a, int32_t* device_out, fe_stream stream) {
  if (!a || !device_out) return FE_ERR_INVALID_ARGUMENT;
  FE_CUDA(cudaMemcpyAsync(device_out, a->adj.overflow, sizeof(int32_t), cudaMemcpyDeviceToDevice,
                          (cudaStream_t)stream));
  return FE_OK;
}

int fe_track_diff(fe_context* ctx, const fe_pyramid* prev, const fe_pyramid* cur, const fe_track_data* tracks_in,
                  fe_track_data* tracks_out, int n, int mode, int iterations, float tolerance, fe_stream stream) {
  if (!prev) return FE_ERR_INVALID_ARGUMENT;
  // the plan wants gradient outputs; the forward never touches them
  fe_adjoint_job J;
  memset(&J, 0, sizeof(J));
  J.prev = prev;
  J.cur = cur;
  J.tracks_in = tracks_in;
  J.tracks_out = tracks_out;
  J.n_tracks = n;
  J.grad_xy = reinterpret_cast<const float*>(tracks_out);
  J.grad_prev = J.grad_cur = reinterpret_cast<float*>(tracks_out);
  J.grad_prev_pitch_bytes = J.grad_cur_pitch_bytes = (int64_t)prev->width[0] * 4;
  if (n == 0) return FE_OK;
  fe_adjoint* a = nullptr;
  int rc = fe_adjoint_create(ctx, &J, 1, mode, iterations, tolerance, &a);
  if (rc) return rc;
  rc = fe_adjoint_forward(a, stream);
  cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
  fe_adjoint_destroy(a);
  if (rc) return rc;
  return e == cudaSuccess ? FE_OK : cuda_fail(e);
}

int fe_track_backward(fe_context* ctx, const fe_pyramid* prev, const fe_pyramid* cur, const fe_track_data* tracks_in,
                      const fe_track_data* tracks_out, int n, int mode, int iterations, float tolerance,
                      const float* grad_xy, float* grad_prev, int64_t grad_prev_pitch_bytes, float* grad_cur,
                      int64_t grad_cur_pitch_bytes, float* grad_track, float* grad_offset, fe_stream stream) {
  fe_adjoint_job J;
  memset(&J, 0, sizeof(J));
  J.prev = prev;
  J.cur = cur;
  J.tracks_in = tracks_in;
  J.tracks_out = const_cast<fe_track_data*>(tracks_out);
  J.n_tracks = n;
  J.grad_xy = grad_xy;
  J.grad_prev = grad_prev;
  J.grad_prev_pitch_bytes = grad_prev_pitch_bytes;
  J.grad_cur = grad_cur;
  J.grad_cur_pitch_bytes = grad_cur_pitch_bytes;
  J.grad_track = grad_track;
  J.grad_offset = grad_offset;
  fe_adjoint* a = nullptr;
  int rc = fe_adjoint_create(ctx, &J, 1, mode, iterations, tolerance, &a);
  if (rc) return rc;
  rc = fe_adjoint_backward(a, stream);
  cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
  fe_adjoint_destroy(a);
  if (rc) return rc;
  return e == cudaSuccess ? FE_OK : cuda_fail(e);
}

}  // extern "C"
