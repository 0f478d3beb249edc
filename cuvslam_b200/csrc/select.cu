// Shi-Tomasi response, non-maximum suppression and deterministic feature selection.
//
// Launch sequence (all on one stream, every step over all cameras of a batch):
//   alive_kernel   : compacts alive features (explicit list, or tracks that LK kept) in order,
//                    burns their 9x9 neighbourhoods into a bit mask, marks the cells they reach and
//                    counts them per bin.
//   tile_kernel    : one CTA per 64x32 tile: structure tensor (separable 7-tap Gaussian), the
//                    response log(1 + lambda_min), 3x3 NMS, one candidate per 8x8 cell with
//                    sub-pixel refinement, and the 16x16 sub-tile strength sums.  Single camera:
//                    after alive_kernel, with the burn applied.  Batched: before the burn, so it
//                    does not depend on tracking and runs concurrently with LK; cells_kernel then
//                    redoes the cells that alive features burned into.
//   quota_kernel   : per camera: 64 bin sums in a fixed order, the strength total, per-bin quotas.
//   bin_kernel     : per (bin, camera): filter the bin's candidates (borders, mask) and keep the
//                    best `quota` of them (a radix select of the quota-th key; final_kernel orders).
//   final_kernel   : per camera: sort the kept candidates and emit the first num_desired.
//
// Parity with GPUSelection::computeGFTTAndSelectFeatures (selection_v2.cpp:27-184):
//   response      gftt_values_kernel (gftt.cu:80-162), same FMA order, __logf as the reference;
//   NMS           non_max_suppression_kernel (selection_v2.cu:189-244), clamped neighbours, <=;
//   burn          filter_maximums_kernel (selection_v2.cu:251-277), first min(n_alive, cells)
//                 alive features, __float2int_rn centres;
//   cells         downsample_gftt_x8_kernel (selection_v2.cu:107-178), identical lane order and
//                 strict-> tie rule; select_features_kernel (:307-329) threshold 1e-2 and
//                 FindMinimum1D (:279-293) with __fdividef;
//   quotas/filter host loop of selection_v2.cpp:108-183.
// Where the reference is nondeterministic a total order is fixed: keypoints are ordered by
// strength descending then cell raster index (the reference's CUB sort sees them in atomicAdd
// order), and each bin sum adds its sub-tile rows left to right, then the row sums top to bottom
// (the reference adds sub-tiles with float atomicAdd).
#include <cuda_runtime.h>

#include "fe_common.cuh"
#include "fe_internal.h"

namespace fe {

namespace {

__device__ __forceinline__ uint64_t make_key(float m, int cell) {
  // strength descending, then cell ascending; m > 0 so its bits order like the value
  return ((uint64_t)(~__float_as_uint(m)) << 32) | (uint32_t)cell;
}

// ---------------------------------------------------------------- alive features
__global__ void alive_kernel(const __grid_constant__ SelectBatch b) {
  const SelectCam& c = b.cam[blockIdx.x];
  __shared__ int warp_counts[32];
  __shared__ int base;
  __shared__ int bin_cnt[64];
  if (threadIdx.x < 64) bin_cnt[threadIdx.x] = 0;
  if (threadIdx.x == 0) base = 0;
  __syncthreads();
  const int ncell = (c.w / 8) * (c.h / 8);
  const int bw = c.w / 8, bh = c.h / 8;
  const int words = (c.w + 31) / 32;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int n = c.n_alive;
  for (int start = 0; start < n; start += blockDim.x) {
    const int i = start + threadIdx.x;
    bool alive = false;
    float x = 0.f, y = 0.f;
    if (i < n) {
      if (c.alive_tracks) {
        const fe_track_data& t = c.alive_tracks[i];
        alive = t.track_status != 0;
        x = t.track[0];
        y = t.track[1];
      } else {
        alive = true;
        x = c.alive_xy[2 * i];
        y = c.alive_xy[2 * i + 1];
      }
    }
    // rank of this alive feature among alive features (in input order)
    const unsigned bal = __ballot_sync(0xffffffffu, alive);
    if (lane == 0) warp_counts[wid] = __popc(bal);
    __syncthreads();
    int before = base;
    for (int k = 0; k < wid; ++k) before += warp_counts[k];
    const int rank = before + __popc(bal & ((1u << lane) - 1u));
    if (alive) {
      if (c.alive_out_xy) {
        c.alive_out_xy[2 * rank] = x;
        c.alive_out_xy[2 * rank + 1] = y;
      }
      // per-bin count of alive features (all of them)
      if (bw > 0 && bh > 0) {
        const unsigned bx = (unsigned)__fdiv_rn(x, (float)bw), by = (unsigned)__fdiv_rn(y, (float)bh);
        if (bx < 8 && by < 8) atomicAdd(&bin_cnt[by * 8 + bx], 1);
      }
      // burn the 9x9 window of the first `ncell` alive features
      if (rank < ncell) {
        const int cx = __float2int_rn(x), cy = __float2int_rn(y);
        const int x0 = max(cx - 4, 0), x1 = min(cx + 4, c.w - 1);
        if (c.touched) {  // batched path: mark the cells this window reaches
          const int vcw = (c.w + 7) / 8;
          const int y0 = max(cy - 4, 0), y1 = min(cy + 4, c.h - 1);
          if (x0 <= x1 && y0 <= y1)
            for (int ty = y0 / 8; ty <= y1 / 8; ++ty)
              for (int tx = x0 / 8; tx <= x1 / 8; ++tx) {
                const int vcell = ty * vcw + tx;
                atomicOr(&c.touched[vcell >> 5], 1u << (vcell & 31));
              }
        }
        for (int yy = max(cy - 4, 0); yy <= min(cy + 4, c.h - 1); ++yy) {
          for (int xx = x0; xx <= x1;) {
            const int wd = xx >> 5;
            const int hi = min(x1, wd * 32 + 31);
            const int nb = hi - xx + 1;
            const uint32_t bits = (nb == 32 ? 0xffffffffu : ((1u << nb) - 1u)) << (xx & 31);
            atomicOr(&c.burn[(size_t)yy * words + wd], bits);
            xx = hi + 1;
          }
        }
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      int s = 0;
      for (int k = 0; k < nw; ++k) s += warp_counts[k];
      base += s;
    }
    __syncthreads();
  }
  if (threadIdx.x < 64) c.bin_want[64 + threadIdx.x] = bin_cnt[threadIdx.x];
  if (threadIdx.x == 0) c.stats[0] = base;  // number of alive features
}

// ---------------------------------------------------------------- response tiles
__device__ __forceinline__ float find_min_1d(float y1, float y2, float y3) {
  const float k = y1 - 2.f * y2 + y3;
  const float m = fabsf(k) <= (10 * 1.1920928955078125e-07f) ? 0.f : __fdividef(0.5f * (y1 - y3), k);
  if (m >= 0.5f) return 0.5f;
  if (m <= -0.5f) return -0.5f;
  return m;
}

// One CTA per 64x32 tile of level 0 (256 threads).  Shared memory holds (gx, gy) on the tile plus
// a 4-pixel halo (tensor taps 3 + NMS 1), the horizontal 7-tap sums as three planes, and later the
// response (aliasing the gradients) and the NMS values (aliasing the sums).
// kSplit = false: the single-camera path; alive_kernel ran first and the burn applies here, the maps
//   are written only for debugging.
// kSplit = true: the batched path; no burn yet, the response map is always written for
//   cells_kernel.
namespace tile {
constexpr int TW = 64, TH = 32;              // core
constexpr int RW = TW + 2;                   // response region width (height TH + 2)
constexpr int GW = TW + 10, GH = TH + 8;     // gradients loaded (two spare columns for 4-wide quads)
constexpr int GS = 76;                       // row stride of the gradient planes (16-byte rows)
constexpr int HS = 68;                       // row stride of the horizontal sums (>= RW, 4-aligned)
constexpr int RS = 68;                       // row stride of the response
constexpr int kThreads = 256;
constexpr int kOffH = 0;                                     // 3 planes [GH][HS]
constexpr int kOffG = kOffH + 3 * GH * HS * 4;               // 2 planes [GH][GS]
constexpr int kSmem = kOffG + 2 * GH * GS * 4;
}  // namespace tile

__device__ __forceinline__ float2 dup(float c) { return make_float2(c, c); }

// Bounded wait on phase `phase` of the mbarrier at shared address `bar`: false when `limit` polls
// all found it incomplete.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t phase, int limit) {
  for (int i = 0; i < limit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(bar), "r"(phase)
        : "memory");
    if (done) return true;
  }
  return false;
}


template <bool kSplit>
__global__ void __launch_bounds__(tile::kThreads) tile_kernel(const __grid_constant__ SelectBatch b) {
  using namespace tile;
  extern __shared__ __align__(128) unsigned char tsm[];
  float* hxx = reinterpret_cast<float*>(tsm + kOffH);
  float* hxy = hxx + GH * HS;
  float* hyy = hxy + GH * HS;
  float* gxs = reinterpret_cast<float*>(tsm + kOffG);
  float* gys = gxs + GH * GS;
  float* resp = reinterpret_cast<float*>(tsm + kOffG);  // after the horizontal pass
  float* nms = hxx;                                      // after the vertical pass
  __shared__ float part[8][8];
  __shared__ __align__(8) uint64_t tbar;  // the TMA staging's mbarrier

  int lo = 0, hi = b.ncams - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (b.cam[mid].tile_begin <= (int)blockIdx.x) lo = mid; else hi = mid - 1;
  }
  const SelectCam& c = b.cam[lo];
  const int t = (int)blockIdx.x - c.tile_begin;
  const int X = (t % c.tiles_x) * TW, Y = (t / c.tiles_x) * TH;
  const int w = c.w, h = c.h;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;

  // A. gradients on [X-4, X+70) x [Y-4, Y+36), mirrored like the reference's tile loader (and
  //    clamped, as its texture does, for images smaller than the mirror span).  Every copy is an
  //    asynchronous global->shared copy issued before the one wait, so a thread has all of its
  //    loads in flight at once.
  const bool interior = X >= 4 && Y >= 4 && X - 4 + GW <= w && Y - 4 + GH <= h;
  if (interior && c.grad_tmap) {
    // interior tile, batched path: one TMA copy per plane of the GS x GH box at (X - 4, Y - 4)
    // (X - 4 is a multiple of 4: its byte offset a multiple of 16; the box's two spare columns are
    // not read), completing on an mbarrier.  The wait is bounded: a copy that does not arrive skips
    // the tile and raises the batch's status flag.
    const uint32_t bar = smem_addr(&tbar);
    if (tid == 0) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar));
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (tid == 0) {
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(2 * GH * GS * 4)
                   : "memory");
#pragma unroll
      for (int plane = 0; plane < 2; ++plane)
        asm volatile(
            "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
            "[%4];" ::"r"(smem_addr(plane ? gys : gxs)),
            "l"(reinterpret_cast<uint64_t>(c.grad_tmap + plane)), "r"(X - 4), "r"(Y - 4), "r"(bar)
            : "memory");
    }
    if (__syncthreads_or(!mbar_wait_bounded(bar, 0, b.wait_limit))) {
      if (tid == 0 && b.status) atomicOr(b.status, 4);
      // the copies may still land: wait once more with the full bound, so that no write targets a
      // retired CTA's shared memory
      mbar_wait_bounded(bar, 0, kDefaultWaitLimit);
      return;
    }
  } else if (interior) {
    // interior tile: 16-byte copies (X - 4 is a multiple of 4 and rows are 16-byte aligned)
    for (int i = tid; i < GH * 19 * 2; i += kThreads) {
      const int plane = i / (GH * 19), k = i - plane * (GH * 19);
      const int r = k / 19, v = k - r * 19;
      const float* src = (plane ? c.gy : c.gx) + (size_t)(Y - 4 + r) * c.pitch + (X - 4);
      float* dst = (plane ? gys : gxs) + r * GS;
      if (v < 18) cp_async16(dst + 4 * v, src + 4 * v);
      else cp_async8(dst + 72, src + 72);
    }
  } else {
    for (int i = tid; i < GH * GW; i += kThreads) {
      const int r = i / GW, q = i - r * GW;
      const int yy = min(max(mirror_index(Y - 4 + r, h), 0), h - 1);
      const int xx = min(max(mirror_index(X - 4 + q, w), 0), w - 1);
      const size_t o = (size_t)yy * c.pitch + xx;
      cp_async4(gxs + r * GS + q, c.gx + o);
      cp_async4(gys + r * GS + q, c.gy + o);
    }
  }
  cp_async_wait_all();
  __syncthreads();

  // B. horizontal 7-tap sums for 40 rows x 68 columns, two column pairs per thread with packed
  //    FP32x2 arithmetic: xx += (c_j gx) gx, xy += (c_j gx) gy, yy += (c_j gy) gy (gftt.cu:131-137)
  for (int qd = tid; qd < GH * (HS / 4); qd += kThreads) {
    const int r = qd / (HS / 4), q0 = (qd - r * (HS / 4)) * 4;
    float2 ax[5], ay[5];
#pragma unroll
    for (int m = 0; m < 5; ++m) {
      ax[m] = *reinterpret_cast<const float2*>(gxs + r * GS + q0 + 2 * m);
      ay[m] = *reinterpret_cast<const float2*>(gys + r * GS + q0 + 2 * m);
    }
    // pairs (v[k], v[k+1]) of columns q0 + k, k = 0..8
    auto px = [&](int k) { return (k & 1) ? make_float2(ax[k >> 1].y, ax[(k >> 1) + 1].x) : ax[k >> 1]; };
    auto py = [&](int k) { return (k & 1) ? make_float2(ay[k >> 1].y, ay[(k >> 1) + 1].x) : ay[k >> 1]; };
    float2 xx0 = dup(0.f), xy0 = dup(0.f), yy0 = dup(0.f), xx1 = dup(0.f), xy1 = dup(0.f), yy1 = dup(0.f);
#pragma unroll
    for (int j = 0; j < 7; ++j) {
      const float2 cj = dup(gauss7(j));
      const float2 gx0 = px(j), gy0 = py(j), gx1 = px(j + 2), gy1 = py(j + 2);
      const float2 cx0 = __fmul2_rn(cj, gx0), cy0 = __fmul2_rn(cj, gy0);
      const float2 cx1 = __fmul2_rn(cj, gx1), cy1 = __fmul2_rn(cj, gy1);
      xx0 = __ffma2_rn(cx0, gx0, xx0);
      xy0 = __ffma2_rn(cx0, gy0, xy0);
      yy0 = __ffma2_rn(cy0, gy0, yy0);
      xx1 = __ffma2_rn(cx1, gx1, xx1);
      xy1 = __ffma2_rn(cx1, gy1, xy1);
      yy1 = __ffma2_rn(cy1, gy1, yy1);
    }
    *reinterpret_cast<float4*>(hxx + r * HS + q0) = make_float4(xx0.x, xx0.y, xx1.x, xx1.y);
    *reinterpret_cast<float4*>(hxy + r * HS + q0) = make_float4(xy0.x, xy0.y, xy1.x, xy1.y);
    *reinterpret_cast<float4*>(hyy + r * HS + q0) = make_float4(yy0.x, yy0.y, yy1.x, yy1.y);
  }
  __syncthreads();

  // C. vertical 7-tap and the measure (gftt.cu:61-66, 148-160) for 34 rows x 66 columns, packed
  //    FP32x2 arithmetic: a column pair and a strip of kStrip rows per thread (the last strip starts
  //    at row 29 and stores rows 30-33 only).  Each staged row of horizontal sums is added into every
  //    output row it is a tap of; an output row's taps still arrive in order j = 0..6.
  {
    constexpr int kStrip = 5, kStrips = (TH + 2 + kStrip - 1) / kStrip;
    static_assert(kStrips * (RW / 2) <= kThreads, "one strip per thread");
    if (tid < kStrips * (RW / 2)) {
      const int s = tid / (RW / 2), q = (tid - s * (RW / 2)) * 2;
      const int r0 = min(s * kStrip, TH + 2 - kStrip), keep = s * kStrip - r0;
      float2 xx[kStrip], xy[kStrip], yy[kStrip];
#pragma unroll
      for (int o = 0; o < kStrip; ++o) xx[o] = xy[o] = yy[o] = dup(0.f);
#pragma unroll
      for (int k = 0; k < kStrip + 6; ++k) {
        const float2 a = *reinterpret_cast<const float2*>(hxx + (r0 + k) * HS + q);
        const float2 bb = *reinterpret_cast<const float2*>(hxy + (r0 + k) * HS + q);
        const float2 cc = *reinterpret_cast<const float2*>(hyy + (r0 + k) * HS + q);
#pragma unroll
        for (int o = 0; o < kStrip; ++o) {
          const int j = k - o;
          if (j < 0 || j > 6) continue;
          const float2 cj = dup(gauss7(j));
          xx[o] = __ffma2_rn(cj, a, xx[o]);
          xy[o] = __ffma2_rn(cj, bb, xy[o]);
          yy[o] = __ffma2_rn(cj, cc, yy[o]);
        }
      }
#pragma unroll
      for (int o = 0; o < kStrip; ++o) {
        if (o < keep) continue;
        const float2 d = __fadd2_rn(xx[o], make_float2(-yy[o].x, -yy[o].y));
        const float2 D2 = __ffma2_rn(__fmul2_rn(dup(4.f), xy[o]), xy[o], __fmul2_rn(d, d));
        const float2 T = __fadd2_rn(xx[o], yy[o]);
        const float2 D = make_float2(__fsqrt_rn(D2.x), __fsqrt_rn(D2.y));
        const float2 e1 = __fadd2_rn(__fmul2_rn(__fadd2_rn(T, make_float2(-D.x, -D.y)), dup(0.5f)), dup(1.f));
        *reinterpret_cast<float2*>(resp + (r0 + o) * RS + q) = make_float2(__logf(e1.x), __logf(e1.y));
      }
    }
  }
  __syncthreads();

  // D. NMS on the core with clamped neighbours, then (single-camera path) the burn mask; four
  //    pixels (x .. x+3, x a multiple of 4) per work item from three rows of six response values
  const int words = (w + 31) / 32;
  const bool resp_vec = (w & 3) == 0 && (reinterpret_cast<uintptr_t>(c.resp) & 15) == 0;
  for (int i = tid; i < TW * TH / 4; i += kThreads) {
    const int r = i / (TW / 4), q = (i - r * (TW / 4)) * 4;
    const int x = X + q, y = Y + r;
    float m[4] = {0.f, 0.f, 0.f, 0.f};
    if (y < h && x < w) {
      float n[3][6];  // response rows y-1 .. y+1, columns x-1 .. x+4
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const float4 a = *reinterpret_cast<const float4*>(resp + (r + k) * RS + q);
        const float2 e = *reinterpret_cast<const float2*>(resp + (r + k) * RS + q + 4);
        n[k][0] = a.x;
        n[k][1] = a.y;
        n[k][2] = a.z;
        n[k][3] = a.w;
        n[k][4] = e.x;
        n[k][5] = e.y;
      }
      const bool inner = x > 0 && y > 0 && x + 4 < w && y < h - 1;  // every pixel's 8 neighbours inside
      const uint32_t burn = kSplit ? 0u : __ldg(c.burn + (size_t)y * words + (x >> 5)) >> (x & 31);
      float v[4];
#pragma unroll
      for (int p = 0; p < 4; ++p) {
        v[p] = n[1][p + 1];
        bool is_max;
        if (inner) {
          is_max = n[0][p] <= v[p] && n[0][p + 1] <= v[p] && n[0][p + 2] <= v[p] && n[1][p] <= v[p] &&
                   n[1][p + 2] <= v[p] && n[2][p] <= v[p] && n[2][p + 1] <= v[p] && n[2][p + 2] <= v[p];
        } else {
          is_max = x + p < w;
#pragma unroll
          for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
            for (int dx = -1; dx <= 1; ++dx) {
              if (!dx && !dy) continue;
              const int yy = min(max(y + dy, 0), h - 1) - Y + 1, xx = min(max(x + p + dx, 0), w - 1) - X + 1;
              is_max = is_max && resp[yy * RS + xx] <= v[p];
            }
        }
        m[p] = is_max && !((burn >> p) & 1u) ? v[p] : 0.f;
      }
      if (kSplit || b.debug) {
        float* o = c.resp + (size_t)y * w + x;
        if (resp_vec && x + 3 < w) {
          *reinterpret_cast<float4*>(o) = make_float4(v[0], v[1], v[2], v[3]);
        } else {
#pragma unroll
          for (int p = 0; p < 4; ++p)
            if (x + p < w) o[p] = v[p];
        }
      }
      if (!kSplit && b.debug)
#pragma unroll
        for (int p = 0; p < 4; ++p)
          if (x + p < w) c.nms[(size_t)y * w + x + p] = m[p];
    }
    *reinterpret_cast<float4*>(nms + r * TW + q) = make_float4(m[0], m[1], m[2], m[3]);
  }
  __syncthreads();

  // E. 32 cells of 8x8 (in the batched path before the burn: cells_kernel redoes the cells that
  //    alive features reach), eight threads per cell.  The reference's warp (lane l holds pixels l and
  //    l + 32, the second taken only when strictly greater, then a shfl_down tree whose merges keep
  //    the lower lane on ties) yields the first maximum in (lane, element) order.  Here thread g of a
  //    cell scans lanes 4g .. 4g+3 in that order with the same strict rule, and a 3-level shfl_down
  //    merge within the cell's eight threads keeps the lower thread on ties: the same pixel.
  const int cw = w / 8, ch = h / 8;
  static_assert(kThreads == 32 * 8, "eight threads per cell");
  {
    const int cc = tid >> 3, g = tid & 7;
    const int ccx = cc & 7, ccy = cc >> 3;
    const int cellx = X / 8 + ccx, celly = Y / 8 + ccy;
    float m = 0.f;
    unsigned idx = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int f = 4 * g + (k >> 1) + 32 * (k & 1), dy = f >> 3, dx = f & 7;
      const float v = nms[(ccy * 8 + dy) * TW + ccx * 8 + dx];
      if (v > m) {
        m = v;
        idx = (unsigned)dx | ((unsigned)dy << 16);
      }
    }
#pragma unroll
    for (int d = 1; d < 8; d <<= 1) {
      const float m2 = __shfl_down_sync(0xffffffffu, m, d, 8);
      const unsigned i2 = __shfl_down_sync(0xffffffffu, idx, d, 8);
      if (m2 > m) {
        m = m2;
        idx = i2;
      }
    }
    if (g == 0 && cellx < cw && celly < ch) {
      const int cell = celly * cw + cellx;
      const int px = cellx * 8 + (int)(idx & 0xffffu), py = celly * 8 + (int)(idx >> 16);
      float out_m = 0.f;
      float2 pos = make_float2((float)px, (float)py);
      if (m > (float)1e-2) {
        out_m = m;
        if (!(px == 0 || px == w - 1 || py == 0 || py == h - 1)) {
          const float* rp = resp + (py - Y + 1) * RS + (px - X + 1);
          const float gc = rp[0];
          pos.x = (float)px + find_min_1d(rp[-1], gc, rp[1]);
          pos.y = (float)py + find_min_1d(rp[-RS], gc, rp[RS]);
        }
      }
      c.cell_m[cell] = out_m;
      c.cell_xy[cell] = pos;
    }
  }

  // F. 16x16 sub-tile sums of the response (accumulateGFTT_kernel's reduction order): warp w sums
  //    rows 2w, 2w+1 of each of the 8 sub-tiles, then a 3-level butterfly over the 8 warp sums
  //    (the eight warp sums share butterflies, three, three and two at a time, each bit-identical to
  //    its own warp_sum)
  {
    float v[8];
#pragma unroll
    for (int s8 = 0; s8 < 8; ++s8) {
      const int si = s8 >> 2, sj = s8 & 3;
      const int ty = 2 * wid + (lane >> 4), tx = lane & 15;
      const int x = X + sj * 16 + tx, y = Y + si * 16 + ty;
      v[s8] = (x < w && y < h) ? resp[(si * 16 + ty + 1) * RS + sj * 16 + tx + 1] : 0.f;
    }
    warp_sum3(v[0], v[1], v[2], lane);
    warp_sum3(v[3], v[4], v[5], lane);
    warp_sum2(v[6], v[7], lane);
    if (lane == 0)
#pragma unroll
      for (int s8 = 0; s8 < 8; ++s8) part[s8][wid] = v[s8];
  }
  __syncthreads();
  {
    float v = lane < 8 ? part[wid][lane] : 0.f;
#pragma unroll
    for (int m = 1; m < 8; m <<= 1) v += __shfl_xor_sync(0xffffffffu, v, m);
    const int si = wid >> 2, sj = wid & 3;
    const int stx = X / 16 + sj, sty = Y / 16 + si;
    const int sw = (w + 15) / 16, sh = (h + 15) / 16;
    if (lane == 0 && stx < sw && sty < sh) c.sub_sum[sty * sw + stx] = v;
  }
}

// ---------------------------------------------------------------- burned cells
// Redoes the cells that an alive feature's 9x9 window reaches: NMS again from the response map,
// burned pixels zeroed (filter_maximums_kernel, selection_v2.cu:251-277), the cell's max/argmax
// again with the reference's lane order, then the refinement.  One warp per 32 cells of the
// touched-cell bit mask, four touched cells at a time.
__global__ void __launch_bounds__(256) cells_kernel(const __grid_constant__ SelectBatch b, int words_total) {
  const int lane = threadIdx.x & 31;
  const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  if (gw >= words_total) return;
  int lo = 0, hi = b.ncams - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (b.cam[mid].touched_begin <= gw) lo = mid; else hi = mid - 1;
  }
  const SelectCam& c = b.cam[lo];
  const int word = gw - c.touched_begin;
  const int vcw = (c.w + 7) / 8, vch = (c.h + 7) / 8;  // cell grid incl. partial border cells
  if (word * 32 >= vcw * vch) return;
  const uint32_t bits = c.touched[word];
  const int w = c.w, h = c.h, cw = w / 8, ch = h / 8;
  const int bwords = (w + 31) / 32;
  // the word's touched cells, four at a time: eight lanes per cell, lane g of a cell scanning the
  // reference's lanes 4g .. 4g+3 (pixels l and l + 32 of lane l, the second taken only when strictly
  // greater) and a 3-level merge that keeps the lower lane on ties: the first maximum in the
  // reference's (lane, element) order, as downsample_gftt_x8_kernel's warp finds it
  const uint32_t valid = (word * 32 + 32 <= vcw * vch) ? 0xffffffffu : ((1u << (vcw * vch - word * 32)) - 1u);
  const uint32_t cells = bits & valid;
  const int ncells = __popc(cells);
  const int j = lane >> 3, g = lane & 7;
  for (int base = 0; base < ncells; base += 4) {
    const int ci = base + j;
    const int k = ci < ncells ? (int)__fns(cells, 0, ci + 1) : -1;
    const int vcell = word * 32 + (k >= 0 ? k : 0);
    const int cellx = vcell % vcw, celly = vcell / vcw;
    float m = 0.f;
    unsigned idx = 0;
    if (k >= 0) {
#pragma unroll
      for (int kk = 0; kk < 8; ++kk) {
        const int f = 4 * g + (kk >> 1) + 32 * (kk & 1), dy = f >> 3, dx = f & 7;
        const int x = cellx * 8 + dx, y = celly * 8 + dy;
        if (x < w && y < h && !((c.burn[(size_t)y * bwords + (x >> 5)] >> (x & 31)) & 1u)) {
          const float v = c.resp[(size_t)y * w + x];
          bool is_max = true;
#pragma unroll
          for (int ny = -1; ny <= 1; ++ny)
#pragma unroll
            for (int nx = -1; nx <= 1; ++nx) {
              if (!nx && !ny) continue;
              const int yy = min(max(y + ny, 0), h - 1), xx = min(max(x + nx, 0), w - 1);
              is_max &= c.resp[(size_t)yy * w + xx] <= v;
            }
          if (is_max && v > m) {
            m = v;
            idx = (unsigned)dx | ((unsigned)dy << 16);
          }
        }
      }
    }
#pragma unroll
    for (int d = 1; d < 8; d <<= 1) {
      const float m2 = __shfl_down_sync(0xffffffffu, m, d, 8);
      const unsigned i2 = __shfl_down_sync(0xffffffffu, idx, d, 8);
      if (m2 > m) {
        m = m2;
        idx = i2;
      }
    }
    if (g == 0 && k >= 0 && cellx < cw && celly < ch) {
      const int cell = celly * cw + cellx;
      const int px = cellx * 8 + (int)(idx & 0xffffu), py = celly * 8 + (int)(idx >> 16);
      float out_m = 0.f;
      float2 pos = make_float2((float)px, (float)py);
      if (m > (float)1e-2) {
        out_m = m;
        if (!(px == 0 || px == w - 1 || py == 0 || py == h - 1)) {
          const float* r = c.resp + (size_t)py * w + px;
          const float gc = r[0];
          pos.x = (float)px + find_min_1d(r[-1], gc, r[1]);
          pos.y = (float)py + find_min_1d(r[-w], gc, r[w]);
        }
      }
      c.cell_m[cell] = out_m;
      c.cell_xy[cell] = pos;
    }
  }
}

// ---------------------------------------------------------------- quotas
// Sub-tile index range [lo, hi) whose centres (16 t + 8) fall in bin b of size `bin_px`.
__device__ __forceinline__ int2 bin_range(int b, int bin_px, int n) {
  const int lo = max(0, (b * bin_px - 8 + 15) / 16);
  const int hi = min(n, ((b + 1) * bin_px - 8 + 15) / 16);
  return make_int2(lo, max(hi, lo));
}

constexpr int kMaxBinRows = 40;  // sub-tile rows per bin for heights <= 4096

__global__ void __launch_bounds__(512) quota_kernel(const __grid_constant__ SelectBatch b) {
  const SelectCam& c = b.cam[blockIdx.x];
  __shared__ float rows[64][kMaxBinRows];
  __shared__ float bins[64];
  const int bw = c.w / 8, bh = c.h / 8;
  const int sw = (c.w + 15) / 16, sh = (c.h + 15) / 16;
  if (bw > 0 && bh > 0) {
    // row sums: one (bin column, sub-tile row) per thread, left to right
    for (int i = threadIdx.x; i < 8 * sh; i += blockDim.x) {
      const int bx = i & 7, ty = i >> 3;
      const int by = (ty * 16 + 8) / bh;
      if (by >= 8) continue;
      const int2 xr = bin_range(bx, bw, sw);
      float row = 0.f;
      for (int tx = xr.x; tx < xr.y; ++tx) row = __fadd_rn(row, c.sub_sum[ty * sw + tx]);
      rows[by * 8 + bx][ty - bin_range(by, bh, sh).x] = row;
    }
  }
  __syncthreads();
  if (threadIdx.x < 64) {
    float acc = 0.f;
    if (bw > 0 && bh > 0) {
      const int2 yr = bin_range(threadIdx.x >> 3, bh, sh);
      for (int k = 0; k < yr.y - yr.x; ++k) acc = __fadd_rn(acc, rows[threadIdx.x][k]);
    }
    bins[threadIdx.x] = acc;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    float sum = 0.f;
    for (int i = 0; i < 64; ++i) sum = __fadd_rn(sum, bins[i]);
    const int n_alive = c.stats[0];
    // MonoSOFGPU::addFeatures asks for num_desired_tracks - alive (sof_mono_gpu.cpp:225-229)
    const int wanted = c.target_total > 0 ? max(c.target_total - n_alive, 0) : c.num_desired;
    c.stats[4] = wanted;
    const float expected = (float)(n_alive + wanted);
    int total = 0;
    for (int i = 0; i < 64; ++i) {
      int want = 0;
      if (sum > 0.f) {
        const float e = roundf(__fdiv_rn(__fmul_rn(expected, bins[i]), sum));
        const int ei = e > 0.f ? (int)e : 0;
        const int prev = c.bin_want[64 + i];
        want = ei > prev ? ei - prev : 0;
      }
      c.bin_want[i] = want;
      total += want;
    }
    c.stats[1] = total;
    c.stats[2] = 0;  // kept candidates (bin_kernel adds)
  }
}

// ---------------------------------------------------------------- per-bin selection
// Ascending bitonic sort of n_pow2 (a power of two) keys in shared memory by the whole block
// (blockDim.x a multiple of 32).  Compare-exchange steps whose partner index i ^ j lies in the same
// run of 32 keys (j <= 16) run in registers, lane i of a warp holding key i of its run and swapping
// through shuffles, so the block meets at a barrier once per merge width k for them instead of once
// per step; wider steps exchange through shared memory.  The network is the same, so is the result.
template <typename K>
__device__ void block_bitonic_sort(K* keys, int n_pow2) {
  const int lane = threadIdx.x & 31;
  for (int k = 2; k <= n_pow2; k <<= 1) {
    for (int j = k >> 1; j >= 32; j >>= 1) {
      for (int i = threadIdx.x; i < n_pow2; i += blockDim.x) {
        const int ixj = i ^ j;
        if (ixj > i) {
          const K a = keys[i], bb = keys[ixj];
          const bool up = (i & k) == 0;
          if ((a > bb) == up) {
            keys[i] = bb;
            keys[ixj] = a;
          }
        }
      }
      __syncthreads();
    }
    // steps j = min(k/2, 16) .. 1: the lower index of a pair keeps the smaller key when the run of
    // width k ascends ((i & k) == 0) and the larger one when it descends
    for (int base = (int)(threadIdx.x & ~31u); base < n_pow2; base += blockDim.x) {
      const int i = base + lane;
      K v = i < n_pow2 ? keys[i] : K(0);
      const bool up = (i & k) == 0;
      for (int j = min(k >> 1, 16); j > 0; j >>= 1) {
        const K o = __shfl_xor_sync(0xffffffffu, v, j);
        const bool lower = (lane & j) == 0;
        v = (lower == up) ? (o < v ? o : v) : (o > v ? o : v);
      }
      if (i < n_pow2) keys[i] = v;
    }
    __syncthreads();
  }
}

// The k-th smallest (1 <= k < n) of n distinct keys in shared memory, by the whole block: a radix
// select from the top byte down.  Each pass histograms the byte of the keys that share the bytes
// fixed so far, and warp 0 finds the bucket that holds the k-th key (each lane scanning eight
// buckets after a prefix sum over the lanes).  Returned to every thread.
__device__ uint64_t block_select_kth(const uint64_t* keys, int n, int k) {
  __shared__ int hist[256];
  __shared__ uint64_t s_prefix;
  __shared__ int s_k;
  if (threadIdx.x == 0) {
    s_prefix = 0ull;
    s_k = k;
  }
  for (int shift = 56; shift >= 0; shift -= 8) {
    for (int i = threadIdx.x; i < 256; i += blockDim.x) hist[i] = 0;
    __syncthreads();
    const uint64_t prefix = s_prefix;
    const uint64_t hi = shift == 56 ? 0ull : (~0ull << (shift + 8));
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      const uint64_t key = keys[i];
      if ((key & hi) == prefix) atomicAdd(&hist[(int)(key >> shift) & 255], 1);
    }
    __syncthreads();
    if (threadIdx.x < 32) {
      const int lane = threadIdx.x;
      int h[8], sum = 0;
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        h[q] = hist[8 * lane + q];
        sum += h[q];
      }
      int incl = sum;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += y;
      }
      const int kk = s_k;
      int cum = incl - sum;
      if (cum < kk && kk <= incl) {
        int sel = 7;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          if (sel == 7 && q < 7 && cum + h[q] >= kk) sel = q;
          else if (sel == 7 && q < 7) cum += h[q];
        }
        s_prefix = prefix | ((uint64_t)(8 * lane + sel) << shift);
        s_k = kk - cum;
      }
    }
    __syncthreads();
  }
  return s_prefix;
}

__global__ void bin_kernel(const __grid_constant__ SelectBatch b, int key_cap) {
  extern __shared__ uint64_t keys[];
  __shared__ int count;
  const SelectCam& c = b.cam[blockIdx.y];
  const int bin = blockIdx.x, bx = bin & 7, by = bin >> 3;
  const int bw = c.w / 8, bh = c.h / 8;
  if (bw <= 0 || bh <= 0) return;
  const int want = c.bin_want[bin];
  if (want <= 0) return;  // block-uniform
  if (threadIdx.x == 0) count = 0;
  __syncthreads();
  const int cw = c.w / 8, ch = c.h / 8;
  // cells whose refined position can land in this bin (refinement moves <= 0.5 px)
  const int cx0 = max((bx * bw - 1) / 8, 0), cx1 = min(((bx + 1) * bw) / 8, cw - 1);
  const int cy0 = max((by * bh - 1) / 8, 0), cy1 = min(((by + 1) * bh) / 8, ch - 1);
  const int ncx = cx1 - cx0 + 1, ncy = cy1 - cy0 + 1;
  const float xmax = (float)(unsigned)(c.w - 1 - c.border[3]), ymax = (float)(unsigned)(c.h - 1 - c.border[1]);
  for (int i = threadIdx.x; i < ncx * ncy; i += blockDim.x) {
    const int cy = cy0 + i / ncx, cx = cx0 + i % ncx;
    const int cell = cy * cw + cx;
    const float m = c.cell_m[cell];
    if (!(m > 0.f)) continue;
    const float2 p = c.cell_xy[cell];
    if (p.x < (float)c.border[2] || p.x > xmax || p.y < (float)c.border[0] || p.y > ymax) continue;
    if (c.mask && c.mask[(size_t)p.y * c.mask_pitch + (size_t)p.x] != 0) continue;
    const unsigned kbx = (unsigned)__fdiv_rn(p.x, (float)bw), kby = (unsigned)__fdiv_rn(p.y, (float)bh);
    if (kbx != (unsigned)bx || kby != (unsigned)by) continue;
    const int slot = atomicAdd(&count, 1);
    if (slot < key_cap) keys[slot] = make_key(m, cell);
  }
  __syncthreads();
  const int n = min(count, key_cap);
  if (count > key_cap && threadIdx.x == 0) atomicOr(&c.stats[3], 1);  // capacity flag
  // the bin keeps its `keep` smallest keys (strongest first); final_kernel orders all kept keys, so
  // only the set matters here: every key up to the keep-th smallest (keys are distinct, a cell each)
  const int keep = min(want, n);
  const uint64_t last = keep < n ? block_select_kth(keys, n, keep) : ~0ull;
  __shared__ int base, written;
  if (threadIdx.x == 0) {
    base = atomicAdd(&c.stats[2], keep);
    written = 0;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const uint64_t key = keys[i];
    if (key > last) continue;
    const int slot = base + atomicAdd(&written, 1);
    if (slot < c.q_cap) c.q_keys[slot] = key;
    else atomicOr(&c.stats[3], 2);
  }
}

// ---------------------------------------------------------------- final order
__global__ void final_kernel(const __grid_constant__ SelectBatch b, int key_cap) {
  extern __shared__ uint64_t keys[];
  const SelectCam& c = b.cam[blockIdx.x];
  const int n = min(min(c.stats[2], c.q_cap), key_cap);
  if (c.stats[2] > key_cap && threadIdx.x == 0) atomicOr(&c.stats[3], 4);
  int np = 1;
  while (np < n) np <<= 1;
  for (int i = threadIdx.x; i < np; i += blockDim.x) keys[i] = i < n ? c.q_keys[i] : ~0ull;
  __syncthreads();
  block_bitonic_sort(keys, np);
  const int out = min(n, c.stats[4]);
  const int cw = c.w / 8;
  (void)cw;
  for (int i = threadIdx.x; i < out; i += blockDim.x) {
    const int cell = (int)(keys[i] & 0xffffffffu);
    const float2 p = c.cell_xy[cell];
    c.out_xy[2 * i] = p.x;
    c.out_xy[2 * i + 1] = p.y;
  }
  if (threadIdx.x == 0) *c.out_count = out;
}

}  // namespace

bool encode_select_grad_tmaps(CUtensorMap* maps, const float* gx, const float* gy, int w, int h, int pitch_floats) {
  return encode_plane_tmap_f32(maps, gx, w, h, pitch_floats, tile::GS, tile::GH) &&
         encode_plane_tmap_f32(maps + 1, gy, w, h, pitch_floats, tile::GS, tile::GH);
}

int select_tile_w() { return tile::TW; }
int select_tile_h() { return tile::TH; }

cudaError_t select_init() {
  cudaError_t e = cudaFuncSetAttribute(tile_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, tile::kSmem);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(tile_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, tile::kSmem);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(bin_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)(sizeof(uint64_t) * kMaxSelectKeys));
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(final_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)(sizeof(uint64_t) * kMaxSelectKeys));
}

cudaError_t launch_select_response(const SelectBatch& b, int total_tiles, cudaStream_t s) {
  tile_kernel<true><<<total_tiles, tile::kThreads, tile::kSmem, s>>>(b);
  return cudaGetLastError();
}

namespace {
cudaError_t launch_quota_bins_final(const SelectBatch& b, int bin_key_cap, int final_key_cap, cudaStream_t s) {
  quota_kernel<<<b.ncams, 512, 0, s>>>(b);
  bin_kernel<<<dim3(64, b.ncams), 256, sizeof(uint64_t) * bin_key_cap, s>>>(b, bin_key_cap);
  final_kernel<<<b.ncams, 1024, sizeof(uint64_t) * final_key_cap, s>>>(b, final_key_cap);
  return cudaGetLastError();
}
}  // namespace

cudaError_t launch_select_rest(const SelectBatch& b, int touched_words, int bin_key_cap, int final_key_cap,
                               cudaStream_t s) {
  if (bin_key_cap > kMaxSelectKeys || final_key_cap > kMaxSelectKeys) return cudaErrorInvalidValue;
  alive_kernel<<<b.ncams, 1024, 0, s>>>(b);
  cells_kernel<<<(touched_words + 7) / 8, 256, 0, s>>>(b, touched_words);
  return launch_quota_bins_final(b, bin_key_cap, final_key_cap, s);
}

cudaError_t launch_select(const SelectBatch& b, int total_tiles, int bin_key_cap, int final_key_cap,
                          cudaStream_t s) {
  if (bin_key_cap > kMaxSelectKeys || final_key_cap > kMaxSelectKeys) return cudaErrorInvalidValue;
  alive_kernel<<<b.ncams, 1024, 0, s>>>(b);
  tile_kernel<false><<<total_tiles, tile::kThreads, tile::kSmem, s>>>(b);
  return launch_quota_bins_final(b, bin_key_cap, final_key_cap, s);
}

}  // namespace fe
