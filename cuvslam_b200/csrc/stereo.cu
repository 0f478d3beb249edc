// Left-to-right matching: LK (horizontal for rectified pairs, 2-D otherwise) from each primary point
// towards its epipolar candidates, first success wins, every camera pair of a rig in one launch.
//
// The reference (MultiSOFGPU::LaunchTrackingPrimaryToSecondary, sof_multicamera_gpu.cpp:118-190)
// runs rounds k = 0, 1, ...: round k tracks candidate k of every point that has no success yet and
// has a k-th candidate (one lk_track_horizontal launch, a device->host copy and a stream
// synchronisation per round); after round k it stops once at least frac * n points are matched.
// An attempt's result does not depend on the other attempts, so the outcome is fixed by f_i, the
// index of point i's first successful candidate: the stop round K is the first round with
// #{i : f_i <= K} >= frac * n, and point i is matched iff f_i <= K.
//
// Here the (point, candidate) attempts form one list in round order, taken by persistent warps
// from an atomic counter.  Before tracking, an attempt (i, k) is skipped when point i already has a
// success at an earlier candidate (best[i] < k) or k lies beyond a round already known to meet the
// early-exit count (stop < k).  A success lowers best[i] with atomicMin and, when it is the point's
// new first success, adds the point to cnt[r] for the rounds r it now counts in; a count that
// reaches frac * n lowers stop to r.  Counts only grow, so a stop round seen by any warp is an upper
// bound of K, every attempt with k <= K whose point has no earlier success is tracked, and the
// final stop equals K whatever the order in which warps ran.  Each success stores its position at
// pos[i * maxc + k]; the last CTA to finish publishes best[i] <= stop as the match.
#include <cuda_runtime.h>

#include <climits>

#include "fe_common.cuh"
#include "fe_internal.h"
#include "lk_common.cuh"
#include "lk_track.cuh"

namespace fe {

namespace {

using namespace lk;

constexpr int kWarps = 8, kMinBlocks = 3;
constexpr unsigned kNone = 0xffffffffu;

__device__ __forceinline__ unsigned load_cg(const unsigned* p) { return __ldcg(p); }

// The earliest round known to meet the early-exit count.  With frac * n <= 0 the reference stops
// after round 0 whatever it matched.
__device__ __forceinline__ unsigned stop_of(const StereoPair& P) { return P.need <= 0.f ? 0u : load_cg(P.stop); }

// Candidate list of one point: an explicit list, or the bilinear blend of the four epipolar curves
// around the point's top-level position (EpipolarCurves::Candidates, epipolar_curves.cpp:64-101,
// evaluated in FP32 without contraction: ((w00 c00 + w01 c01) + w10 c10) + w11 c11).
struct Cands {
  int len;
  const float2* list;
  const float2 *c00, *c01, *c10, *c11;
  float w00, w01, w10, w11;
};

__device__ __forceinline__ Cands cands_of(const StereoPair& P, int i) {
  Cands r;
  r.len = 0;
  r.list = nullptr;
  if (P.valid && !P.valid[i]) return r;
  if (P.cand_off) {
    const int o = P.cand_off[i];
    r.len = min(P.cand_off[i + 1] - o, P.maxc);
    r.list = P.cand_xy + o;
    return r;
  }
  const float2 uv = P.uv[i];
  const float vf = __fmul_rn(uv.y, P.inv_scale), uf = __fmul_rn(uv.x, P.inv_scale);
  // outside the corner grid (or NaN): no candidates
  if (!(vf >= 0.f && vf < (float)P.ch && uf >= 0.f && uf < (float)P.cw)) return r;
  const int v0 = (int)vf, u0 = (int)uf;
  if (v0 + 1 >= P.ch || u0 + 1 >= P.cw) return r;
  const float dv = __fsub_rn(vf, (float)v0), du = __fsub_rn(uf, (float)u0);
  const float edu = __fsub_rn(1.f, du), edv = __fsub_rn(1.f, dv);
  r.w00 = __fmul_rn(edu, edv);
  r.w01 = __fmul_rn(du, edv);
  r.w10 = __fmul_rn(edu, dv);
  r.w11 = __fmul_rn(du, dv);
  const int i00 = v0 * P.cw + u0, i10 = i00 + P.cw;
  const int o00 = P.c_off[i00], o01 = P.c_off[i00 + 1], o10 = P.c_off[i10], o11 = P.c_off[i10 + 1];
  const int n00 = o01 - o00, n01 = P.c_off[i00 + 2] - o01, n10 = o11 - o10, n11 = P.c_off[i10 + 2] - o11;
  r.len = min(min(n00, n01), min(n10, n11));
  r.c00 = P.c_xy + o00;
  r.c01 = P.c_xy + o01;
  r.c10 = P.c_xy + o10;
  r.c11 = P.c_xy + o11;
  return r;
}

__device__ __forceinline__ float blend(float w00, float a, float w01, float b, float w10, float c, float w11, float d) {
  return __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(w00, a), __fmul_rn(w01, b)), __fmul_rn(w10, c)), __fmul_rn(w11, d));
}

__device__ __forceinline__ float2 cand_at(const Cands& r, int k) {
  if (r.list) return r.list[k];
  const float2 a = r.c00[k], b = r.c01[k], c = r.c10[k], d = r.c11[k];
  return make_float2(blend(r.w00, a.x, r.w01, b.x, r.w10, c.x, r.w11, d.x),
                     blend(r.w00, a.y, r.w01, b.y, r.w10, c.y, r.w11, d.y));
}

// Full list length of a point (before the maxc cut), for the flags.
__device__ __forceinline__ int list_len(const StereoPair& P, int i) {
  if (!P.cand_off || (P.valid && !P.valid[i])) return 0;
  return P.cand_off[i + 1] - P.cand_off[i];
}

__device__ __forceinline__ int pair_of(const StereoLaunch& p, int g) {
  int lo = 0, hi = p.npairs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (p.pair[mid].begin <= g) lo = mid; else hi = mid - 1;
  }
  return lo;
}

template <int SAMPLING, bool HORIZ>
__global__ void __launch_bounds__(kWarps * 32, kMinBlocks) stereo_kernel(const __grid_constant__ StereoLaunch p) {
  __shared__ WarpSmem smem[kWarps];
  __shared__ fe_track_data tds[kWarps];
  __shared__ int s_last;
  __shared__ int s_matched[kMaxStereoPairs], s_rounds[kMaxStereoPairs], s_flags[kMaxStereoPairs];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const long long total = (long long)p.rounds * p.round;
  fe_track_data& td = tds[wid];
  for (;;) {
    int t = 0;
    if (lane == 0) t = atomicAdd(p.counter, 1);
    t = __shfl_sync(kFull, t, 0);
    if ((long long)t >= total) break;
    const int k = t / p.round, g = t - k * p.round;
    const StereoPair& P = p.pair[pair_of(p, g)];
    const int i = g - P.begin;
    if (k >= P.maxc) continue;
    if ((unsigned)k > stop_of(P)) {
      // every later attempt has a round >= k: leave once that is past every pair's stop or lists
      bool beyond = true;
      if (lane < p.npairs) beyond = k >= p.pair[lane].maxc || (unsigned)k > stop_of(p.pair[lane]);
      if (__all_sync(kFull, beyond)) break;
      continue;
    }
    if (load_cg(&P.best[i]) < (unsigned)k) continue;
    const Cands cs = cands_of(P, i);
    if (k >= cs.len) continue;
    const float2 uv = P.uv[i];
    const float2 c = cand_at(cs, k);
    __syncwarp();
    if (lane < 20) {
      uint32_t w = 0;
      switch (lane) {
        case 0: w = __float_as_uint(uv.x); break;
        case 1: w = __float_as_uint(uv.y); break;
        case 2: w = __float_as_uint(__fsub_rn(c.x, uv.x)); break;
        case 3: w = __float_as_uint(__fsub_rn(c.y, uv.y)); break;
        case 9: w = 0xffffffffu; break;  // cache_index = -1
        case 12: case 15: w = __float_as_uint(1.f); break;  // initial_guess_map = identity
        case 16: w = __float_as_uint(P.radius); break;
        case 17: w = __float_as_uint(P.ncc_thr); break;
        default: break;
      }
      reinterpret_cast<uint32_t*>(&td)[lane] = w;
    }
    __syncwarp();
    track_one<SAMPLING, HORIZ, kModeRef>(P.lk, td, smem[wid], lane, 0, 0.f);
    __syncwarp();
    const bool ok = td.track_status != 0;
    unsigned old = kNone;
    if (lane == 0) {
      atomicAdd(P.attempts, 1);
      if (ok) {
        P.pos[(size_t)i * P.maxc + k] = make_float2(td.track[0], td.track[1]);
        old = atomicMin(&P.best[i], (unsigned)k);
      }
    }
    old = __shfl_sync(kFull, old, 0);
    if (ok && (unsigned)k < old) {
      // point i's first success is now k: it counts in rounds k .. old - 1
      const int hi = old < (unsigned)P.maxc ? (int)old : P.maxc;
      for (int r = k + lane; r < hi; r += 32) {
        const int cnt = atomicAdd(&P.cnt[r], 1) + 1;
        if ((float)cnt >= P.need) atomicMin(P.stop, (unsigned)r);
      }
    }
  }

  // the last CTA to finish publishes every pair's results
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = atomicAdd(p.done, 1) == (int)gridDim.x - 1;
  if (threadIdx.x < kMaxStereoPairs) {
    s_matched[threadIdx.x] = 0;
    s_rounds[threadIdx.x] = 0;
    s_flags[threadIdx.x] = 0;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  for (int q = 0; q < p.npairs; ++q) {
    const StereoPair& P = p.pair[q];
    const unsigned stop = stop_of(P);
    int matched = 0, rounds = 0, flags = 0;
    for (int i = threadIdx.x; i < P.n; i += blockDim.x) {
      const unsigned b = load_cg(&P.best[i]);
      const bool ok = b != kNone && b <= stop;
      const Cands cs = cands_of(P, i);
      const bool valid = !(P.valid && !P.valid[i]);
      const float2 uv = valid ? P.uv[i] : make_float2(0.f, 0.f);
      float4 r0, r1, r2, r3, r4;
      if (ok) {
        const float2 pos = __ldcg(&P.pos[(size_t)i * P.maxc + b]);
        const float2 c = cand_at(cs, (int)b);
        r0 = make_float4(pos.x, pos.y, __fsub_rn(c.x, uv.x), __fsub_rn(c.y, uv.y));
        r1 = make_float4(1.f / 9.f, 0.f, 0.f, 1.f / 9.f);
      } else {
        r0 = make_float4(uv.x, uv.y, 0.f, 0.f);
        r1 = make_float4(0.f, 0.f, 0.f, 0.f);
      }
      r2 = make_float4(__uint_as_float(ok ? 1u : 0u), __uint_as_float(0xffffffffu), 0.f, 0.f);
      r3 = make_float4(1.f, 0.f, 0.f, 1.f);
      r4 = make_float4(P.radius, P.ncc_thr, 0.f, 0.f);
      float4* o = reinterpret_cast<float4*>(P.out + i);
      o[0] = r0;
      o[1] = r1;
      o[2] = r2;
      o[3] = r3;
      o[4] = r4;
      if (P.winner) P.winner[i] = ok ? (int)b : -1;
      matched += ok;
      // rounds the reference runs for this point: while it is unmatched and has a candidate
      const int fi = b == kNone ? INT_MAX : (int)b;
      rounds = max(rounds, fi < cs.len ? fi + 1 : cs.len);
      if (list_len(P, i) > P.maxc) flags |= 1;
    }
    atomicAdd(&s_matched[q], matched);
    atomicMax(&s_rounds[q], rounds);
    atomicOr(&s_flags[q], flags);
  }
  __syncthreads();
  if (threadIdx.x < p.npairs) {
    const StereoPair& P = p.pair[threadIdx.x];
    if (P.stats) {
      const unsigned stop = stop_of(P);
      int rounds = s_rounds[threadIdx.x];
      if (stop != kNone) rounds = min(rounds, (int)stop + 1);
      P.stats[0] = s_matched[threadIdx.x];
      P.stats[1] = rounds;
      P.stats[2] = *(volatile int*)P.attempts;
      P.stats[3] = s_flags[threadIdx.x];
    }
  }
}

template <int SAMPLING, bool HORIZ>
cudaError_t launch_sampling(const StereoLaunch& p, cudaStream_t s) {
  // blocks resident on the device (persistent grid), found once per process
  static const int resident = [] {
    int per_sm = 0, dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, stereo_kernel<SAMPLING, HORIZ>, kWarps * 32, 0);
    return (per_sm > 0 ? per_sm : 1) * (sms > 0 ? sms : 1);
  }();
  const long long total = (long long)p.rounds * p.round;
  const int blocks = (int)max(1LL, min((long long)resident, (total + kWarps - 1) / kWarps));
  stereo_kernel<SAMPLING, HORIZ><<<blocks, kWarps * 32, 0, s>>>(p);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_stereo(const StereoLaunch& p, cudaStream_t s) {
  if (p.horizontal) {
    if (p.sampling == FE_SAMPLE_EXACT) return launch_sampling<FE_SAMPLE_EXACT, true>(p, s);
    if (p.sampling == FE_SAMPLE_TEXTURE_WIDE) return launch_sampling<FE_SAMPLE_TEXTURE_WIDE, true>(p, s);
    return launch_sampling<FE_SAMPLE_TEXTURE, true>(p, s);
  }
  if (p.sampling == FE_SAMPLE_EXACT) return launch_sampling<FE_SAMPLE_EXACT, false>(p, s);
  if (p.sampling == FE_SAMPLE_TEXTURE_WIDE) return launch_sampling<FE_SAMPLE_TEXTURE_WIDE, false>(p, s);
  return launch_sampling<FE_SAMPLE_TEXTURE, false>(p, s);
}

}  // namespace fe
