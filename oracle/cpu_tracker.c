/* CPU restatement of cuVSLAM's CPU tracking front-end (use_gpu = false).  TEST AND CPU-baseline
 * INFRASTRUCTURE ONLY: bench.py times it as the reference CPU arm; nothing in the product links it.
 *
 * The reference's own CPU code cannot be compiled here (it needs Eigen 3.4.1, fetched over the network
 * by its CMake), so this file restates, per camera and single-threaded like MonoSOFCPU:
 *   u8 pyramid      ImagePyramidU8::build + BasicImageDownscaler::scale
 *                   (libs/sof/image_pyramid_u8.cpp:24-57, basic_image_downscaler.cpp:26-195):
 *                   separable [1 4 6 4 1] on uint8 with (v+128)/256 rounding, mirrored edges,
 *                   d/2 sizes while both sides >= 15; levels cast to float (image_context.cpp:113-127)
 *   gradients       BasicConvolutor::convKernelGradDerivX/Y (basic_convolutor.cpp:143-185), 3-px zero
 *                   border; level 0 dense (selection forces it, selection.cpp:188-191)
 *   GFTT            GFTT::compute (sof/gftt.cpp:50-83): separable mirrored 7-tap Gaussian of gx^2,
 *                   gx*gy, gy^2 (basic_convolutor.cpp:25-141), measure 2x/(x+2) of lambda_min
 *   selection       GoodFeaturesToTrackDetector::selectFeatures (selection.cpp:211-294): 8x8 bins with
 *                   max-heaps of left-neighbour maxima, apportioned quotas, 3x3 maximum check,
 *                   9x9 burn masks, parabola refinement (selection.cpp:29-60)
 *   LK              LKFeatureTracker::trackPoint (sof/lk_tracker.cpp:81-186): exact bilinear patches
 *                   on integer boxes (image_pyramid_float.h:56-65,158-208), +1 regulariser, <= 10
 *                   iterations, |v| < 0.08 px, radius and 5x5 NCC gates; MonoSOFCPU::trackFeatures
 *                   (sof_mono_cpu.cpp:140-185) retries a failed track without prediction at NCC 0.85.
 * A frame step over many cameras runs one camera per thread (pthreads), or the cameras in turn with
 * each camera's tracking spread over threads in chunks of features (cpu_frame_step_features).
 */
#include <float.h>
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define CPU_MAX_LEVELS 10

typedef struct {
  int levels;
  int w[CPU_MAX_LEVELS], h[CPU_MAX_LEVELS];
  uint8_t* u8[CPU_MAX_LEVELS];
  float* img[CPU_MAX_LEVELS];
  float* gx[CPU_MAX_LEVELS];
  float* gy[CPU_MAX_LEVELS];
  uint16_t* buf;    /* downscaler row buffer */
  float* tmp[4];    /* GFTT scratch at level 0 */
  float* resp;      /* GFTT response */
  uint8_t* mask;    /* selection mask */
  int32_t* heap;    /* selection heaps */
} cpu_cam;

/* ---------------------------------------------------------------- pyramid */
static uint16_t binom1(int v1, int v2, int v3, int v4, int v5) { return (uint16_t)(v1 + v5 + 4 * (v2 + v4) + 6 * v3); }
static uint8_t binom2(int v1, int v2, int v3, int v4, int v5) {
  return (uint8_t)((v1 + v5 + 4 * (v2 + v4) + 6 * v3 + 128) / 256);
}

static void scale_down(const uint8_t* in, int iw, int ih, uint8_t* out, int ow, int oh, uint16_t* b) {
  for (int y = 0; y < ih; ++y) {
    const uint8_t* s = in + (size_t)iw * y;
    uint16_t* t = b + (size_t)ow * y;
    t[0] = binom1(s[1], s[0], s[0], s[1], s[2]);
    for (int x = 1; x < ow - 1; ++x) {
      const uint8_t* c = s + 2 * x;
      t[x] = binom1(c[-2], c[-1], c[0], c[1], c[2]);
    }
    const uint8_t* c = s + 2 * (ow - 1);
    t[ow - 1] = (2 * ow == iw) ? binom1(c[-2], c[-1], c[0], c[1], c[1]) : binom1(c[-2], c[-1], c[0], c[1], c[2]);
  }
  const int w = ow;
  for (int x = 0; x < w; ++x) out[x] = binom2(b[w + x], b[x], b[x], b[w + x], b[2 * w + x]);
  for (int y = 1; y < oh - 1; ++y) {
    const uint16_t* s = b + (size_t)w * 2 * y;
    uint8_t* t = out + (size_t)w * y;
    for (int x = 0; x < w; ++x) t[x] = binom2(s[x - 2 * w], s[x - w], s[x], s[x + w], s[x + 2 * w]);
  }
  const uint16_t* s = b + (size_t)w * 2 * (oh - 1);
  uint8_t* t = out + (size_t)w * (oh - 1);
  for (int x = 0; x < w; ++x)
    t[x] = (2 * oh == ih) ? binom2(s[x - 2 * w], s[x - w], s[x], s[x + w], s[x + w])
                          : binom2(s[x - 2 * w], s[x - w], s[x], s[x + w], s[x + 2 * w]);
}

static const float kDsp[7] = {112.0f / 8418.0f, 913.0f / 8418.0f, 3047.0f / 8418.0f, 0.0f,
                              -3047.0f / 8418.0f, -913.0f / 8418.0f, -112.0f / 8418.0f};

static void gradients(const float* in, int w, int h, float* gx, float* gy) {
  for (int y = 0; y < h; ++y) {
    const float* r = in + (size_t)y * w;
    float* o = gx + (size_t)y * w;
    o[0] = o[1] = o[2] = 0.f;
    for (int x = 3; x < w - 3; ++x) {
      float s = 0.f;
      for (int i = 0; i < 7; ++i) s += kDsp[i] * r[x - 3 + i];
      o[x] = s;
    }
    o[w - 3] = o[w - 2] = o[w - 1] = 0.f;
  }
  memset(gy, 0, sizeof(float) * (size_t)w * 3);
  memset(gy + (size_t)(h - 3) * w, 0, sizeof(float) * (size_t)w * 3);
  for (int y = 3; y < h - 3; ++y) {
    float* o = gy + (size_t)y * w;
    for (int x = 0; x < w; ++x) {
      float s = 0.f;
      for (int i = 0; i < 7; ++i) s += kDsp[i] * in[(size_t)(y - 3 + i) * w + x];
      o[x] = s;
    }
  }
}

cpu_cam* cpu_cam_create(int w, int h) {
  cpu_cam* c = (cpu_cam*)calloc(1, sizeof(cpu_cam));
  int n = 0;
  int lw = w, lh = h;
  while (n < CPU_MAX_LEVELS) {
    c->w[n] = lw;
    c->h[n] = lh;
    ++n;
    lw /= 2;
    lh /= 2;
    if (lw < 15 || lh < 15) break;
  }
  c->levels = n;
  for (int l = 0; l < n; ++l) {
    size_t px = (size_t)c->w[l] * c->h[l];
    c->u8[l] = (uint8_t*)malloc(px);
    c->img[l] = (float*)malloc(px * 4);
    c->gx[l] = (float*)malloc(px * 4);
    c->gy[l] = (float*)malloc(px * 4);
  }
  c->buf = (uint16_t*)malloc(sizeof(uint16_t) * (size_t)w * h);
  for (int i = 0; i < 4; ++i) c->tmp[i] = (float*)malloc(sizeof(float) * (size_t)w * h);
  c->resp = (float*)malloc(sizeof(float) * (size_t)w * h);
  c->mask = (uint8_t*)malloc((size_t)w * h);
  c->heap = (int32_t*)malloc(sizeof(int32_t) * (size_t)w * h);
  return c;
}

void cpu_cam_destroy(cpu_cam* c) {
  if (!c) return;
  for (int l = 0; l < c->levels; ++l) {
    free(c->u8[l]);
    free(c->img[l]);
    free(c->gx[l]);
    free(c->gy[l]);
  }
  free(c->buf);
  for (int i = 0; i < 4; ++i) free(c->tmp[i]);
  free(c->resp);
  free(c->mask);
  free(c->heap);
  free(c);
}

/* BoxBlur3Cpu (sof/box_blur.cpp:25-55): interior pixels get the [1 2 1] x [1 2 1] / 16 window sum,
 * truncated to uint8 (the sum of exact float products is exact, so it is the integer sum >> 4); the
 * one-pixel border keeps the input. */
static void box_blur3(const uint8_t* in, int w, int h, uint8_t* out) {
  for (int y = 1; y < h - 1; ++y)
    for (int x = 1; x < w - 1; ++x) {
      const uint8_t* r0 = in + (size_t)(y - 1) * w + x;
      const uint8_t* r1 = r0 + w;
      const uint8_t* r2 = r1 + w;
      const int s = r0[-1] + 2 * r0[0] + r0[1] + 2 * (r1[-1] + 2 * r1[0] + r1[1]) + r2[-1] + 2 * r2[0] + r2[1];
      out[(size_t)y * w + x] = (uint8_t)(s >> 4);
    }
  for (int x = 0; x < w; ++x) {
    out[x] = in[x];
    out[(size_t)(h - 1) * w + x] = in[(size_t)(h - 1) * w + x];
  }
  for (int y = 1; y < h - 1; ++y) {
    out[(size_t)y * w] = in[(size_t)y * w];
    out[(size_t)y * w + w - 1] = in[(size_t)y * w + w - 1];
  }
}

/* ImagePyramidU8::build (image_pyramid_u8.cpp:24-57) with blur_filter = box3, then the levels cast
 * to float and their gradients. */
void cpu_cam_build_ex(cpu_cam* c, const uint8_t* image, int box3) {
  if (box3)
    box_blur3(image, c->w[0], c->h[0], c->u8[0]);
  else
    memcpy(c->u8[0], image, (size_t)c->w[0] * c->h[0]);
  for (int l = 1; l < c->levels; ++l)
    scale_down(c->u8[l - 1], c->w[l - 1], c->h[l - 1], c->u8[l], c->w[l], c->h[l], c->buf);
  for (int l = 0; l < c->levels; ++l) {
    size_t px = (size_t)c->w[l] * c->h[l];
    for (size_t i = 0; i < px; ++i) c->img[l][i] = (float)c->u8[l][i];
    gradients(c->img[l], c->w[l], c->h[l], c->gx[l], c->gy[l]);
  }
}

void cpu_cam_build(cpu_cam* c, const uint8_t* image) { cpu_cam_build_ex(c, image, 0); }

int cpu_cam_levels(const cpu_cam* c) { return c->levels; }

/* computePatch (image_pyramid_float.h:158-208) of a 9x9 patch at (x, y) on level l's image; 0 when
 * its integer box leaves the level. */
int cpu_cam_patch(const cpu_cam* c, int l, float x, float y, float* out);

void cpu_cam_level(const cpu_cam* c, int l, int* w, int* h, float* img, float* gx, float* gy) {
  *w = c->w[l];
  *h = c->h[l];
  size_t px = (size_t)c->w[l] * c->h[l];
  if (img) memcpy(img, c->img[l], px * 4);
  if (gx) memcpy(gx, c->gx[l], px * 4);
  if (gy) memcpy(gy, c->gy[l], px * 4);
}

/* ---------------------------------------------------------------- GFTT */
static const float kG7[4] = {0.00598f, 0.060626f, 0.241843f, 0.383103f};

static float conv7(float v0, float v1, float v2, float v3, float v4, float v5, float v6) {
  return kG7[0] * (v0 + v6) + kG7[1] * (v1 + v5) + kG7[2] * (v2 + v4) + kG7[3] * v3;
}

static void conv_w(int w, int h, const float* in, float* out) {
  for (int y = 0; y < h; ++y) {
    const float* s = in + (size_t)w * y;
    float* t = out + (size_t)w * y;
    t[0] = conv7(s[3], s[2], s[1], s[0], s[1], s[2], s[3]);
    t[1] = conv7(s[1], s[0], s[0], s[1], s[2], s[3], s[4]);
    t[2] = conv7(s[0], s[0], s[1], s[2], s[3], s[4], s[5]);
    for (int x = 3; x < w - 3; ++x) t[x] = conv7(s[x - 3], s[x - 2], s[x - 1], s[x], s[x + 1], s[x + 2], s[x + 3]);
    int x = w - 3;
    t[x] = conv7(s[x - 3], s[x - 2], s[x - 1], s[x], s[x + 1], s[x + 2], s[x + 2]);
    x = w - 2;
    t[x] = conv7(s[x - 3], s[x - 2], s[x - 1], s[x], s[x + 1], s[x + 1], s[x]);
    x = w - 1;
    t[x] = conv7(s[x - 3], s[x - 2], s[x - 1], s[x], s[x], s[x - 1], s[x - 2]);
  }
}

static void conv_h(int w, int h, const float* in, float* out) {
#define R(y) (in + (size_t)(y) * w)
  for (int x = 0; x < w; ++x) {
    out[x] = conv7(R(2)[x], R(1)[x], R(0)[x], R(0)[x], R(1)[x], R(2)[x], R(3)[x]);
    out[w + x] = conv7(R(1)[x], R(0)[x], R(0)[x], R(1)[x], R(2)[x], R(3)[x], R(4)[x]);
    out[2 * (size_t)w + x] = conv7(R(0)[x], R(0)[x], R(1)[x], R(2)[x], R(3)[x], R(4)[x], R(5)[x]);
  }
  for (int y = 3; y < h - 3; ++y) {
    const float *a = R(y - 3), *b = R(y - 2), *c = R(y - 1), *d = R(y), *e = R(y + 1), *f = R(y + 2), *g = R(y + 3);
    float* t = out + (size_t)w * y;
    for (int x = 0; x < w; ++x) t[x] = conv7(a[x], b[x], c[x], d[x], e[x], f[x], g[x]);
  }
  int y = h - 3;
  for (int x = 0; x < w; ++x)
    out[(size_t)y * w + x] = conv7(R(y - 3)[x], R(y - 2)[x], R(y - 1)[x], R(y)[x], R(y + 1)[x], R(y + 2)[x], R(y + 2)[x]);
  y = h - 2;
  for (int x = 0; x < w; ++x)
    out[(size_t)y * w + x] = conv7(R(y - 3)[x], R(y - 2)[x], R(y - 1)[x], R(y)[x], R(y + 1)[x], R(y + 1)[x], R(y)[x]);
  y = h - 1;
  for (int x = 0; x < w; ++x)
    out[(size_t)y * w + x] = conv7(R(y - 3)[x], R(y - 2)[x], R(y - 1)[x], R(y)[x], R(y)[x], R(y - 1)[x], R(y - 2)[x]);
#undef R
}

static void gftt(cpu_cam* c) {
  const int w = c->w[0], h = c->h[0];
  const size_t px = (size_t)w * h;
  const float *gx = c->gx[0], *gy = c->gy[0];
  float *xy = c->tmp[0], *xx = c->tmp[1], *yy = c->tmp[2], *t = c->tmp[3];
  for (size_t i = 0; i < px; ++i) t[i] = gx[i] * gy[i];
  conv_w(w, h, t, c->resp);
  conv_h(w, h, c->resp, xy);
  for (size_t i = 0; i < px; ++i) t[i] = gx[i] * gx[i];
  conv_w(w, h, t, c->resp);
  conv_h(w, h, c->resp, xx);
  for (size_t i = 0; i < px; ++i) t[i] = gy[i] * gy[i];
  conv_w(w, h, t, c->resp);
  conv_h(w, h, c->resp, yy);
  for (size_t i = 0; i < px; ++i) {
    const float d = xx[i] - yy[i];
    const float D = sqrtf(d * d + 4.f * xy[i] * xy[i]);
    const float e = (xx[i] + yy[i] - D) / 2.f;
    c->resp[i] = 2 * e / (e + 2);
  }
}

/* ---------------------------------------------------------------- selection */
static float find_min_1d(float y1, float y2, float y3) {
  const float k = y1 - 2 * y2 + y3;
  const float m = fabsf(k) <= 10 * FLT_EPSILON ? 0 : 0.5f * (y1 - y3) / k;
  return m >= 0.5f ? 0.5f : (m <= -0.5f ? -0.5f : m);
}

static void heap_sift_down(int32_t* hp, int n, int i, const float* v) {
  for (;;) {
    int l = 2 * i + 1, r = l + 1, m = i;
    if (l < n && v[hp[l]] > v[hp[m]]) m = l;
    if (r < n && v[hp[r]] > v[hp[m]]) m = r;
    if (m == i) return;
    int32_t t = hp[i];
    hp[i] = hp[m];
    hp[m] = t;
    i = m;
  }
}

static void burn(uint8_t* mask, int w, int h, int x, int y, int half) {
  int r0 = y - half < 0 ? 0 : y - half, c0 = x - half < 0 ? 0 : x - half;
  int r1 = y + half > h - 1 ? h - 1 : y + half, c1 = x + half > w - 1 ? w - 1 : x + half;
  for (int r = r0; r <= r1; ++r) memset(mask + (size_t)r * w + c0, 1, (size_t)(c1 - c0 + 1));
}

static int is_max3x3(const float* s, int w, int h, int x, int y) {
  float m = -INFINITY;
  for (int r = (y > 0 ? y - 1 : 0); r <= (y < h - 1 ? y + 1 : h - 1); ++r)
    for (int q = (x > 0 ? x - 1 : 0); q <= (x < w - 1 ? x + 1 : w - 1); ++q)
      if (s[(size_t)r * w + q] > m) m = s[(size_t)r * w + q];
  return m == s[(size_t)y * w + x];
}

int cpu_cam_select(cpu_cam* c, const float* alive_xy, int n_alive, int num_desired, int bt, int bb, int bl, int br,
                   float* out_xy) {
  gftt(c);
  const int w = c->w[0], h = c->h[0];
  const float* s = c->resp;
  memset(c->mask, 0, (size_t)w * h);
  for (int r = 0; r < bt; ++r) memset(c->mask + (size_t)r * w, 1, (size_t)w);
  for (int r = h - 1 - bb; r < h - 1; ++r) memset(c->mask + (size_t)r * w, 1, (size_t)w);
  for (int r = 0; r < h; ++r) {
    memset(c->mask + (size_t)r * w, 1, (size_t)bl);
    memset(c->mask + (size_t)r * w + (w - 1 - br), 1, (size_t)br);
  }
  for (int i = 0; i < n_alive; ++i) burn(c->mask, w, h, (int)(size_t)alive_xy[2 * i], (int)(size_t)alive_xy[2 * i + 1], 4);
  const int bh = h / 8, bw = w / 8;
  float acc[64], sum = 0.f;
  int start[65];
  int n = 0;
  for (int by = 0; by < 8; ++by) {
    for (int bx = 0; bx < 8; ++bx) {
      const int b = by * 8 + bx;
      start[b] = n;
      float a = 0.f;
      for (int y = by * bh; y < by * bh + bh; ++y) {
        float prev = 0.f;
        for (int x = bx * bw; x < bx * bw + bw; ++x) {
          const float v = s[(size_t)y * w + x];
          a += v;
          if (v >= prev) c->heap[n++] = y * w + x;
          prev = v;
        }
      }
      acc[b] = a;
      /* heapify this bin */
      const int m = n - start[b];
      for (int i = m / 2 - 1; i >= 0; --i) heap_sift_down(c->heap + start[b], m, i, s);
    }
  }
  start[64] = n;
  for (int b = 0; b < 64; ++b) sum += acc[b];
  const size_t expected = (size_t)n_alive + (size_t)num_desired;
  int out = 0;
  for (int b = 0; b < 64; ++b) {
    const int bx = b % 8, by = b / 8;
    size_t prev_cnt = 0;
    for (int i = 0; i < n_alive; ++i) {
      const float x = alive_xy[2 * i], y = alive_xy[2 * i + 1];
      if (bx * bw <= x && x <= bx * bw + bw && by * bh <= y && y <= by * bh + bh) ++prev_cnt;
    }
    if (sum == 0) continue;
    const size_t e = (size_t)roundf((float)expected * acc[b] / sum);
    const size_t want = e > prev_cnt ? e - prev_cnt : 0;
    int32_t* hp = c->heap + start[b];
    int m = start[b + 1] - start[b];
    size_t added = 0;
    while (m > 0 && added < want) {
      const int32_t idx = hp[0];
      hp[0] = hp[m - 1];
      --m;
      heap_sift_down(hp, m, 0, s);
      const int x = idx % w, y = idx / w;
      if (c->mask[idx] || !is_max3x3(s, w, h, x, y)) continue;
      if (out >= num_desired) return out;
      float rx = (float)x, ry = (float)y;
      if (!(x == 0 || x == w - 1 || y == 0 || y == h - 1)) {
        rx = x + find_min_1d(s[(size_t)y * w + x - 1], s[idx], s[(size_t)y * w + x + 1]);
        ry = y + find_min_1d(s[(size_t)(y - 1) * w + x], s[idx], s[(size_t)(y + 1) * w + x]);
      }
      out_xy[2 * out] = rx;
      out_xy[2 * out + 1] = ry;
      ++out;
      burn(c->mask, w, h, x, y, 4);
      ++added;
    }
  }
  return out;
}

/* ---------------------------------------------------------------- LK */
static const float kG9[9] = {0.0135196f, 0.0476622f, 0.11723f, 0.201168f, 0.240841f,
                             0.201168f,  0.11723f,   0.0476622f, 0.0135196f};

/* computePatch (image_pyramid_float.h:158-208): 9x9 exact-bilinear patch on the integer box. */
static int patch(const float* img, int w, int h, float x, float y, float* out) {
  const float x0 = x - 0.5f, y0 = y - 0.5f;
  const int ix = (int)x0, iy = (int)y0;
  const int tlx = ix - 4, tly = iy - 4;
  if (tlx < 0 || tlx + 10 >= w || tly < 0 || tly + 10 >= h) return 0;
  const float dx = x0 - (float)ix, dy = y0 - (float)iy;
  if (!(dx >= 0 && dy >= 0 && dx <= 1 && dy <= 1)) return 0;
  const float k0 = (1.f - dx) * (1.f - dy), k1 = dx * (1.f - dy), k2 = (1.f - dx) * dy, k3 = dx * dy;
  for (int r = 0; r < 9; ++r) {
    const float* s = img + (size_t)(tly + r) * w + tlx;
    for (int q = 0; q < 9; ++q) out[r * 9 + q] = k0 * s[q] + k1 * s[q + 1] + k2 * s[q + w] + k3 * s[q + w + 1];
  }
  return 1;
}

int cpu_cam_patch(const cpu_cam* c, int l, float x, float y, float* out) {
  if (l < 0 || l >= c->levels) return 0;
  return patch(c->img[l], c->w[l], c->h[l], x, y, out);
}

static int lk_point(const cpu_cam* P, const cpu_cam* C, float tx, float ty, float ox, float oy, float radius,
                    float ncc_thr, float* out_x, float* out_y) {
  if (radius < 0.f) return 0;
  const int levels = P->levels, top = levels - 1;
  if (!(tx >= 0 && tx < P->w[0] && ty >= 0 && ty < P->h[0])) return 0;
  if (!(tx + ox >= 0 && tx + ox < C->w[0] && ty + oy >= 0 && ty + oy < C->h[0])) return 0;
  const float scale = 1.f / (float)(1 << top);
  float x1 = (tx - 0.5f) * scale + 0.5f, y1 = (ty - 0.5f) * scale + 0.5f;
  float x2 = (tx + ox - 0.5f) * scale + 0.5f, y2 = (ty + oy - 0.5f) * scale + 0.5f;
  int conv = 0;
  float gxp[81], gyp[81], p1[81], p2[81], wt[81];
  for (int i = 0; i < 81; ++i) wt[i] = kG9[i / 9] * kG9[i % 9];
  for (int i = 0; i < levels; ++i) {
    const int level = top - i;
    const int W = P->w[level], H = P->h[level];
    if (patch(P->gx[level], W, H, x1, y1, gxp) && patch(P->gy[level], W, H, x1, y1, gyp)) {
      float sx = 0, sy = 0;
      for (int k = 0; k < 81; ++k) {
        sx += gxp[k];
        sy += gyp[k];
      }
      for (int k = 0; k < 81; ++k) {
        gxp[k] -= sx / 81.f;
        gyp[k] -= sy / 81.f;
      }
      float gxx = 0, gxy = 0, gyy = 0;
      for (int k = 0; k < 81; ++k) {
        gxx += wt[k] * gxp[k] * gxp[k];
        gxy += wt[k] * gxp[k] * gyp[k];
        gyy += wt[k] * gyp[k] * gyp[k];
      }
      gxx += 1.f;
      gyy += 1.f;
      const float det = gxx * gyy - gxy * gxy;
      if (det < FLT_EPSILON) return 0;
      if (patch(P->img[level], W, H, x1, y1, p1)) {
        const float sx2 = x2, sy2 = y2;
        for (int it = 0; it < 10; ++it) {
          if (!patch(C->img[level], W, H, x2, y2, p2)) break;
          float s1 = 0, s2 = 0;
          for (int k = 0; k < 81; ++k) {
            s1 += p1[k];
            s2 += p2[k];
          }
          const float delta = (s2 - s1) / 81.f;
          float ex = 0, ey = 0;
          for (int k = 0; k < 81; ++k) {
            const float t = p2[k] - p1[k] - delta;
            ex += wt[k] * gxp[k] * t;
            ey += wt[k] * gyp[k] * t;
          }
          const float vx = (gyy * ex - gxy * ey) / det, vy = (gxx * ey - gxy * ex) / det;
          conv = sqrtf(vx * vx + vy * vy) < 0.08f;
          if (conv) break;
          x2 += vx;
          y2 += vy;
        }
        if (conv) {
          const float r = radius / (float)(1 << level);
          if (sqrtf((x2 - sx2) * (x2 - sx2) + (y2 - sy2) * (y2 - sy2)) > r) conv = 0;
        }
        int ncc_ok = 0;
        if (conv) {
          float a = 0, b = 0, aa = 0, bb = 0, ab = 0;
          for (int r = 2; r < 7; ++r)
            for (int q = 2; q < 7; ++q) {
              const float u = p1[r * 9 + q], v = p2[r * 9 + q];
              a += u;
              b += v;
              aa += u * u;
              bb += v * v;
              ab += u * v;
            }
          const float a1 = a / 25.f, a2 = b / 25.f;
          const float d1 = aa / 25.f - a1 * a1, d2 = bb / 25.f - a2 * a2, d12 = ab / 25.f - a1 * a2;
          const float d1d2 = d1 * d2;
          const float ncc = d1d2 < FLT_EPSILON ? 0.f : d12 / sqrtf(d1d2);
          ncc_ok = ncc > ncc_thr;
        }
        if (!ncc_ok && level > 0) {
          x2 = sx2;
          y2 = sy2;
        }
        conv = level == 0 && ncc_ok;
      }
    }
    if (i != levels - 1) {
      x1 = x1 * 2.f - 0.5f;
      y1 = y1 * 2.f - 0.5f;
      x2 = x2 * 2.f - 0.5f;
      y2 = y2 * 2.f - 0.5f;
    }
  }
  if (conv) {
    *out_x = x2;
    *out_y = y2;
  }
  return conv;
}

/* MonoSOFCPU::trackFeatures: predicted attempt at NCC 0.8, retry from the old position at 0.85. */
int cpu_cam_track(const cpu_cam* prev, const cpu_cam* cur, const float* xy, const float* pred_xy, int n,
                  float* out_xy, uint8_t* status) {
  int ok = 0;
  const float radius = (float)prev->w[0];
  for (int k = 0; k < n; ++k) {
    const float x = xy[2 * k], y = xy[2 * k + 1];
    const float px = pred_xy ? pred_xy[2 * k] : x, py = pred_xy ? pred_xy[2 * k + 1] : y;
    float nx = x, ny = y;
    int r = lk_point(prev, cur, x, y, px - x, py - y, radius, 0.8f, &nx, &ny);
    if (!r) r = lk_point(prev, cur, x, y, 0.f, 0.f, radius, 0.85f, &nx, &ny);
    out_xy[2 * k] = nx;
    out_xy[2 * k + 1] = ny;
    status[k] = (uint8_t)r;
    ok += r;
  }
  return ok;
}

/* The same over the features on nthreads threads: chunks of 16 features taken from a shared
 * counter (a dynamic schedule; each feature's attempts are independent, the pyramids only read). */
typedef struct {
  const cpu_cam *prev, *cur;
  const float *xy, *pred;
  int n;
  float* out;
  uint8_t* status;
  int next, ok;
  pthread_mutex_t lock;
} track_job;

static void* track_worker(void* arg) {
  track_job* j = (track_job*)arg;
  const float radius = (float)j->prev->w[0];
  int ok = 0;
  for (;;) {
    pthread_mutex_lock(&j->lock);
    const int b = j->next;
    j->next += 16;
    pthread_mutex_unlock(&j->lock);
    if (b >= j->n) break;
    const int e = b + 16 < j->n ? b + 16 : j->n;
    for (int k = b; k < e; ++k) {
      const float x = j->xy[2 * k], y = j->xy[2 * k + 1];
      const float px = j->pred ? j->pred[2 * k] : x, py = j->pred ? j->pred[2 * k + 1] : y;
      float nx = x, ny = y;
      int r = lk_point(j->prev, j->cur, x, y, px - x, py - y, radius, 0.8f, &nx, &ny);
      if (!r) r = lk_point(j->prev, j->cur, x, y, 0.f, 0.f, radius, 0.85f, &nx, &ny);
      j->out[2 * k] = nx;
      j->out[2 * k + 1] = ny;
      j->status[k] = (uint8_t)r;
      ok += r;
    }
  }
  pthread_mutex_lock(&j->lock);
  j->ok += ok;
  pthread_mutex_unlock(&j->lock);
  return NULL;
}

int cpu_cam_track_par(const cpu_cam* prev, const cpu_cam* cur, const float* xy, const float* pred_xy, int n,
                      float* out_xy, uint8_t* status, int nthreads) {
  if (nthreads <= 1) return cpu_cam_track(prev, cur, xy, pred_xy, n, out_xy, status);
  track_job j = {prev, cur, xy, pred_xy, n, out_xy, status, 0, 0};
  pthread_mutex_init(&j.lock, NULL);
  pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * (size_t)nthreads);
  for (int t = 0; t < nthreads; ++t) pthread_create(&th[t], NULL, track_worker, &j);
  for (int t = 0; t < nthreads; ++t) pthread_join(th[t], NULL);
  free(th);
  pthread_mutex_destroy(&j.lock);
  return j.ok;
}

/* ---------------------------------------------------------------- multi-camera frame step */
typedef struct {
  cpu_cam** prev;
  cpu_cam** cur;
  const uint8_t** images;
  const float** xy;
  const float** pred;
  const int* n;
  const int* num_desired;
  float** out_xy;
  uint8_t** status;
  float** new_xy;
  int* new_n;
  int ncams;
  int next;
  pthread_mutex_t lock;
} frame_job;

static void* frame_worker(void* arg) {
  frame_job* j = (frame_job*)arg;
  for (;;) {
    pthread_mutex_lock(&j->lock);
    const int i = j->next++;
    pthread_mutex_unlock(&j->lock);
    if (i >= j->ncams) return NULL;
    cpu_cam_build(j->cur[i], j->images[i]);
    int n = j->n[i];
    float* alive = (float*)malloc(sizeof(float) * 2 * (size_t)(n > 0 ? n : 1));
    int na = 0;
    if (j->prev && j->prev[i] && n > 0) {
      cpu_cam_track(j->prev[i], j->cur[i], j->xy[i], j->pred ? j->pred[i] : NULL, n, j->out_xy[i], j->status[i]);
      for (int k = 0; k < n; ++k)
        if (j->status[i][k]) {
          alive[2 * na] = j->out_xy[i][2 * k];
          alive[2 * na + 1] = j->out_xy[i][2 * k + 1];
          ++na;
        }
    }
    j->new_n[i] = j->num_desired[i] > 0 ? cpu_cam_select(j->cur[i], alive, na, j->num_desired[i], 0, 0, 0, 0, j->new_xy[i]) : 0;
    free(alive);
  }
}

/* The features-parallel variant of a frame step: the cameras one after another, each camera's
 * tracking spread over nthreads threads (pyramid build and selection stay single-threaded, as in
 * MonoSOFCPU). */
int cpu_frame_step_features(cpu_cam** prev, cpu_cam** cur, const uint8_t** images, const float** xy, const float** pred,
                       const int* n, const int* num_desired, float** out_xy, uint8_t** status, float** new_xy,
                       int* new_n, int ncams, int nthreads) {
  for (int i = 0; i < ncams; ++i) {
    cpu_cam_build(cur[i], images[i]);
    const int m = n[i];
    float* alive = (float*)malloc(sizeof(float) * 2 * (size_t)(m > 0 ? m : 1));
    int na = 0;
    if (prev && prev[i] && m > 0) {
      cpu_cam_track_par(prev[i], cur[i], xy[i], pred ? pred[i] : NULL, m, out_xy[i], status[i], nthreads);
      for (int k = 0; k < m; ++k)
        if (status[i][k]) {
          alive[2 * na] = out_xy[i][2 * k];
          alive[2 * na + 1] = out_xy[i][2 * k + 1];
          ++na;
        }
    }
    new_n[i] = num_desired[i] > 0 ? cpu_cam_select(cur[i], alive, na, num_desired[i], 0, 0, 0, 0, new_xy[i]) : 0;
    free(alive);
  }
  return 0;
}

/* One frame step of `ncams` cameras on `nthreads` threads (one camera per thread at a time):
 * build the current pyramids, track each camera's points from its previous pyramid, select new
 * features with the survivors as alive tracks. */
int cpu_frame_step(cpu_cam** prev, cpu_cam** cur, const uint8_t** images, const float** xy, const float** pred,
                   const int* n, const int* num_desired, float** out_xy, uint8_t** status, float** new_xy, int* new_n,
                   int ncams, int nthreads) {
  frame_job j = {prev, cur, images, xy, pred, n, num_desired, out_xy, status, new_xy, new_n, ncams, 0};
  pthread_mutex_init(&j.lock, NULL);
  if (nthreads < 1) nthreads = 1;
  pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * (size_t)nthreads);
  for (int t = 0; t < nthreads; ++t) pthread_create(&th[t], NULL, frame_worker, &j);
  for (int t = 0; t < nthreads; ++t) pthread_join(th[t], NULL);
  free(th);
  pthread_mutex_destroy(&j.lock);
  return 0;
}
