/* CPU oracle, reference-GPU semantics.  TEST INFRASTRUCTURE ONLY (see fe_oracle.h).
 *
 * Compiled with -ffp-contract=off: every fused multiply-add that the reference's nvcc build
 * contracts is written here as an explicit fmaf(), so the evaluation order is pinned.
 * Citations are to cuVSLAM (VERSION 18.0.0) paths under libs/.
 */
#include "fe_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define MIN_DIM 15
#define MAX_LEVELS 10

/* ------------------------------------------------------------------------------------------ */
/* Pyramid                                                                                      */
/* ------------------------------------------------------------------------------------------ */

/* GPUImagePyramid::prepare_levels (cuda_modules/image_pyramid.h:136-151), ScaleDownDim
 * (cuda_modules/image_pyramid.cpp:24): (d+1)/2 while both sides stay >= 15. */
int or_level_sizes(int w, int h, int max_levels, int* ws, int* hs) {
  int n = 0;
  if (max_levels > MAX_LEVELS) max_levels = MAX_LEVELS;
  while (n < max_levels) {
    ws[n] = w;
    hs[n] = h;
    ++n;
    w = (w + 1) / 2;
    h = (h + 1) / 2;
    if (w < MIN_DIM || h < MIN_DIM) break;
  }
  return n;
}

/* cast_image_kernel (cuda_kernels/image_cast.cu:24-36). */
void or_cast_u8(const uint8_t* src, int w, int h, float* dst) {
  for (size_t i = 0; i < (size_t)w * h; ++i) dst[i] = (float)src[i];
}

/* cast_image_kernel_rgb (cuda_kernels/image_cast.cu:52-70): gray = 0.299 r + 0.587 g + 0.114 b in
 * FP32.  nvcc contracts the expression into fused multiply-adds; `variant` names the contraction:
 *   0: no fusion   ((0.299 r + 0.587 g) + 0.114 b), each product and sum rounded
 *   1: fma(0.114, b, fma(0.587, g, 0.299 r))
 *   2: fma(0.114, b, fma(0.299, r, 0.587 g))
 *   3: fma(0.587, g, 0.299 r) + 0.114 b
 *   4: fma(0.299, r, 0.587 g) + 0.114 b
 * (the tests pin which one the reference kernel computes against its own outputs). */
void or_rgb_to_gray(const uint8_t* rgb, int w, int h, int64_t pitch, float* dst, int variant) {
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      const uint8_t* p = rgb + (size_t)y * pitch + 3 * (size_t)x;
      const float r = (float)p[0], g = (float)p[1], b = (float)p[2];
      const float pr = 0.299f * r, pg = 0.587f * g, pb = 0.114f * b;
      float v;
      switch (variant) {
        case 1: v = fmaf(0.114f, b, fmaf(0.587f, g, pr)); break;
        case 2: v = fmaf(0.114f, b, fmaf(0.299f, r, pg)); break;
        case 3: v = fmaf(0.587f, g, pr) + pb; break;
        case 4: v = fmaf(0.299f, r, pg) + pb; break;
        default: v = (pr + pg) + pb; break;
      }
      dst[(size_t)y * w + x] = v;
    }
}

/* CudaBoxPrefilter::prefilter (cuda_modules/box_prefilter.cpp:31-38): box_blur_x_kernel, then
 * box_blur_y_kernel on its output, then copy_border_kernel with border 1 (convolutions.cu:141-220).
 * x pass: 0.25 v[x-1] + 0.5 v[x] + 0.25 v[x+1], 0 in columns 0 and w-1; y pass: the same down the
 * x pass's columns, 0 in rows 0 and h-1, then truncated to an integer (the kernel stores
 * (uint8_t)v); finally the one-pixel border ring is the input itself.  The weights are powers of
 * two, so each product is exact and each sum rounds once whether or not it is fused. */
void or_box3(const float* src, int w, int h, float* dst) {
  float* xb = (float*)malloc(sizeof(float) * (size_t)w * h);
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      float v = 0.f;
      if (x > 0 && x < w - 1) {
        const float* r = src + (size_t)y * w + x;
        v = 0.25f * r[-1];
        v = fmaf(0.5f, r[0], v);
        v = fmaf(0.25f, r[1], v);
      }
      xb[(size_t)y * w + x] = v;
    }
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      float v;
      if (x == 0 || x == w - 1 || y == 0 || y == h - 1) {
        v = src[(size_t)y * w + x];
      } else {
        const float* c = xb + (size_t)y * w + x;
        float s = 0.25f * c[-w];
        s = fmaf(0.5f, c[0], s);
        s = fmaf(0.25f, c[w], s);
        v = (float)(uint8_t)s;
      }
      dst[(size_t)y * w + x] = v;
    }
  free(xb);
}

/* gaussian_scaling_kernel (cuda_kernels/image_pyramid.cu:56-102): 5x5 [1 4 6 4 1]^T[1 4 6 4 1]/256
 * evaluated at even source coordinates, taps visited row-major and accumulated with FMA, mirror
 * addressing -x-1 / 2n-x-1, and the taps whose row AND column both fall outside are skipped. */
void or_gauss_downscale(const float* src, int sw, int sh, float* dst, int dw, int dh) {
  static const float k1[5] = {1.f / 16.f, 4.f / 16.f, 6.f / 16.f, 4.f / 16.f, 1.f / 16.f};
  float k2[25];
  for (int i = 0; i < 5; ++i)
    for (int j = 0; j < 5; ++j) k2[i * 5 + j] = k1[i] * k1[j];
  for (int y = 0; y < dh; ++y) {
    for (int x = 0; x < dw; ++x) {
      float acc = 0.f;
      for (int k = 0; k < 5; ++k) {
        for (int l = 0; l < 5; ++l) {
          int xc = 2 * x - 2 + l, yc = 2 * y - 2 + k;
          int xo = xc < 0 || xc >= sw, yo = yc < 0 || yc >= sh;
          if (xo && yo) continue;
          xc = xc < 0 ? -xc - 1 : xc;
          xc = xc >= sw ? 2 * sw - xc - 1 : xc;
          yc = yc < 0 ? -yc - 1 : yc;
          yc = yc >= sh ? 2 * sh - yc - 1 : yc;
          acc = fmaf(k2[k * 5 + l], src[(size_t)yc * sw + xc], acc);
        }
      }
      dst[(size_t)y * dw + x] = acc;
    }
  }
}

/* conv_grad_x_kernel / conv_grad_y_kernel (cuda_kernels/convolutions.cu:74-139): 7-tap DSP
 * derivative [112 913 3047 0 -3047 -913 -112]/8418 accumulated j = -3..3 with FMA; results within
 * 3 px of the border (x <= 2 or x >= w-3, resp. y) are zero. */
static const float kDsp[7] = {112.0f / 8418.0f, 913.0f / 8418.0f, 3047.0f / 8418.0f, 0.0f,
                              -3047.0f / 8418.0f, -913.0f / 8418.0f, -112.0f / 8418.0f};

void or_gradients(const float* in, int w, int h, float* gx, float* gy) {
  for (int y = 0; y < h; ++y) {
    for (int x = 0; x < w; ++x) {
      float sx = 0.f, sy = 0.f;
      if (x > 2 && x < w - 3) {
        for (int j = 0; j < 7; ++j) sx = fmaf(kDsp[j], in[(size_t)y * w + x - 3 + j], sx);
      }
      if (y > 2 && y < h - 3) {
        for (int j = 0; j < 7; ++j) sy = fmaf(kDsp[j], in[(size_t)(y - 3 + j) * w + x], sy);
      }
      gx[(size_t)y * w + x] = sx;
      gy[(size_t)y * w + x] = sy;
    }
  }
}

/* ------------------------------------------------------------------------------------------ */
/* Shi-Tomasi response                                                                          */
/* ------------------------------------------------------------------------------------------ */

static const float kGauss7[7] = {0.00598f, 0.060626f, 0.241843f, 0.383103f, 0.241843f, 0.060626f, 0.00598f};

static inline int mirror(int i, int n) {
  i = i >= 0 ? i : -i - 1;
  i = i < n ? i : 2 * n - i - 1;
  return i;
}

/* gftt_values_kernel (cuda_kernels/gftt.cu:80-162): separable 7-tap Gaussian of gx^2, gx*gy, gy^2
 * (horizontal pass first, taps j = 0..6, each as fma(c*g1, g2, acc); vertical pass as
 * fma(c, h, acc)), mirror addressing, then GFTTMeasure (gftt.cu:61-66):
 * log(1 + (T - sqrt((xx-yy)^2 + 4 xy^2)) / 2), where the reference build fuses the second product:
 * fma(4 xy, xy, (xx-yy)^2) (identified against the reference's outputs on a B200).  The reference
 * evaluates the log with __logf; the oracle uses logf. */
void or_gftt_response(const float* gx, const float* gy, int w, int h, float* resp) {
  float* hxx = (float*)malloc(sizeof(float) * (size_t)w * h);
  float* hxy = (float*)malloc(sizeof(float) * (size_t)w * h);
  float* hyy = (float*)malloc(sizeof(float) * (size_t)w * h);
  for (int y = 0; y < h; ++y) {
    for (int x = 0; x < w; ++x) {
      float xx = 0.f, xy = 0.f, yy = 0.f;
      for (int j = 0; j < 7; ++j) {
        int xc = mirror(x - 3 + j, w);
        float a = gx[(size_t)y * w + xc], b = gy[(size_t)y * w + xc];
        float ca = kGauss7[j] * a, cb = kGauss7[j] * b;
        xx = fmaf(ca, a, xx);
        xy = fmaf(ca, b, xy);
        yy = fmaf(cb, b, yy);
      }
      hxx[(size_t)y * w + x] = xx;
      hxy[(size_t)y * w + x] = xy;
      hyy[(size_t)y * w + x] = yy;
    }
  }
  for (int y = 0; y < h; ++y) {
    for (int x = 0; x < w; ++x) {
      float xx = 0.f, xy = 0.f, yy = 0.f;
      for (int i = 0; i < 7; ++i) {
        size_t o = (size_t)mirror(y - 3 + i, h) * w + x;
        xx = fmaf(kGauss7[i], hxx[o], xx);
        xy = fmaf(kGauss7[i], hxy[o], xy);
        yy = fmaf(kGauss7[i], hyy[o], yy);
      }
      float d = xx - yy;
      float D = sqrtf(fmaf(4.f * xy, xy, d * d));
      float T = xx + yy;
      float emin = (T - D) * 0.5f;
      resp[(size_t)y * w + x] = logf(emin + 1.f);
    }
  }
  free(hxx);
  free(hxy);
  free(hyy);
}

/* ------------------------------------------------------------------------------------------ */
/* Selection                                                                                    */
/* ------------------------------------------------------------------------------------------ */

/* xor-butterfly sum over 32 lanes, as `x += __shfl_xor_sync(.., x, m)` for m = 1..16 (lane 0's value). */
static float butterfly(float* v, int levels) {
  float t[32];
  memcpy(t, v, sizeof(t));
  for (int s = 0, m = 1; s < levels; ++s, m <<= 1) {
    float u[32];
    for (int l = 0; l < 32; ++l) u[l] = t[l] + t[l ^ m];
    memcpy(t, u, sizeof(t));
  }
  return t[0];
}

/* Per-bin strength sums.  accumulateGFTT_kernel (cuda_kernels/selection_v2.cu:39-92) sums each
 * 16x16 sub-tile (warp butterfly over 2 rows x 16 columns, then a 3-level butterfly over the 8
 * warps) and adds the sub-tile into the 8x8 bin containing its centre with a float atomicAdd, in
 * arbitrary order.  Here the order is fixed as the CUDA kernels fix it: a bin adds its sub-tiles
 * row by row (left to right), then adds the row sums top to bottom. */
void or_bins(const float* resp, int w, int h, float* bins64) {
  const int bw = w / 8, bh = h / 8;
  memset(bins64, 0, sizeof(float) * 64);
  const int tw = (w + 15) / 16, th = (h + 15) / 16;
  float* sub = (float*)malloc(sizeof(float) * (size_t)(tw > 0 ? tw : 1) * (th > 0 ? th : 1));
  for (int ty = 0; ty < th; ++ty) {
    for (int tx = 0; tx < tw; ++tx) {
      float part[32] = {0};
      for (int wp = 0; wp < 8; ++wp) {
        float lanes[32];
        for (int l = 0; l < 32; ++l) {
          int yy = ty * 16 + 2 * wp + l / 16, xx = tx * 16 + (l % 16);
          lanes[l] = (xx < w && yy < h) ? resp[(size_t)yy * w + xx] : 0.f;
        }
        part[wp] = butterfly(lanes, 5);
      }
      sub[ty * tw + tx] = butterfly(part, 3);
    }
  }
  if (bw > 0 && bh > 0) {
    for (int b = 0; b < 64; ++b) {
      const unsigned bx = (unsigned)(b & 7), by = (unsigned)(b >> 3);
      float acc = 0.f;
      for (int ty = 0; ty < th; ++ty) {
        if ((unsigned)(ty * 16 + 8) / (unsigned)bh != by) continue;
        float row = 0.f;
        for (int tx = 0; tx < tw; ++tx)
          if ((unsigned)(tx * 16 + 8) / (unsigned)bw == bx) row += sub[ty * tw + tx];
        acc += row;
      }
      bins64[b] = acc;
    }
  }
  free(sub);
}

static int rint_even(float v) { return (int)nearbyintf(v); }

/* FindMinimum1D (cuda_kernels/selection_v2.cu:279-293); the reference divides with __fdividef. */
static float find_min_1d(float y1, float y2, float y3) {
  const float k = fmaf(-2.f, y2, y1) + y3;
  const float m = fabsf(k) <= (10 * FLT_EPSILON) ? 0.f : (0.5f * (y1 - y3)) / k;
  if (m >= 0.5f) return 0.5f;
  if (m <= -0.5f) return -0.5f;
  return m;
}

typedef struct {
  float x, y, s;
  int cell;
} kp_t;

static int kp_cmp(const void* a, const void* b) {
  const kp_t* p = (const kp_t*)a;
  const kp_t* q = (const kp_t*)b;
  if (p->s > q->s) return -1;
  if (p->s < q->s) return 1;
  return p->cell - q->cell;
}

/* GPUSelection::computeGFTTAndSelectFeatures (cuda_modules/selection_v2.cpp:27-184) on a response
 * map: 3x3 NMS with clamped neighbours (non_max_suppression_kernel, selection_v2.cu:189-244), zero
 * 9x9 windows around alive tracks (filter_maximums_kernel, :251-277), per-8x8-cell max/argmax
 * (downsample_gftt_x8_kernel, :107-178, including its lane-order tie rule), keep cells above 1e-2
 * and refine by a parabola (select_features_kernel, :307-329), sort by strength descending with
 * ties broken by cell raster index (the reference's CUB sort leaves ties in atomic order), then the
 * per-bin quota and border/mask filter of the host loop (selection_v2.cpp:108-183).
 * Returns the number of selected features written to sel (x, y pairs). */
int or_select(const float* resp, int w, int h, const float* alive_xy, int n_alive, int num_desired, int border_top,
              int border_bottom, int border_left, int border_right, const uint8_t* mask, float* nms, float* cell_max,
              uint32_t* cell_idx, float* kp, int* n_kp, float* bins, float* sel) {
  /* NMS */
  for (int y = 0; y < h; ++y) {
    for (int x = 0; x < w; ++x) {
      float c = resp[(size_t)y * w + x];
      int is_max = 1;
      for (int t = 0; t < 9; ++t) {
        int i = t / 3, j = t % 3;
        if (i == 1 && j == 1) continue;
        int yy = y - 1 + i, xx = x - 1 + j;
        yy = yy < 0 ? 0 : (yy >= h ? h - 1 : yy);
        xx = xx < 0 ? 0 : (xx >= w ? w - 1 : xx);
        is_max &= resp[(size_t)yy * w + xx] <= c;
      }
      nms[(size_t)y * w + x] = is_max ? c : 0.f;
    }
  }
  /* alive tracks burn their 9x9 neighbourhood (the reference copies at most cw*ch of them) */
  const int cw = w / 8, ch = h / 8, ncell = cw * ch;
  int n_burn = n_alive < ncell ? n_alive : ncell;
  for (int k = 0; k < n_burn; ++k) {
    int x = rint_even(alive_xy[2 * k]), y = rint_even(alive_xy[2 * k + 1]);
    for (int dy = -4; dy <= 4; ++dy)
      for (int dx = -4; dx <= 4; ++dx)
        if (x + dx >= 0 && y + dy >= 0 && x + dx < w && y + dy < h) nms[(size_t)(y + dy) * w + x + dx] = 0.f;
  }
  /* cell max / argmax with the reference's lane order */
  for (int cy = 0; cy < ch; ++cy) {
    for (int cx = 0; cx < cw; ++cx) {
      float m[32];
      unsigned idx[32];
      for (int l = 0; l < 32; ++l) {
        m[l] = 0.f;
        idx[l] = 0;
        for (int e = 0; e < 2; ++e) {
          int f = l + 32 * e, dy = f / 8, dx = f % 8;
          float v = nms[(size_t)(cy * 8 + dy) * w + cx * 8 + dx];
          if (v > m[l]) {
            m[l] = v;
            idx[l] = (unsigned)dx | ((unsigned)dy << 16);
          }
        }
      }
      for (int d = 1; d < 32; d <<= 1) {
        float m2[32];
        unsigned i2[32];
        for (int l = 0; l < 32; ++l) {
          int src = l + d < 32 ? l + d : l;
          m2[l] = m[src];
          i2[l] = idx[src];
        }
        for (int l = 0; l < 32; ++l) {
          if (m2[l] > m[l]) {
            m[l] = m2[l];
            idx[l] = i2[l];
          }
        }
      }
      cell_max[cy * cw + cx] = m[0];
      cell_idx[2 * (cy * cw + cx)] = (unsigned)(cx * 8) + (idx[0] & 0xffffu);
      cell_idx[2 * (cy * cw + cx) + 1] = (unsigned)(cy * 8) + (idx[0] >> 16);
    }
  }
  /* keypoints */
  kp_t* list = (kp_t*)malloc(sizeof(kp_t) * (size_t)(ncell > 0 ? ncell : 1));
  int nk = 0;
  for (int c = 0; c < ncell; ++c) {
    float m = cell_max[c];
    if (m > (float)1e-2) {
      int x = (int)cell_idx[2 * c], y = (int)cell_idx[2 * c + 1];
      float rx = (float)x, ry = (float)y;
      if (!(x == 0 || x == w - 1 || y == 0 || y == h - 1)) {
        float g = resp[(size_t)y * w + x];
        rx = (float)x + find_min_1d(resp[(size_t)y * w + x - 1], g, resp[(size_t)y * w + x + 1]);
        ry = (float)y + find_min_1d(resp[(size_t)(y - 1) * w + x], g, resp[(size_t)(y + 1) * w + x]);
      }
      list[nk].x = rx;
      list[nk].y = ry;
      list[nk].s = m;
      list[nk].cell = c;
      ++nk;
    }
  }
  qsort(list, (size_t)nk, sizeof(kp_t), kp_cmp);
  for (int i = 0; i < nk; ++i) {
    kp[3 * i] = list[i].x;
    kp[3 * i + 1] = list[i].y;
    kp[3 * i + 2] = list[i].s;
  }
  *n_kp = nk;
  /* quota */
  or_bins(resp, w, h, bins);
  float sum = 0.f;
  for (int i = 0; i < 64; ++i) sum += bins[i];
  const float bsx = (float)(w / 8), bsy = (float)(h / 8);
  size_t prev_cnt[64] = {0}, want[64] = {0}, added[64] = {0};
  for (int i = 0; i < n_alive; ++i) {
    unsigned bx = (unsigned)(alive_xy[2 * i] / bsx), by = (unsigned)(alive_xy[2 * i + 1] / bsy);
    if (bx < 8 && by < 8) prev_cnt[by * 8 + bx]++;
  }
  const size_t expected = (size_t)n_alive + (size_t)num_desired;
  if (sum > 0.f) {
    for (int i = 0; i < 64; ++i) {
      float e = roundf((float)expected * bins[i] / sum);
      size_t ei = e > 0.f ? (size_t)e : 0;
      if (ei > prev_cnt[i]) want[i] = ei - prev_cnt[i];
    }
  }
  int n_out = 0;
  for (int i = 0; i < nk; ++i) {
    float x = list[i].x, y = list[i].y;
    if (x < (float)border_left || x > (float)(w - 1 - border_right) || y < (float)border_top ||
        y > (float)(h - 1 - border_bottom))
      continue;
    if (mask && mask[(size_t)y * w + (size_t)x] != 0) continue;
    unsigned bx = (unsigned)(x / bsx), by = (unsigned)(y / bsy);
    if (bx < 8 && by < 8) {
      unsigned b = by * 8 + bx;
      if (added[b] < want[b]) {
        added[b]++;
        if (n_out < num_desired) {
          sel[2 * n_out] = x;
          sel[2 * n_out + 1] = y;
          ++n_out;
        } else {
          break;
        }
      }
    }
  }
  free(list);
  return n_out;
}

/* ------------------------------------------------------------------------------------------ */
/* Lucas-Kanade                                                                                 */
/* ------------------------------------------------------------------------------------------ */

/* Bilinear sample at texture coordinate (x, y): texel i covers [i, i+1), so the taps are
 * floor(x - 0.5) and +1 with fraction a = (x - 0.5) - floor(x - 0.5); indices are clamped to the
 * image (unnormalised texture coordinates clamp; cuda_helper.h:419-429).
 *
 * OR_SAMPLE_TEXTURE emulates cudaFilterModeLinear.  The CUDA Programming Guide ("Texture
 * Fetching") states that the weights carry 8 fractional bits; the exact rule below was measured on
 * a B200 against hardware tex2D (tests/golden/reference.npz, entries tex/sweep and tex/random):
 *   A = floor(256 a + 1/2), B = floor(256 b + 1/2)                      (fractions, round half up)
 *   P00 = (256-A)(256-B), P10 = A(256-B), P01 = (256-A)B, P11 = AB      (exact products, /65536)
 *   W00 = round_half_up(P00/256), W11 = round_half_up(P11/256),
 *   W10 = round_half_down(P10/256), W01 = round_half_down(P01/256)      (so the W sum to 256)
 *   value = sum W_ij t_ij / 256
 * The hardware's final accumulation is not restated bit-for-bit (it differs from an exact sum by
 * at most a few ulp); the sum here is the FP32 FMA chain the CUDA kernel uses. */
static void tex_weights(float frac_x, float frac_y, float w4[4]) {
  int A = (int)floorf(frac_x * 256.f + 0.5f), B = (int)floorf(frac_y * 256.f + 0.5f);
  int p00 = (256 - A) * (256 - B), p10 = A * (256 - B), p01 = (256 - A) * B, p11 = A * B;
  w4[0] = (float)((p00 + 128) >> 8) * (1.f / 256.f);
  w4[1] = (float)((p10 + 127) >> 8) * (1.f / 256.f);
  w4[2] = (float)((p01 + 127) >> 8) * (1.f / 256.f);
  w4[3] = (float)((p11 + 128) >> 8) * (1.f / 256.f);
}

float or_tex_sample(const float* img, int w, int h, float x, float y, int mode) {
  float xb = x - 0.5f, yb = y - 0.5f;
  float fx = floorf(xb), fy = floorf(yb);
  float a = xb - fx, b = yb - fy;
  int i0 = (int)fx, j0 = (int)fy;
  int i1 = i0 + 1, j1 = j0 + 1;
  i0 = i0 < 0 ? 0 : (i0 >= w ? w - 1 : i0);
  i1 = i1 < 0 ? 0 : (i1 >= w ? w - 1 : i1);
  j0 = j0 < 0 ? 0 : (j0 >= h ? h - 1 : j0);
  j1 = j1 < 0 ? 0 : (j1 >= h ? h - 1 : j1);
  float t00 = img[(size_t)j0 * w + i0], t10 = img[(size_t)j0 * w + i1];
  float t01 = img[(size_t)j1 * w + i0], t11 = img[(size_t)j1 * w + i1];
  if (mode == OR_SAMPLE_TEXTURE_WIDE) {
    float wq[4];
    tex_weights(a, b, wq);
    double v = (double)wq[0] * t00 + (double)wq[1] * t10 + (double)wq[2] * t01 + (double)wq[3] * t11;
    return (float)v;
  }
  if (mode == OR_SAMPLE_TEXTURE) {
    float wq[4];
    tex_weights(a, b, wq);
    float v = wq[0] * t00;
    v = fmaf(wq[1], t10, v);
    v = fmaf(wq[2], t01, v);
    return fmaf(wq[3], t11, v);
  }
  float top = fmaf(a, t10 - t00, t00);
  float bot = fmaf(a, t11 - t01, t01);
  return fmaf(b, bot - top, top);
}

#define PATCH 9
#define NE 3 /* elements per lane: ceil(81 / 32) */

static const float kGauss9[9] = {0.0135196f, 0.0476622f, 0.11723f, 0.201168f, 0.240841f,
                                 0.201168f,  0.11723f,   0.0476622f, 0.0135196f};

typedef struct {
  int valid, ix, iy, ncc;
  float w;
} lk_elem;

static void lk_layout(lk_elem el[NE][32]) {
  for (int e = 0; e < NE; ++e) {
    for (int l = 0; l < 32; ++l) {
      int f = l + 32 * e;
      int iy = f / PATCH, ix = f - iy * PATCH;
      el[e][l].valid = f < PATCH * PATCH;
      el[e][l].ix = ix;
      el[e][l].iy = iy;
      el[e][l].ncc = ix >= 2 && ix < 7 && iy >= 2 && iy < 7;
      el[e][l].w = el[e][l].valid ? kGauss9[iy] * kGauss9[ix] : 0.f;
    }
  }
}

/* lane-sequential partial sums over elements 0..2, then the 5-level butterfly */
#define LANE_SUM(expr_valid, expr)               \
  ({                                             \
    float lanes_[32];                            \
    for (int l = 0; l < 32; ++l) {               \
      float acc_ = 0.f;                          \
      for (int e = 0; e < NE; ++e)               \
        if (expr_valid) acc_ = acc_ + (expr);    \
      lanes_[l] = acc_;                          \
    }                                            \
    butterfly(lanes_, 5);                        \
  })

/* lk_track_kernel (cuda_kernels/lk_tracker.cu:69-379) for one feature: coarse-to-fine Gauss-Newton
 * on a 9x9 Gaussian-weighted window with mean-subtracted gradients, H = sum w g g^T + I (1/32 per
 * lane), mean-compensated residual, <= 11 iterations per level, stop when |v|^2 < 0.12^2, level
 * radius gate, 5x5 NCC gate, pyramid coordinates scaled about (0.5, 0.5).  `horizontal` follows
 * lk_track_horizontal_kernel (:381-665): x only, H = sum w gx^2 + 1. */
static void lk_one(int levels, const int* ws, const int* hs, const float* const* pgx, const float* const* pgy,
                   const float* const* pim, const float* const* cim, or_track_data* t, int mode, int horizontal) {
  static lk_elem el[NE][32];
  static int init = 0;
  if (!init) {
    lk_layout(el);
    init = 1;
  }
  if (t->search_radius_px < 0.f) {
    t->track_status = 0;
    return;
  }
  t->info[0] = 1.f / 9.f;
  t->info[1] = 0.f;
  t->info[2] = 0.f;
  t->info[3] = 1.f / 9.f;
  const int top = levels - 1;
  const float tx = t->track[0], ty = t->track[1];
  const float ox = t->offset[0], oy = t->offset[1];
  int in_prev = tx >= 0 && tx < (float)ws[0] && ty >= 0 && ty < (float)hs[0];
  float cx0 = tx + ox, cy0 = ty + oy;
  int in_cur = cx0 >= 0 && cx0 < (float)ws[0] && cy0 >= 0 && cy0 < (float)hs[0];
  if (!in_prev || !in_cur) {
    t->track_status = 0;
    return;
  }
  const float scale = 1.f / (float)(1 << top);
  float sx = (tx - 0.5f) * scale + 0.5f, sy = (ty - 0.5f) * scale + 0.5f;
  float cx = (cx0 - 0.5f) * scale + 0.5f, cy = (cy0 - 0.5f) * scale + 0.5f;
  const float rcp81 = 1.f / 81.f, rcp25 = 1.f / 25.f;
  const float thr2 = (float)(0.12f * 0.12f);
  int conv = 0;
  float gxp[NE][32], gyp[NE][32], p1[NE][32], p2[NE][32];
  for (int i = 0; i < levels; ++i) {
    const int level = top - i;
    const int W = ws[level], H = hs[level];
    float xmin = sx + (0.5f - 4.5f), xmax = sx + (0.5f - 4.5f + 9.f);
    float ymin = sy + (0.5f - 4.5f), ymax = sy + (0.5f - 4.5f + 9.f);
    int good = xmin >= 0 && xmax < (float)W && ymin >= 0 && ymax < (float)H;
    if (good) {
      for (int e = 0; e < NE; ++e)
        for (int l = 0; l < 32; ++l) {
          if (!el[e][l].valid) continue;
          float px = xmin + (float)el[e][l].ix, py = ymin + (float)el[e][l].iy;
          gxp[e][l] = or_tex_sample(pgx[level], W, H, px, py, mode);
          gyp[e][l] = horizontal ? 0.f : or_tex_sample(pgy[level], W, H, px, py, mode);
          p1[e][l] = or_tex_sample(pim[level], W, H, px, py, mode);
        }
      float sgx = LANE_SUM(el[e][l].valid, gxp[e][l]);
      float sgy = horizontal ? 0.f : LANE_SUM(el[e][l].valid, gyp[e][l]);
      float sp = LANE_SUM(el[e][l].valid, p1[e][l]);
      float lxx[32], lxy[32], lyy[32];
      for (int l = 0; l < 32; ++l) {
        lxx[l] = horizontal ? 0.f : 1.f / 32.f;
        lxy[l] = 0.f;
        lyy[l] = 1.f / 32.f;
        for (int e = 0; e < NE; ++e) {
          if (!el[e][l].valid) continue;
          float a = fmaf(-sgx, rcp81, gxp[e][l]);
          gxp[e][l] = a;
          if (horizontal) {
            lxx[l] = fmaf(el[e][l].w * a, a, lxx[l]);
          } else {
            float b = fmaf(-sgy, rcp81, gyp[e][l]);
            gyp[e][l] = b;
            lxx[l] = fmaf(a * a, el[e][l].w, lxx[l]);
            lxy[l] = fmaf(a * b, el[e][l].w, lxy[l]);
            lyy[l] = fmaf(b * b, el[e][l].w, lyy[l]);
          }
        }
      }
      if (horizontal) {
        /* the horizontal kernel starts its per-lane gxx at 1/32 too */
        for (int l = 0; l < 32; ++l) {
          float acc = 1.f / 32.f;
          for (int e = 0; e < NE; ++e)
            if (el[e][l].valid) acc = fmaf(el[e][l].w * gxp[e][l], gxp[e][l], acc);
          lxx[l] = acc;
        }
      }
      const float gxx = butterfly(lxx, 5);
      const float gxy = horizontal ? 0.f : butterfly(lxy, 5);
      const float gyy = horizontal ? 0.f : butterfly(lyy, 5);
      float det_rcp;
      if (horizontal) {
        if (gxx < FLT_EPSILON) {
          t->track_status = 0;
          return;
        }
        det_rcp = 1.0f / gxx;
      } else {
        const float det = fmaf(gxx, gyy, -(gxy * gxy));
        if (det < FLT_EPSILON) {
          t->track_status = 0;
          return;
        }
        det_rcp = 1.0f / det;
      }
      const float savex = cx, savey = cy;
      for (int it = 0; it < 11; ++it) {
        xmin = cx + (0.5f - 4.5f);
        xmax = cx + (0.5f - 4.5f + 9.f);
        ymin = cy + (0.5f - 4.5f);
        ymax = cy + (0.5f - 4.5f + 9.f);
        if (!(xmin >= 0 && xmax < (float)W && ymin >= 0 && ymax < (float)H)) good = 0;
        if (!good) break;
        for (int e = 0; e < NE; ++e)
          for (int l = 0; l < 32; ++l) {
            if (!el[e][l].valid) continue;
            p2[e][l] = or_tex_sample(cim[level], W, H, xmin + (float)el[e][l].ix, ymin + (float)el[e][l].iy, mode);
          }
        float sc = LANE_SUM(el[e][l].valid, p2[e][l]);
        float delta = (sc - sp) * rcp81;
        float lex[32], ley[32];
        for (int l = 0; l < 32; ++l) {
          float ax = 0.f, ay = 0.f;
          for (int e = 0; e < NE; ++e) {
            if (!el[e][l].valid) continue;
            float diff = (p2[e][l] - p1[e][l]) - delta;
            float wd = el[e][l].w * diff;
            ax = fmaf(wd, gxp[e][l], ax);
            ay = fmaf(wd, gyp[e][l], ay);
          }
          lex[l] = ax;
          ley[l] = ay;
        }
        const float ex = butterfly(lex, 5);
        float vx, vy;
        if (horizontal) {
          vx = ex * det_rcp;
          vy = 0.f;
          conv = fabsf(vx) < 0.12f;
        } else {
          const float ey = butterfly(ley, 5);
          vx = fmaf(gyy, ex, -(gxy * ey)) * det_rcp;
          vy = fmaf(gxx, ey, -(gxy * ex)) * det_rcp;
          conv = fmaf(vx, vx, vy * vy) < thr2;
        }
        if (conv) break;
        cx += vx;
        cy += vy;
      }
      if (conv) {
        const float r = t->search_radius_px / (float)(1 << level);
        const float dx = cx - savex, dy = cy - savey;
        if (fmaf(dx, dx, dy * dy) > r * r) conv = 0;
      }
      if (conv) {
        float s1 = LANE_SUM(el[e][l].ncc, p1[e][l]);
        float s2 = LANE_SUM(el[e][l].ncc, p2[e][l]);
        float q[3][32];
        for (int l = 0; l < 32; ++l) {
          float a = 0.f, b = 0.f, c = 0.f;
          for (int e = 0; e < NE; ++e) {
            if (!el[e][l].ncc) continue;
            a = fmaf(p1[e][l], p1[e][l], a);
            b = fmaf(p2[e][l], p2[e][l], b);
            c = fmaf(p2[e][l], p1[e][l], c);
          }
          q[0][l] = a;
          q[1][l] = b;
          q[2][l] = c;
        }
        const float s11 = butterfly(q[0], 5), s22 = butterfly(q[1], 5), s12 = butterfly(q[2], 5);
        const float a1 = s1 * rcp25, a2 = s2 * rcp25;
        const float d1 = fmaf(s11, rcp25, -(a1 * a1));
        const float d2 = fmaf(s22, rcp25, -(a2 * a2));
        const float d12 = fmaf(s12, rcp25, -(a1 * a2));
        const float d1d2 = d1 * d2;
        const float ncc = d1d2 < FLT_EPSILON ? 0.f : d12 * (float)(1.0 / sqrt((double)d1d2));
        conv = ncc > t->ncc_threshold;
      }
      if (!conv && level > 0) {
        cx = savex;
        cy = savey;
      }
      conv = level == 0 && conv;
    }
    if (i != levels - 1) {
      sx = sx * 2.f - 0.5f;
      sy = sy * 2.f - 0.5f;
      cx = cx * 2.f - 0.5f;
      cy = cy * 2.f - 0.5f;
    }
  }
  if (conv) {
    t->track[0] = cx;
    t->track[1] = cy;
  }
  t->track_status = (uint8_t)conv;
}

void or_lk_track(int levels, const int* ws, const int* hs, const float* const* prev_gx, const float* const* prev_gy,
                 const float* const* prev_img, const float* const* cur_img, or_track_data* td, int n, int mode) {
  for (int k = 0; k < n; ++k) lk_one(levels, ws, hs, prev_gx, prev_gy, prev_img, cur_img, &td[k], mode, 0);
}

void or_lk_track_horizontal(int levels, const int* ws, const int* hs, const float* const* prev_gx,
                            const float* const* prev_img, const float* const* cur_img, or_track_data* td, int n,
                            int mode) {
  for (int k = 0; k < n; ++k) lk_one(levels, ws, hs, prev_gx, prev_gx, prev_img, cur_img, &td[k], mode, 1);
}

/* EpipolarCurves::Candidates (libs/sof/epipolar_curves.cpp:64-101): the corner grid position of the
 * point at the top level, nothing outside the grid (or when the right or bottom corner is missing),
 * else the four corner curves blended with bilinear weights up to the shortest of them, each
 * coordinate ((w00 c00 + w01 c01) + w10 c10) + w11 c11 in FP32. */
int or_epipolar_candidates(int cw, int ch, float inv_scale, const int32_t* offsets, const float* xy, float u, float v,
                           float* out, int cap) {
  const float vf = v * inv_scale, uf = u * inv_scale;
  if (!(vf >= 0.f && vf < (float)ch && uf >= 0.f && uf < (float)cw)) return 0;
  const int v0 = (int)vf, u0 = (int)uf;
  if (v0 + 1 >= ch || u0 + 1 >= cw) return 0;
  const float dv = vf - (float)v0, du = uf - (float)u0;
  const float w00 = (1.0f - du) * (1.0f - dv);
  const float w01 = du * (1.0f - dv);
  const float w10 = (1.0f - du) * dv;
  const float w11 = du * dv;
  const int i00 = v0 * cw + u0, i01 = i00 + 1, i10 = i00 + cw, i11 = i10 + 1;
  int n = offsets[i00 + 1] - offsets[i00];
  const int n01 = offsets[i01 + 1] - offsets[i01], n10 = offsets[i10 + 1] - offsets[i10];
  const int n11 = offsets[i11 + 1] - offsets[i11];
  if (n01 < n) n = n01;
  if (n10 < n) n = n10;
  if (n11 < n) n = n11;
  if (n > cap) n = cap;
  const float* c00 = xy + 2 * (size_t)offsets[i00];
  const float* c01 = xy + 2 * (size_t)offsets[i01];
  const float* c10 = xy + 2 * (size_t)offsets[i10];
  const float* c11 = xy + 2 * (size_t)offsets[i11];
  for (int k = 0; k < n; ++k)
    for (int d = 0; d < 2; ++d)
      out[2 * k + d] = w00 * c00[2 * k + d] + w01 * c01[2 * k + d] + w10 * c10[2 * k + d] + w11 * c11[2 * k + d];
  return n;
}

/* The unmatched record of the scan: track = uv, everything the tracker would write cleared. */
static void stereo_record(or_track_data* t, float x, float y, float radius, float ncc_thr) {
  memset(t, 0, sizeof(*t));
  t->track[0] = x;
  t->track[1] = y;
  t->cache_index = -1;
  t->initial_guess_map[0] = 1.f;
  t->initial_guess_map[3] = 1.f;
  t->search_radius_px = radius;
  t->ncc_threshold = ncc_thr;
}

/* MultiSOFGPU::LaunchTrackingPrimaryToSecondary (libs/sof/sof_multicamera_gpu.cpp:118-190), with the
 * horizontal (lr_tracker = LKHorizontal) or the 2-D tracker (LK): round k
 * tracks candidate k of every point without a match that has one (the reference's sentinel
 * entries, tracked with a zero offset and discarded, are left out); no round when none has; after
 * round k, stop once matched >= early_exit_fraction * n (kL2REarlyExitFraction). */
void or_stereo_scan(int levels, const int* ws, const int* hs, const float* const* prim_gx,
                    const float* const* prim_gy, const float* const* prim_img, const float* const* sec_img,
                    const float* uv, const uint8_t* valid, int n, const int32_t* cand_off, const float* cand_xy,
                    float search_radius, float ncc_threshold, float early_exit_fraction, int horizontal, int mode,
                    or_track_data* out, int32_t* winner, int32_t* stats) {
  int max_candidates = 0;
  for (int i = 0; i < n; ++i) {
    const int len = (valid && !valid[i]) ? 0 : cand_off[i + 1] - cand_off[i];
    if (len > max_candidates) max_candidates = len;
    winner[i] = -1;
    if (valid && !valid[i])
      stereo_record(&out[i], 0.f, 0.f, search_radius, ncc_threshold);
    else
      stereo_record(&out[i], uv[2 * i], uv[2 * i + 1], search_radius, ncc_threshold);
  }
  int tracked = 0, rounds = 0, attempts = 0;
  for (int k = 0; k < max_candidates; ++k) {
    int any_active = 0;
    for (int i = 0; i < n; ++i) {
      const int len = (valid && !valid[i]) ? 0 : cand_off[i + 1] - cand_off[i];
      if (winner[i] >= 0 || k >= len) continue;
      any_active = 1;
      or_track_data t;
      stereo_record(&t, uv[2 * i], uv[2 * i + 1], search_radius, ncc_threshold);
      const float* c = cand_xy + 2 * ((size_t)cand_off[i] + k);
      t.offset[0] = c[0] - uv[2 * i];
      t.offset[1] = c[1] - uv[2 * i + 1];
      lk_one(levels, ws, hs, prim_gx, horizontal ? prim_gx : prim_gy, prim_img, sec_img, &t, mode, horizontal);
      ++attempts;
      if (t.track_status) {
        out[i] = t;
        winner[i] = k;
        ++tracked;
      }
    }
    if (!any_active) break;
    rounds = k + 1;
    if ((float)tracked >= early_exit_fraction * (float)n) break;
  }
  stats[0] = tracked;
  stats[1] = rounds;
  stats[2] = attempts;
  stats[3] = 0;
}

/* MonoSOFGPU::finish's track filters (libs/sof/sof_mono_gpu.cpp:80-104 collect, :144-170 finish;
 * sof_mono_base.cpp:51-109 filterByPredictionError and IncrementTracksAge, :121-133
 * KillTracksWithinMask; selector_stereo.cpp:109-125 KillTracksOnBorder; sof_mono_gpu.cpp:249-280
 * collapseTracks), over the n tracks of one camera after LK, in the reference's order:
 *   collect:    an alive track (age > 0) whose LK record has track_status keeps the record's track
 *               as its position, else it dies (age 0; records merge the track and retrack passes);
 *   age:        every alive track's age + 1;
 *   prediction: with pred (x, y per track, NaN x = no prediction) and at least 3 alive predicted
 *               tracks, d = |pred - position| (sqrt of dx*dx + dy*dy), m = the (count/2)-th smallest
 *               d (nth_element), and tracks with d > max(3, 2 m) die;
 *   border:     a track dies unless bl <= x <= w-1-br and bt <= y <= h-1-bb (integer bounds computed
 *               as size_t, then compared as float);
 *   mask:       a track on a nonzero mask pixel (row (size_t)y, column (size_t)x) dies;
 *   collapse:   per 3x3-pixel cell ((size_t)(x / 3), (size_t)(y / 3)) only the first track (in index
 *               order) with the cell's largest age survives.
 * Dead tracks get track_status 0 in their record.  Returns the number of tracks alive. */
int or_finish_tracks(or_track_data* td, uint32_t* age, int n, const float* pred, int w, int h, const int* border,
                     const uint8_t* mask, int64_t mask_pitch, int collapse) {
  for (int i = 0; i < n; ++i) {
    if (age[i] == 0) {
      td[i].track_status = 0;
      continue;
    }
    if (td[i].track_status)
      age[i] += 1;
    else
      age[i] = 0;
  }
  if (pred) {
    float* d = (float*)malloc(sizeof(float) * (size_t)(n > 0 ? n : 1));
    float* sorted = (float*)malloc(sizeof(float) * (size_t)(n > 0 ? n : 1));
    int m = 0;
    for (int i = 0; i < n; ++i) {
      if (age[i] == 0 || pred[2 * i] != pred[2 * i]) continue;
      const float dx = pred[2 * i] - td[i].track[0], dy = pred[2 * i + 1] - td[i].track[1];
      d[i] = sqrtf(dx * dx + dy * dy);
      sorted[m++] = d[i];
    }
    if (m >= 3) {
      /* the (m/2)-th smallest: insertion-free selection by counting (m is small) */
      float kth = 0.f;
      for (int a = 0; a < m; ++a) {
        int below = 0, equal = 0;
        for (int b = 0; b < m; ++b) {
          below += sorted[b] < sorted[a];
          equal += sorted[b] == sorted[a];
        }
        if (below <= m / 2 && m / 2 < below + equal) {
          kth = sorted[a];
          break;
        }
      }
      const float thr = 2.f * kth > 3.f ? 2.f * kth : 3.f;
      for (int i = 0; i < n; ++i) {
        if (age[i] == 0 || pred[2 * i] != pred[2 * i]) continue;
        if (d[i] > thr) age[i] = 0;
      }
    }
    free(d);
    free(sorted);
  }
  const uint64_t W = (uint64_t)w, H = (uint64_t)h;
  const uint64_t bt = (uint64_t)border[0], bb = (uint64_t)border[1], bl = (uint64_t)border[2],
                 br = (uint64_t)border[3];
  for (int i = 0; i < n; ++i) {
    if (age[i] == 0) continue;
    const float x = td[i].track[0], y = td[i].track[1];
    if (!((float)bl <= x && x <= (float)(W - 1 - br) && (float)bt <= y && y <= (float)(H - 1 - bb))) age[i] = 0;
  }
  if (mask)
    for (int i = 0; i < n; ++i) {
      if (age[i] == 0) continue;
      const float x = td[i].track[0], y = td[i].track[1];
      if (x >= 0.f && y >= 0.f && x < (float)w && y < (float)h && mask[(size_t)y * mask_pitch + (size_t)x]) age[i] = 0;
    }
  if (collapse) {
    const int cw = (w + 2) / 3, ch = (h + 2) / 3;
    uint32_t* best = (uint32_t*)calloc((size_t)cw * ch, sizeof(uint32_t));
    for (int i = 0; i < n; ++i) {
      if (age[i] == 0) continue;
      const int cx = (int)(td[i].track[0] / 3.f), cy = (int)(td[i].track[1] / 3.f);
      if (cx < 0 || cy < 0 || cx >= cw || cy >= ch) continue;
      uint32_t* p = &best[(size_t)cy * cw + cx];
      if (*p < age[i]) *p = age[i];
    }
    for (int i = 0; i < n; ++i) {
      if (age[i] == 0) continue;
      const int cx = (int)(td[i].track[0] / 3.f), cy = (int)(td[i].track[1] / 3.f);
      if (cx < 0 || cy < 0 || cx >= cw || cy >= ch) continue;
      uint32_t* p = &best[(size_t)cy * cw + cx];
      if (age[i] == *p)
        *p = 0;
      else
        age[i] = 0;
    }
    free(best);
  }
  int alive = 0;
  for (int i = 0; i < n; ++i) {
    if (age[i] == 0) td[i].track_status = 0;
    alive += age[i] != 0;
  }
  return alive;
}

/* FP64 restatement of the same LK (exact bilinear weights, double arithmetic, plain summation
 * order).  Used only to state per-track error of the FP32 paths. */
static double samp64(const float* img, int w, int h, double x, double y) {
  double xb = x - 0.5, yb = y - 0.5;
  double fx = floor(xb), fy = floor(yb);
  double a = xb - fx, b = yb - fy;
  int i0 = (int)fx, j0 = (int)fy, i1 = i0 + 1, j1 = j0 + 1;
  i0 = i0 < 0 ? 0 : (i0 >= w ? w - 1 : i0);
  i1 = i1 < 0 ? 0 : (i1 >= w ? w - 1 : i1);
  j0 = j0 < 0 ? 0 : (j0 >= h ? h - 1 : j0);
  j1 = j1 < 0 ? 0 : (j1 >= h ? h - 1 : j1);
  return (1 - a) * (1 - b) * img[(size_t)j0 * w + i0] + a * (1 - b) * img[(size_t)j0 * w + i1] +
         (1 - a) * b * img[(size_t)j1 * w + i0] + a * b * img[(size_t)j1 * w + i1];
}

void or_lk_track_f64(int levels, const int* ws, const int* hs, const float* const* pgx, const float* const* pgy,
                     const float* const* pim, const float* const* cim, or_track_data* td, int n) {
  for (int k = 0; k < n; ++k) {
    or_track_data* t = &td[k];
    if (t->search_radius_px < 0.f) {
      t->track_status = 0;
      continue;
    }
    const int top = levels - 1;
    double tx = t->track[0], ty = t->track[1], ox = t->offset[0], oy = t->offset[1];
    if (!(tx >= 0 && tx < ws[0] && ty >= 0 && ty < hs[0] && tx + ox >= 0 && tx + ox < ws[0] && ty + oy >= 0 &&
          ty + oy < hs[0])) {
      t->track_status = 0;
      continue;
    }
    double scale = 1.0 / (double)(1 << top);
    double sx = (tx - 0.5) * scale + 0.5, sy = (ty - 0.5) * scale + 0.5;
    double cx = (tx + ox - 0.5) * scale + 0.5, cy = (ty + oy - 0.5) * scale + 0.5;
    int conv = 0, fail = 0;
    for (int i = 0; i < levels && !fail; ++i) {
      const int level = top - i;
      const int W = ws[level], H = hs[level];
      if (!(sx - 4 < 0 || sx + 5 >= W || sy - 4 < 0 || sy + 5 >= H)) {
        double gx[81], gy[81], p1[81], p2[81], mgx = 0, mgy = 0, mp = 0;
        for (int f = 0; f < 81; ++f) {
          double px = sx - 4 + f % 9, py = sy - 4 + f / 9;
          gx[f] = samp64(pgx[level], W, H, px, py);
          gy[f] = samp64(pgy[level], W, H, px, py);
          p1[f] = samp64(pim[level], W, H, px, py);
          mgx += gx[f];
          mgy += gy[f];
          mp += p1[f];
        }
        double gxx = 1, gxy = 0, gyy = 1;
        for (int f = 0; f < 81; ++f) {
          double wgt = (double)kGauss9[f / 9] * (double)kGauss9[f % 9];
          gx[f] -= mgx / 81;
          gy[f] -= mgy / 81;
          gxx += wgt * gx[f] * gx[f];
          gxy += wgt * gx[f] * gy[f];
          gyy += wgt * gy[f] * gy[f];
        }
        double det = gxx * gyy - gxy * gxy;
        if (det < FLT_EPSILON) {
          fail = 1;
          break;
        }
        double savex = cx, savey = cy;
        int good = 1;
        conv = 0;
        for (int it = 0; it < 11; ++it) {
          if (cx - 4 < 0 || cx + 5 >= W || cy - 4 < 0 || cy + 5 >= H) {
            good = 0;
            break;
          }
          double mc = 0;
          for (int f = 0; f < 81; ++f) {
            p2[f] = samp64(cim[level], W, H, cx - 4 + f % 9, cy - 4 + f / 9);
            mc += p2[f];
          }
          double delta = (mc - mp) / 81, ex = 0, ey = 0;
          for (int f = 0; f < 81; ++f) {
            double wgt = (double)kGauss9[f / 9] * (double)kGauss9[f % 9];
            double d = p2[f] - p1[f] - delta;
            ex += wgt * d * gx[f];
            ey += wgt * d * gy[f];
          }
          double vx = (gyy * ex - gxy * ey) / det, vy = (gxx * ey - gxy * ex) / det;
          conv = vx * vx + vy * vy < 0.12 * 0.12;
          if (conv) break;
          cx += vx;
          cy += vy;
        }
        (void)good;
        if (conv) {
          double r = t->search_radius_px / (double)(1 << level);
          if ((cx - savex) * (cx - savex) + (cy - savey) * (cy - savey) > r * r) conv = 0;
        }
        if (conv) {
          double s1 = 0, s2 = 0, s11 = 0, s22 = 0, s12 = 0;
          for (int yy = 2; yy < 7; ++yy)
            for (int xx = 2; xx < 7; ++xx) {
              double a = p1[yy * 9 + xx], b = p2[yy * 9 + xx];
              s1 += a;
              s2 += b;
              s11 += a * a;
              s22 += b * b;
              s12 += a * b;
            }
          double a1 = s1 / 25, a2 = s2 / 25;
          double d1 = s11 / 25 - a1 * a1, d2 = s22 / 25 - a2 * a2, d12 = s12 / 25 - a1 * a2;
          double ncc = d1 * d2 < FLT_EPSILON ? 0 : d12 / sqrt(d1 * d2);
          conv = ncc > t->ncc_threshold;
        }
        if (!conv && level > 0) {
          cx = savex;
          cy = savey;
        }
        conv = level == 0 && conv;
      }
      if (i != levels - 1) {
        sx = sx * 2 - 0.5;
        sy = sy * 2 - 0.5;
        cx = cx * 2 - 0.5;
        cy = cy * 2 - 0.5;
      }
    }
    if (fail) {
      t->track_status = 0;
      continue;
    }
    if (conv) {
      t->track[0] = (float)cx;
      t->track[1] = (float)cy;
    }
    t->track_status = (uint8_t)conv;
  }
}
