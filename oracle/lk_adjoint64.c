/* FP64 reference of the differentiable LK tracker and its adjoint.  TEST INFRASTRUCTURE ONLY
 * (see fe_oracle.h): the tests compare the CUDA adjoint with or64_backward and with central finite
 * differences of or64_track.
 *
 * Forward model (the one the CUDA diff tracker runs in FP32), per track, as lk_track_kernel
 * (cuda_kernels/lk_tracker.cu:69-379) with exact bilinear sampling:
 *   pyramid   gaussian_scaling_kernel (image_pyramid.cu:56-102) and conv_grad_x/y
 *             (convolutions.cu:74-139) as linear maps, in double;
 *   level l   template P1, Gx, Gy at s_l + o_k (9x9 taps), a = Gx - mean, b = Gy - mean,
 *             H = I + sum w g g^T, det >= FLT_EPSILON else the track fails;
 *             iteration: P2 at c + o_k, r = P2 - P1 - (mean P2 - mean P1), e = sum w r g,
 *             v = H^-1 e, c += v;
 *   OR64_IMPLICIT: the reference iteration rule (<= 11 iterations, stop when |v| < 0.12 without
 *             applying that v, radius and NCC gates) on every level, then at level 0 the fixed
 *             point is refined: up to `iters` Newton steps on e(c) = 0 (exact Jacobian), stopping
 *             after the step shorter than tol; a track fails whose refinement does not get there,
 *             takes a step or drifts from the reference result beyond 2 px, or ends where
 *             |det J| < 0.01 |J|_F^2 (sigma_min / sigma_max below about 0.01).  Its adjoint is the
 *             implicit-function theorem at e(c*) = 0.
 *   OR64_UNROLLED: exactly `iters` steps on every level (no early stop); the level succeeds when
 *             the last |v| < 0.12 and the radius and NCC gates pass; a level that fails at
 *             l > 0 restarts the next level from its own start.  Its adjoint runs back through
 *             every step (the gates are piecewise constant and carry no gradient).
 * Coordinates map between levels as s_l = 2 s_{l+1} - 1/2.
 */
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "fe_oracle.h"

#define L64_MAX_LEVELS 10
#define L64_MAX_IT 64

/* implicit mode: smallest accepted |det J| / |J|_F^2 (about sigma_min / sigma_max) */
static const double kCondMin = 0.01;

static const float kDsp32[7] = {112.0f / 8418.0f, 913.0f / 8418.0f, 3047.0f / 8418.0f, 0.0f,
                                -3047.0f / 8418.0f, -913.0f / 8418.0f, -112.0f / 8418.0f};
static const float kG9[9] = {0.0135196f, 0.0476622f, 0.11723f, 0.201168f, 0.240841f,
                             0.201168f,  0.11723f,   0.0476622f, 0.0135196f};

struct or64_cam {
  int levels, ws[L64_MAX_LEVELS], hs[L64_MAX_LEVELS];
  double *pimg[L64_MAX_LEVELS], *pgx[L64_MAX_LEVELS], *pgy[L64_MAX_LEVELS], *cimg[L64_MAX_LEVELS];
  /* adjoint planes */
  double *dpimg[L64_MAX_LEVELS], *dpgx[L64_MAX_LEVELS], *dpgy[L64_MAX_LEVELS], *dcimg[L64_MAX_LEVELS];
};

or64_cam* or64_cam_create(int w, int h, int max_levels) {
  or64_cam* c = (or64_cam*)calloc(1, sizeof(or64_cam));
  c->levels = or_level_sizes(w, h, max_levels, c->ws, c->hs);
  for (int l = 0; l < c->levels; ++l) {
    size_t n = (size_t)c->ws[l] * c->hs[l];
    c->pimg[l] = calloc(n, sizeof(double));
    c->pgx[l] = calloc(n, sizeof(double));
    c->pgy[l] = calloc(n, sizeof(double));
    c->cimg[l] = calloc(n, sizeof(double));
    c->dpimg[l] = calloc(n, sizeof(double));
    c->dpgx[l] = calloc(n, sizeof(double));
    c->dpgy[l] = calloc(n, sizeof(double));
    c->dcimg[l] = calloc(n, sizeof(double));
  }
  return c;
}

void or64_cam_destroy(or64_cam* c) {
  if (!c) return;
  for (int l = 0; l < c->levels; ++l) {
    free(c->pimg[l]);
    free(c->pgx[l]);
    free(c->pgy[l]);
    free(c->cimg[l]);
    free(c->dpimg[l]);
    free(c->dpgx[l]);
    free(c->dpgy[l]);
    free(c->dcimg[l]);
  }
  free(c);
}

int or64_cam_levels(const or64_cam* c) { return c->levels; }

/* ------------------------------------------------------------------ pyramid and its adjoint */
static inline int mir(int i, int n) {
  i = i < 0 ? -i - 1 : i;
  return i >= n ? 2 * n - i - 1 : i;
}

static double k2(int k, int l) {
  static const double k1[5] = {1.0 / 16, 4.0 / 16, 6.0 / 16, 4.0 / 16, 1.0 / 16};
  return (double)((float)k1[k] * (float)k1[l]);
}

static void down64(const double* src, int sw, int sh, double* dst, int dw, int dh) {
  for (int y = 0; y < dh; ++y)
    for (int x = 0; x < dw; ++x) {
      double acc = 0;
      for (int k = 0; k < 5; ++k)
        for (int l = 0; l < 5; ++l) {
          int xc = 2 * x - 2 + l, yc = 2 * y - 2 + k;
          if ((xc < 0 || xc >= sw) && (yc < 0 || yc >= sh)) continue;
          acc += k2(k, l) * src[(size_t)mir(yc, sh) * sw + mir(xc, sw)];
        }
      dst[(size_t)y * dw + x] = acc;
    }
}

static void down64_adj(const double* dout, int dw, int dh, double* din, int sw, int sh) {
  for (int y = 0; y < dh; ++y)
    for (int x = 0; x < dw; ++x) {
      const double g = dout[(size_t)y * dw + x];
      if (g == 0) continue;
      for (int k = 0; k < 5; ++k)
        for (int l = 0; l < 5; ++l) {
          int xc = 2 * x - 2 + l, yc = 2 * y - 2 + k;
          if ((xc < 0 || xc >= sw) && (yc < 0 || yc >= sh)) continue;
          din[(size_t)mir(yc, sh) * sw + mir(xc, sw)] += k2(k, l) * g;
        }
    }
}

static void grad64(const double* in, int w, int h, double* gx, double* gy) {
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      double sx = 0, sy = 0;
      if (x > 2 && x < w - 3)
        for (int j = 0; j < 7; ++j) sx += (double)kDsp32[j] * in[(size_t)y * w + x - 3 + j];
      if (y > 2 && y < h - 3)
        for (int j = 0; j < 7; ++j) sy += (double)kDsp32[j] * in[(size_t)(y - 3 + j) * w + x];
      gx[(size_t)y * w + x] = sx;
      gy[(size_t)y * w + x] = sy;
    }
}

static void grad64_adj(const double* dgx, const double* dgy, int w, int h, double* din) {
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      const double a = dgx[(size_t)y * w + x], b = dgy[(size_t)y * w + x];
      if (a != 0 && x > 2 && x < w - 3)
        for (int j = 0; j < 7; ++j) din[(size_t)y * w + x - 3 + j] += (double)kDsp32[j] * a;
      if (b != 0 && y > 2 && y < h - 3)
        for (int j = 0; j < 7; ++j) din[(size_t)(y - 3 + j) * w + x] += (double)kDsp32[j] * b;
    }
}

void or64_cam_set(or64_cam* c, const double* prev0, const double* cur0) {
  memcpy(c->pimg[0], prev0, sizeof(double) * c->ws[0] * c->hs[0]);
  memcpy(c->cimg[0], cur0, sizeof(double) * c->ws[0] * c->hs[0]);
  for (int l = 1; l < c->levels; ++l) {
    down64(c->pimg[l - 1], c->ws[l - 1], c->hs[l - 1], c->pimg[l], c->ws[l], c->hs[l]);
    down64(c->cimg[l - 1], c->ws[l - 1], c->hs[l - 1], c->cimg[l], c->ws[l], c->hs[l]);
  }
  for (int l = 0; l < c->levels; ++l) grad64(c->pimg[l], c->ws[l], c->hs[l], c->pgx[l], c->pgy[l]);
}

/* the planes of level l: 0 prev image, 1 prev grad_x, 2 prev grad_y, 3 current image */
void or64_cam_plane(const or64_cam* c, int level, int plane, double* out) {
  const double* src = plane == 0 ? c->pimg[level] : plane == 1 ? c->pgx[level] : plane == 2 ? c->pgy[level] : c->cimg[level];
  memcpy(out, src, sizeof(double) * c->ws[level] * c->hs[level]);
}

/* ------------------------------------------------------------------ bilinear taps */
typedef struct {
  int i0, i1, j0, j1;
  double a, b;
} tap64;

static tap64 tap_at(int w, int h, double x, double y) {
  tap64 t;
  double xb = x - 0.5, yb = y - 0.5, fx = floor(xb), fy = floor(yb);
  t.a = xb - fx;
  t.b = yb - fy;
  int i0 = (int)fx, j0 = (int)fy;
  t.i0 = i0 < 0 ? 0 : (i0 >= w ? w - 1 : i0);
  t.i1 = i0 + 1 < 0 ? 0 : (i0 + 1 >= w ? w - 1 : i0 + 1);
  t.j0 = j0 < 0 ? 0 : (j0 >= h ? h - 1 : j0);
  t.j1 = j0 + 1 < 0 ? 0 : (j0 + 1 >= h ? h - 1 : j0 + 1);
  return t;
}

static double tval(const double* im, int w, tap64 t) {
  return (1 - t.a) * (1 - t.b) * im[(size_t)t.j0 * w + t.i0] + t.a * (1 - t.b) * im[(size_t)t.j0 * w + t.i1] +
         (1 - t.a) * t.b * im[(size_t)t.j1 * w + t.i0] + t.a * t.b * im[(size_t)t.j1 * w + t.i1];
}

/* spatial derivative of the bilinear interpolant */
static void tgrad(const double* im, int w, tap64 t, double* dx, double* dy) {
  const double t00 = im[(size_t)t.j0 * w + t.i0], t10 = im[(size_t)t.j0 * w + t.i1];
  const double t01 = im[(size_t)t.j1 * w + t.i0], t11 = im[(size_t)t.j1 * w + t.i1];
  *dx = (t.i1 == t.i0) ? 0 : (1 - t.b) * (t10 - t00) + t.b * (t11 - t01);
  *dy = (t.j1 == t.j0) ? 0 : (1 - t.a) * (t01 - t00) + t.a * (t11 - t10);
}

static void tscatter(double* d, int w, tap64 t, double v) {
  d[(size_t)t.j0 * w + t.i0] += (1 - t.a) * (1 - t.b) * v;
  d[(size_t)t.j0 * w + t.i1] += t.a * (1 - t.b) * v;
  d[(size_t)t.j1 * w + t.i0] += (1 - t.a) * t.b * v;
  d[(size_t)t.j1 * w + t.i1] += t.a * t.b * v;
}

static inline double wk(int k) { return (double)(kG9[k / 9] * kG9[k % 9]); }

/* ------------------------------------------------------------------ forward with records */
typedef struct {
  int processed, ok, K;
  double sx, sy;
  double cx[L64_MAX_IT + 1], cy[L64_MAX_IT + 1];
} lrec;

typedef struct {
  int status;
  double x, y;
  lrec lv[L64_MAX_LEVELS];
} trec;

typedef struct {
  double p1[81], gx[81], gy[81], a[81], b[81], mp1;
  double hxx, hxy, hyy, det;
} templ;

static void make_templ(const or64_cam* c, int level, double sx, double sy, templ* T) {
  const int W = c->ws[level], H = c->hs[level];
  double mgx = 0, mgy = 0, mp = 0;
  for (int k = 0; k < 81; ++k) {
    tap64 t = tap_at(W, H, sx - 4 + k % 9, sy - 4 + k / 9);
    T->p1[k] = tval(c->pimg[level], W, t);
    T->gx[k] = tval(c->pgx[level], W, t);
    T->gy[k] = tval(c->pgy[level], W, t);
    mgx += T->gx[k];
    mgy += T->gy[k];
    mp += T->p1[k];
  }
  T->mp1 = mp / 81;
  T->hxx = 1;
  T->hxy = 0;
  T->hyy = 1;
  for (int k = 0; k < 81; ++k) {
    T->a[k] = T->gx[k] - mgx / 81;
    T->b[k] = T->gy[k] - mgy / 81;
    T->hxx += wk(k) * T->a[k] * T->a[k];
    T->hxy += wk(k) * T->a[k] * T->b[k];
    T->hyy += wk(k) * T->b[k] * T->b[k];
  }
  T->det = T->hxx * T->hyy - T->hxy * T->hxy;
}

/* one step at c: samples P2 (into p2), residuals r, the update v */
static void step(const or64_cam* c, int level, const templ* T, double cx, double cy, double* p2, double* r, double* vx,
                 double* vy) {
  const int W = c->ws[level], H = c->hs[level];
  double mc = 0;
  for (int k = 0; k < 81; ++k) {
    p2[k] = tval(c->cimg[level], W, tap_at(W, H, cx - 4 + k % 9, cy - 4 + k / 9));
    mc += p2[k];
  }
  const double delta = mc / 81 - T->mp1;
  double ex = 0, ey = 0;
  for (int k = 0; k < 81; ++k) {
    r[k] = p2[k] - T->p1[k] - delta;
    ex += wk(k) * r[k] * T->a[k];
    ey += wk(k) * r[k] * T->b[k];
  }
  *vx = (T->hyy * ex - T->hxy * ey) / T->det;
  *vy = (T->hxx * ey - T->hxy * ex) / T->det;
}

/* J = de/dc at c: sum w g (dP2/dc - mean dP2/dc)^T, row-major [J00 J01 J10 J11] */
static void jacobian(const or64_cam* c, int level, const templ* T, double cx, double cy, double* J) {
  const int W = c->ws[level], H = c->hs[level];
  double dx[81], dy[81], mdx = 0, mdy = 0;
  for (int k = 0; k < 81; ++k) {
    tgrad(c->cimg[level], W, tap_at(W, H, cx - 4 + k % 9, cy - 4 + k / 9), &dx[k], &dy[k]);
    mdx += dx[k] / 81;
    mdy += dy[k] / 81;
  }
  J[0] = J[1] = J[2] = J[3] = 0;
  for (int k = 0; k < 81; ++k) {
    J[0] += wk(k) * T->a[k] * (dx[k] - mdx);
    J[1] += wk(k) * T->a[k] * (dy[k] - mdy);
    J[2] += wk(k) * T->b[k] * (dx[k] - mdx);
    J[3] += wk(k) * T->b[k] * (dy[k] - mdy);
  }
}

static int box_ok(double x, double y, int W, int H) { return x - 4 >= 0 && x + 5 < W && y - 4 >= 0 && y + 5 < H; }

static double ncc(const templ* T, const double* p2) {
  double s1 = 0, s2 = 0, s11 = 0, s22 = 0, s12 = 0;
  for (int yy = 2; yy < 7; ++yy)
    for (int xx = 2; xx < 7; ++xx) {
      double a = T->p1[yy * 9 + xx], b = p2[yy * 9 + xx];
      s1 += a;
      s2 += b;
      s11 += a * a;
      s22 += b * b;
      s12 += a * b;
    }
  double a1 = s1 / 25, a2 = s2 / 25;
  double d1 = s11 / 25 - a1 * a1, d2 = s22 / 25 - a2 * a2, d12 = s12 / 25 - a1 * a2;
  return d1 * d2 < FLT_EPSILON ? 0 : d12 / sqrt(d1 * d2);
}

static void track_one(const or64_cam* c, const or_track_data* td, int mode, int iters, double tol, trec* R) {
  memset(R, 0, sizeof(*R));
  const double thr2 = 0.12 * 0.12;
  const double tx = td->track[0], ty = td->track[1], ox = td->offset[0], oy = td->offset[1];
  R->x = tx;
  R->y = ty;
  if (td->search_radius_px < 0.f) return;
  if (!(tx >= 0 && tx < c->ws[0] && ty >= 0 && ty < c->hs[0] && tx + ox >= 0 && tx + ox < c->ws[0] && ty + oy >= 0 &&
        ty + oy < c->hs[0]))
    return;
  const int top = c->levels - 1;
  const double scale = 1.0 / (double)(1 << top);
  double sx = (tx - 0.5) * scale + 0.5, sy = (ty - 0.5) * scale + 0.5;
  double cx = (tx + ox - 0.5) * scale + 0.5, cy = (ty + oy - 0.5) * scale + 0.5;
  int conv = 0;
  templ T;
  double p2[81], r[81];
  for (int i = 0; i < c->levels; ++i) {
    const int level = top - i;
    const int W = c->ws[level], H = c->hs[level];
    lrec* L = &R->lv[level];
    L->sx = sx;
    L->sy = sy;
    if (box_ok(sx, sy, W, H)) {
      L->processed = 1;
      make_templ(c, level, sx, sy, &T);
      if (T.det < FLT_EPSILON) return; /* the track fails */
      const double savex = cx, savey = cy;
      double vx = 0, vy = 0;
      int good = 1, sampled = 0;
      conv = 0;
      if (mode == OR64_UNROLLED) {
        L->K = 0;
        for (int t = 0; t < iters; ++t) {
          if (!box_ok(cx, cy, W, H)) {
            good = 0;
            break;
          }
          L->cx[t] = cx;
          L->cy[t] = cy;
          step(c, level, &T, cx, cy, p2, r, &vx, &vy);
          sampled = 1;
          cx += vx;
          cy += vy;
          L->K = t + 1;
        }
        L->cx[L->K] = cx;
        L->cy[L->K] = cy;
        conv = good && sampled && vx * vx + vy * vy < thr2;
      } else {
        for (int it = 0; it < 11; ++it) {
          if (!box_ok(cx, cy, W, H)) {
            good = 0;
            break;
          }
          step(c, level, &T, cx, cy, p2, r, &vx, &vy);
          sampled = 1;
          conv = vx * vx + vy * vy < thr2;
          if (conv) break;
          cx += vx;
          cy += vy;
        }
        if (!good) conv = 0;
      }
      if (conv) {
        const double rr = td->search_radius_px / (double)(1 << level);
        if ((cx - savex) * (cx - savex) + (cy - savey) * (cy - savey) > rr * rr) conv = 0;
      }
      if (conv) conv = ncc(&T, p2) > td->ncc_threshold;
      if (!conv && level > 0) {
        cx = savex;
        cy = savey;
      }
      if (mode == OR64_IMPLICIT && level == 0 && conv) {
        /* Newton steps on e(c) = 0 with its exact Jacobian (the fixed point of the steps above) */
        int settled = 0;
        const double rx = cx, ry = cy;
        for (int it = 0; it < iters; ++it) {
          if (!box_ok(cx, cy, W, H)) break;
          step(c, level, &T, cx, cy, p2, r, &vx, &vy);
          double J[4], ex = 0, ey = 0;
          jacobian(c, level, &T, cx, cy, J);
          for (int k = 0; k < 81; ++k) {
            ex += wk(k) * r[k] * T.a[k];
            ey += wk(k) * r[k] * T.b[k];
          }
          const double det = J[0] * J[3] - J[1] * J[2];
          if (det == 0) break;
          const double dx = -(J[3] * ex - J[1] * ey) / det, dy = -(J[0] * ey - J[2] * ex) / det;
          if (!(dx * dx + dy * dy <= 4)) break; /* steps and drift stay within 2 px */
          cx += dx;
          cy += dy;
          if (!((cx - rx) * (cx - rx) + (cy - ry) * (cy - ry) <= 4)) break;
          if (dx * dx + dy * dy < tol * tol) {
            /* kept only when J is well conditioned: sigma_min / sigma_max >= ~0.01 */
            settled = fabs(det) >= kCondMin * (J[0] * J[0] + J[1] * J[1] + J[2] * J[2] + J[3] * J[3]);
            break;
          }
        }
        conv = settled;
      }
      L->ok = conv;
      conv = level == 0 && conv;
    }
    if (i != c->levels - 1) {
      sx = sx * 2 - 0.5;
      sy = sy * 2 - 0.5;
      cx = cx * 2 - 0.5;
      cy = cy * 2 - 0.5;
    }
  }
  R->status = conv;
  if (conv) {
    R->x = cx;
    R->y = cy;
  }
}

void or64_track(const or64_cam* c, const or_track_data* in, int n, int mode, int iters, double tol, double* out_xy,
                uint8_t* status) {
  trec* R = (trec*)malloc(sizeof(trec));
  for (int i = 0; i < n; ++i) {
    track_one(c, &in[i], mode, iters, tol, R);
    out_xy[2 * i] = R->x;
    out_xy[2 * i + 1] = R->y;
    status[i] = (uint8_t)R->status;
  }
  free(R);
}

/* ------------------------------------------------------------------ adjoint */
/* Adjoint of the template quantities of one level: P1bar, Gxbar, Gybar scattered into the level's
 * planes; returns the gradient with respect to the template position s. */
static void templ_adjoint(or64_cam* c, int level, double sx, double sy, const double* p1bar, const double* gxbar,
                          const double* gybar, double* dsx, double* dsy) {
  const int W = c->ws[level], H = c->hs[level];
  double gsx = 0, gsy = 0;
  for (int k = 0; k < 81; ++k) {
    tap64 t = tap_at(W, H, sx - 4 + k % 9, sy - 4 + k / 9);
    tscatter(c->dpimg[level], W, t, p1bar[k]);
    tscatter(c->dpgx[level], W, t, gxbar[k]);
    tscatter(c->dpgy[level], W, t, gybar[k]);
    double dx, dy;
    tgrad(c->pimg[level], W, t, &dx, &dy);
    gsx += p1bar[k] * dx;
    gsy += p1bar[k] * dy;
    tgrad(c->pgx[level], W, t, &dx, &dy);
    gsx += gxbar[k] * dx;
    gsy += gxbar[k] * dy;
    tgrad(c->pgy[level], W, t, &dx, &dy);
    gsx += gybar[k] * dx;
    gsy += gybar[k] * dy;
  }
  *dsx = gsx;
  *dsy = gsy;
}

static void backward_one(or64_cam* c, const trec* R, int mode, double gx_out, double gy_out, double* dtrack,
                         double* doffset) {
  dtrack[0] = dtrack[1] = doffset[0] = doffset[1] = 0;
  if (!R->status) return;
  templ T;
  double p2[81], r[81], p1bar[81], abar[81], bbar[81], gxbar[81], gybar[81], u[81];
  if (mode == OR64_IMPLICIT) {
    const lrec* L = &R->lv[0];
    const int W = c->ws[0], H = c->hs[0];
    make_templ(c, 0, L->sx, L->sy, &T);
    double vx, vy;
    step(c, 0, &T, R->x, R->y, p2, r, &vx, &vy);
    /* J = de/dc = sum w g (grad P2 - mean grad P2)^T */
    double dx[81], dy[81], mdx = 0, mdy = 0;
    tap64 tp[81];
    for (int k = 0; k < 81; ++k) {
      tp[k] = tap_at(W, H, R->x - 4 + k % 9, R->y - 4 + k / 9);
      tgrad(c->cimg[0], W, tp[k], &dx[k], &dy[k]);
      mdx += dx[k] / 81;
      mdy += dy[k] / 81;
    }
    double J00 = 0, J01 = 0, J10 = 0, J11 = 0;
    for (int k = 0; k < 81; ++k) {
      J00 += wk(k) * T.a[k] * (dx[k] - mdx);
      J01 += wk(k) * T.a[k] * (dy[k] - mdy);
      J10 += wk(k) * T.b[k] * (dx[k] - mdx);
      J11 += wk(k) * T.b[k] * (dy[k] - mdy);
    }
    const double det = J00 * J11 - J01 * J10;
    if (det == 0) return;
    /* J^T lambda = dL/dc */
    const double lx = (J11 * gx_out - J10 * gy_out) / det, ly = (-J01 * gx_out + J00 * gy_out) / det;
    /* dL/dtheta = -lambda^T de/dtheta */
    double mu = 0, ma = 0, mb = 0;
    for (int k = 0; k < 81; ++k) {
      u[k] = -wk(k) * (lx * T.a[k] + ly * T.b[k]);
      mu += u[k] / 81;
      abar[k] = -wk(k) * r[k] * lx;
      bbar[k] = -wk(k) * r[k] * ly;
      ma += abar[k] / 81;
      mb += bbar[k] / 81;
    }
    for (int k = 0; k < 81; ++k) {
      tscatter(c->dcimg[0], W, tp[k], u[k] - mu);
      p1bar[k] = -(u[k] - mu);
      gxbar[k] = abar[k] - ma;
      gybar[k] = bbar[k] - mb;
    }
    double dsx, dsy;
    templ_adjoint(c, 0, L->sx, L->sy, p1bar, gxbar, gybar, &dsx, &dsy);
    dtrack[0] = dsx;
    dtrack[1] = dsy;
    return;
  }
  /* unrolled */
  const int top = c->levels - 1;
  double cbx = gx_out, cby = gy_out; /* gradient with respect to the end position of the level */
  for (int level = 0; level <= top; ++level) {
    const lrec* L = &R->lv[level];
    const int W = c->ws[level], H = c->hs[level];
    if (L->processed && L->ok) {
      make_templ(c, level, L->sx, L->sy, &T);
      for (int k = 0; k < 81; ++k) p1bar[k] = abar[k] = bbar[k] = 0;
      double Hbxx = 0, Hbxy = 0, Hbyx = 0, Hbyy = 0;
      double gx = cbx, gy = cby;
      for (int t = L->K - 1; t >= 0; --t) {
        double vx, vy;
        step(c, level, &T, L->cx[t], L->cy[t], p2, r, &vx, &vy);
        const double mux = (T.hyy * gx - T.hxy * gy) / T.det, muy = (T.hxx * gy - T.hxy * gx) / T.det;
        Hbxx -= mux * vx;
        Hbxy -= mux * vy;
        Hbyx -= muy * vx;
        Hbyy -= muy * vy;
        double mu = 0;
        for (int k = 0; k < 81; ++k) {
          u[k] = wk(k) * (mux * T.a[k] + muy * T.b[k]);
          mu += u[k] / 81;
          abar[k] += wk(k) * r[k] * mux;
          bbar[k] += wk(k) * r[k] * muy;
        }
        double ngx = gx, ngy = gy;
        for (int k = 0; k < 81; ++k) {
          const double p2b = u[k] - mu;
          tap64 tp = tap_at(W, H, L->cx[t] - 4 + k % 9, L->cy[t] - 4 + k / 9);
          tscatter(c->dcimg[level], W, tp, p2b);
          double dx, dy;
          tgrad(c->cimg[level], W, tp, &dx, &dy);
          ngx += p2b * dx;
          ngy += p2b * dy;
          p1bar[k] -= p2b;
        }
        gx = ngx;
        gy = ngy;
      }
      double ma = 0, mb = 0;
      for (int k = 0; k < 81; ++k) {
        abar[k] += wk(k) * (2 * Hbxx * T.a[k] + (Hbxy + Hbyx) * T.b[k]);
        bbar[k] += wk(k) * ((Hbxy + Hbyx) * T.a[k] + 2 * Hbyy * T.b[k]);
        ma += abar[k] / 81;
        mb += bbar[k] / 81;
      }
      for (int k = 0; k < 81; ++k) {
        gxbar[k] = abar[k] - ma;
        gybar[k] = bbar[k] - mb;
      }
      double dsx, dsy;
      templ_adjoint(c, level, L->sx, L->sy, p1bar, gxbar, gybar, &dsx, &dsy);
      dtrack[0] += dsx / (double)(1 << level);
      dtrack[1] += dsy / (double)(1 << level);
      cbx = gx;
      cby = gy;
    }
    if (level < top) {
      cbx *= 2;
      cby *= 2;
    }
  }
  const double scale = 1.0 / (double)(1 << top);
  dtrack[0] += cbx * scale;
  dtrack[1] += cby * scale;
  doffset[0] = cbx * scale;
  doffset[1] = cby * scale;
}

/* Test hook: or64_backward stops before the pyramid adjoint, leaving the per-level record sums in
 * the planes that or64_cam_adjoint_plane reads. */
static int g_skip_pyramid_adjoint = 0;
void or64_debug_skip_pyramid_adjoint(int on) { g_skip_pyramid_adjoint = on; }

/* level `level` adjoint plane: 0 previous image, 1 previous grad_x, 2 previous grad_y, 3 current image */
void or64_cam_adjoint_plane(const or64_cam* c, int level, int plane, double* out) {
  const double* src = plane == 0 ? c->dpimg[level] : plane == 1 ? c->dpgx[level] : plane == 2 ? c->dpgy[level] : c->dcimg[level];
  memcpy(out, src, sizeof(double) * c->ws[level] * c->hs[level]);
}

/* Vector-Jacobian product: grad_xy (n x 2) is dL/d(output position) of each track; the outputs are
 * dL/d(level-0 previous image), dL/d(level-0 current image) (w x h each), dL/d(track position) and
 * dL/d(offset) (n x 2 each).  Tracks that fail contribute nothing. */
void or64_backward(or64_cam* c, const or_track_data* in, int n, int mode, int iters, double tol,
                   const double* grad_xy, double* grad_prev0, double* grad_cur0, double* grad_track,
                   double* grad_offset) {
  for (int l = 0; l < c->levels; ++l) {
    size_t np = (size_t)c->ws[l] * c->hs[l];
    memset(c->dpimg[l], 0, np * sizeof(double));
    memset(c->dpgx[l], 0, np * sizeof(double));
    memset(c->dpgy[l], 0, np * sizeof(double));
    memset(c->dcimg[l], 0, np * sizeof(double));
  }
  trec* R = (trec*)malloc(sizeof(trec));
  for (int i = 0; i < n; ++i) {
    track_one(c, &in[i], mode, iters, tol, R);
    double dt[2], dof[2];
    backward_one(c, R, mode, grad_xy[2 * i], grad_xy[2 * i + 1], dt, dof);
    if (grad_track) {
      grad_track[2 * i] = dt[0];
      grad_track[2 * i + 1] = dt[1];
    }
    if (grad_offset) {
      grad_offset[2 * i] = dof[0];
      grad_offset[2 * i + 1] = dof[1];
    }
  }
  free(R);
  if (g_skip_pyramid_adjoint) return;
  /* pyramid adjoint: gradients, then decimation, from the top level down */
  for (int l = c->levels - 1; l >= 0; --l) {
    grad64_adj(c->dpgx[l], c->dpgy[l], c->ws[l], c->hs[l], c->dpimg[l]);
    if (l > 0) {
      down64_adj(c->dpimg[l], c->ws[l], c->hs[l], c->dpimg[l - 1], c->ws[l - 1], c->hs[l - 1]);
      down64_adj(c->dcimg[l], c->ws[l], c->hs[l], c->dcimg[l - 1], c->ws[l - 1], c->hs[l - 1]);
    }
  }
  memcpy(grad_prev0, c->dpimg[0], sizeof(double) * c->ws[0] * c->hs[0]);
  memcpy(grad_cur0, c->dcimg[0], sizeof(double) * c->ws[0] * c->hs[0]);
}

/* A track's discrete decisions: status, and per level whether it was set up and accepted and how
 * many steps it took. */
static uint64_t decisions(const trec* R) {
  uint64_t h = 1469598103934665603ull ^ (uint64_t)R->status;
  for (int l = 0; l < L64_MAX_LEVELS; ++l) {
    h = (h ^ (uint64_t)(R->lv[l].processed + 2 * R->lv[l].ok)) * 1099511628211ull;
    h = (h ^ (uint64_t)R->lv[l].K) * 1099511628211ull;
  }
  return h;
}

/* Mean squared distance to gt over the tracks in `mask` (tracks the caller counts), divided by n:
 * L = sum_{mask} |c_i - gt_i|^2 / n.  Sets *flipped when a masked track fails, or, given base
 * (one value per track), when its decisions differ from base's. */
static double mse(const or64_cam* c, const or_track_data* in, int n, int mode, int iters, double tol,
                  const double* gt, const uint8_t* mask, int* flipped, const uint64_t* base) {
  trec* R = (trec*)malloc(sizeof(trec));
  double L = 0;
  for (int i = 0; i < n; ++i) {
    if (!mask[i]) continue;
    track_one(c, &in[i], mode, iters, tol, R);
    if (base && decisions(R) != base[i]) *flipped = 1;
    if (!R->status) {
      *flipped = 1;
      continue;
    }
    const double dx = R->x - gt[2 * i], dy = R->y - gt[2 * i + 1];
    L += dx * dx + dy * dy;
  }
  free(R);
  return L / n;
}

/* Central finite differences of the loss above.  which[q]: 0 previous-image pixel index[q],
 * 1 current-image pixel index[q], 2 / 3 x / y of track index[q]'s position.  out[q] is NaN where
 * a perturbation changed which tracks succeed, or, with strict != 0, any counted track's decisions
 * (levels set up and accepted, steps per level): the loss then jumps and the difference is not a
 * derivative. */
void or64_fd(or64_cam* c, const double* prev0, const double* cur0, const or_track_data* in, int n, int mode,
             int iters, double tol, const double* gt, const uint8_t* mask, int nq, const int* which,
             const int64_t* index, double h, double* out, int strict) {
  uint64_t* base = NULL;
  if (strict) {
    base = (uint64_t*)calloc(n > 0 ? n : 1, sizeof(uint64_t));
    trec* R = (trec*)malloc(sizeof(trec));
    for (int i = 0; i < n; ++i)
      if (mask[i]) {
        track_one(c, &in[i], mode, iters, tol, R);
        base[i] = decisions(R);
      }
    free(R);
  }
  const size_t np = (size_t)c->ws[0] * c->hs[0];
  double* p = (double*)malloc(np * sizeof(double));
  double* q = (double*)malloc(np * sizeof(double));
  or_track_data* tr = (or_track_data*)malloc(sizeof(or_track_data) * (n > 0 ? n : 1));
  memcpy(p, prev0, np * sizeof(double));
  memcpy(q, cur0, np * sizeof(double));
  memcpy(tr, in, sizeof(or_track_data) * n);
  for (int k = 0; k < nq; ++k) {
    double lv[2];
    int flipped = 0;
    for (int sgn = 0; sgn < 2; ++sgn) {
      const double d = sgn ? -h : h;
      double save = 0;
      float fsave = 0;
      if (which[k] == 0) {
        save = p[index[k]];
        p[index[k]] = save + d;
      } else if (which[k] == 1) {
        save = q[index[k]];
        q[index[k]] = save + d;
      } else {
        fsave = tr[index[k]].track[which[k] - 2];
        tr[index[k]].track[which[k] - 2] = (float)(fsave + d);
      }
      if (which[k] <= 1) or64_cam_set(c, p, q);
      lv[sgn] = mse(c, tr, n, mode, iters, tol, gt, mask, &flipped, which[k] <= 1 ? base : NULL);
      if (which[k] == 0) p[index[k]] = save;
      else if (which[k] == 1) q[index[k]] = save;
      else tr[index[k]].track[which[k] - 2] = fsave;
    }
    if (which[k] <= 1) or64_cam_set(c, p, q);
    /* a track position perturbed in FP32 moves by the rounded step, not by h */
    double step = 2 * h;
    if (which[k] >= 2) {
      const float base = in[index[k]].track[which[k] - 2];
      step = (double)(float)(base + h) - (double)(float)(base - h);
    }
    out[k] = flipped ? NAN : (lv[0] - lv[1]) / step;
  }
  or64_cam_set(c, prev0, cur0);
  free(p);
  free(q);
  free(tr);
  free(base);
}
