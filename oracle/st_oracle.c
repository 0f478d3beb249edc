/* CPU oracle of the affine (Shi-Tomasi) feature tracker: st_track_kernel, st_build_cache_kernel and
 * st_track_with_cache_kernel (libs/cuda_modules/cuda_kernels/st_tracker.cu:320-1370).
 *
 * TEST INFRASTRUCTURE ONLY (see fe_oracle.h).  The reference runs one thread per track and sums the
 * 81 patch taps sequentially; this restatement keeps the reference's algorithm (coarse-to-fine
 * levels, shift-only then full affine Gauss-Newton steps on mean-subtracted current-frame gradients,
 * the 2x2 convergence test |v| < 0.04, column-pivoting Householder QR solves, 5x5 NCC gate) but sums
 * in the CUDA kernel's order (lane-major partial sums over taps lane, lane+32, lane+64, then an
 * xor butterfly over 32 lanes), so that the kernel can be compared bit for bit; against the
 * reference the agreement is within float tolerance (tests/golden).  Arithmetic is FP32 without
 * contraction (-ffp-contract=off); the kernel writes the same operations unfused. */
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "fe_oracle.h"

#define PD 9
#define PS 81
#define NE 3

static const float kG9[9] = {0.0135196f, 0.0476622f, 0.11723f, 0.201168f, 0.240841f,
                             0.201168f,  0.11723f,   0.0476622f, 0.0135196f};
static const float kEps = 1.1920928955078125e-07f;

static float bfly(const float* lanes) {
  float t[32], u[32];
  memcpy(t, lanes, sizeof(t));
  for (int m = 1; m < 32; m <<= 1) {
    for (int l = 0; l < 32; ++l) u[l] = t[l] + t[l ^ m];
    memcpy(t, u, sizeof(t));
  }
  return t[0];
}

/* sum over the 81 taps of v[f] (f valid) in the kernel's order */
static float tap_sum(const float* v, const uint8_t* use) {
  float lanes[32];
  for (int l = 0; l < 32; ++l) {
    float a = 0.f;
    for (int e = 0; e < NE; ++e) {
      const int f = l + 32 * e;
      if (f < PS && (!use || use[f])) a = a + v[f];
    }
    lanes[l] = a;
  }
  return bfly(lanes);
}

static int in_image(float x, float y, int w, int h) { return x >= 0.f && x < (float)w && y >= 0.f && y < (float)h; }

/* ColPivHouseholderQR + solve (st_tracker.cu:50-244): Householder QR with column pivoting by the
 * largest (down-dated) column norm, the reference's norm down-dating and re-computation rule, its
 * rank rule (nonzero pivots: the first step whose pivot norm^2 < (max_norm eps)^2 / D * (D - q)), its
 * reflector (v_q = c0 - sign-adjusted norm, tau = 1 / (norm^2 + c0 norm), 0 when that is below eps),
 * Q^T b applied reflector by reflector, back substitution over the nonzero pivots (a zero diagonal
 * with a nonzero right side fails), and the column permutation undone.  a: row-major D x D. */
int or_st_qr_solve(int D, const float* a, const float* b, float* x) {
  float R[36], qb[6], cn[6], cnd[6];
  int perm[6];
  memcpy(R, a, sizeof(float) * D * D);
  memcpy(qb, b, sizeof(float) * D);
  float max_norm = -1.f;
  for (int c = 0; c < D; ++c) {
    float s = 0.f;
    for (int r = 0; r < D; ++r) s = s + R[r * D + c] * R[r * D + c];
    cn[c] = sqrtf(s);
    cnd[c] = cn[c];
    if (cn[c] > max_norm) max_norm = cn[c];
    perm[c] = c;
  }
  float th = max_norm * kEps;
  th = th * th / (float)D;
  int nzp = D;
  for (int q = 0; q < D - 1; ++q) {
    float mn = -1.f;
    int mc = -1;
    for (int c = q; c < D; ++c)
      if (cn[c] > mn) {
        mn = cn[c];
        mc = c;
      }
    if (nzp == D && mn * mn < th * (float)(D - q)) nzp = q;
    if (mc >= 0 && q != mc) { /* mc < 0: no column norm above -1 (all NaN), nothing to swap */
      int t = perm[q];
      perm[q] = perm[mc];
      perm[mc] = t;
      float f = cn[q];
      cn[q] = cn[mc];
      cn[mc] = f;
      f = cnd[q];
      cnd[q] = cnd[mc];
      cnd[mc] = f;
      for (int r = 0; r < D; ++r) {
        f = R[r * D + q];
        R[r * D + q] = R[r * D + mc];
        R[r * D + mc] = f;
      }
    }
    const float c0 = R[q * D + q];
    if (c0 >= 0.f) mn = -mn;
    const float div = mn * mn + c0 * mn;
    float tau = 1.f / div;
    if (fabsf(div) < kEps) tau = 0.f;
    float v[6];
    for (int r = 0; r < D; ++r) v[r] = r < q ? 0.f : R[r * D + q];
    v[q] = c0 + mn;
    /* R <- (I - tau v v^T) R on rows q.., and the same on Q^T b */
    for (int c = 0; c < D; ++c) {
      float s = 0.f;
      for (int r = q; r < D; ++r) s = s + v[r] * R[r * D + c];
      const float ts = tau * s;
      for (int r = q; r < D; ++r) R[r * D + c] = R[r * D + c] - ts * v[r];
    }
    {
      float s = 0.f;
      for (int r = q; r < D; ++r) s = s + v[r] * qb[r];
      const float ts = tau * s;
      for (int r = q; r < D; ++r) qb[r] = qb[r] - ts * v[r];
    }
    for (int c = q + 1; c < D; ++c) {
      if (cn[c] != 0.f) {
        float t = fabsf(R[q * D + c]) / cn[c];
        t = (1.f + t) * (1.f - t);
        if (t < 0.f) t = 0.f;
        const float rr = cn[c] / cnd[c];
        const float t2 = t * rr * rr;
        if (t2 <= kEps) {
          float s = 0.f;
          for (int r = q + 1; r < D; ++r) s = s + R[r * D + c] * R[r * D + c];
          cnd[c] = sqrtf(s);
          cn[c] = cnd[c];
        } else {
          cn[c] = cn[c] * sqrtf(t);
        }
      }
    }
  }
  for (int i = nzp - 1; i >= 0; --i) {
    if (fabsf(R[i * D + i]) < kEps) {
      if (fabsf(qb[i]) > kEps) return 0;
    } else {
      qb[i] = qb[i] / R[i * D + i];
    }
    for (int j = i - 1; j >= 0; --j) qb[j] = qb[j] - qb[i] * R[j * D + i];
  }
  for (int i = 0; i < D; ++i) x[perm[i]] = qb[i];
  return 1;
}

/* the patch tap f of an identity-mapped patch with top-left sample (xmin, ymin), or of the affine
 * patch whose first tap is (x00, y00): sample coordinates, and whether the affine tap is inside */
static int tap_pos(int f, int identity, float xmin, float ymin, float x00, float y00, const float* m, int w, int h,
                   float* sx, float* sy) {
  const int ix = f % PD, iy = f / PD;
  if (identity) {
    *sx = xmin + (float)ix;
    *sy = ymin + (float)iy;
    return 1;
  }
  const float x = (x00 + m[0] * (float)ix) + m[1] * (float)iy;
  const float y = (y00 + m[2] * (float)ix) + m[3] * (float)iy;
  if (x < 0.f || x >= (float)w || y < 0.f || y >= (float)h) return 0;
  *sx = x + 0.5f;
  *sy = y + 0.5f;
  return 1;
}

static int is_identity(const float* m) { return m[0] == 1.f && m[1] == 0.f && m[2] == 0.f && m[3] == 1.f; }

/* Samples the current patch (image, grad_x, grad_y) at map m around (cx, cy); 0 when out of the image. */
static int sample_current(const float* img, const float* gxi, const float* gyi, int w, int h, float cx, float cy,
                          const float* m, int mode, float* p, float* gx, float* gy) {
  const int id = is_identity(m);
  float xmin = 0.f, ymin = 0.f, x00 = 0.f, y00 = 0.f;
  if (id) {
    xmin = (cx - 4.5f) + 0.5f;
    ymin = (cy - 4.5f) + 0.5f;
    if (xmin < 0.f || xmin + (float)PD >= (float)w || ymin < 0.f || ymin + (float)PD >= (float)h) return 0;
  } else {
    x00 = (cx - 0.5f) - (8.f * (m[0] + m[1])) / 2.f;
    y00 = (cy - 0.5f) - (8.f * (m[2] + m[3])) / 2.f;
  }
  for (int f = 0; f < PS; ++f) {
    float sx, sy;
    if (!tap_pos(f, id, xmin, ymin, x00, y00, m, w, h, &sx, &sy)) return 0;
    p[f] = or_tex_sample(img, w, h, sx, sy, mode);
    if (gx) gx[f] = or_tex_sample(gxi, w, h, sx, sy, mode);
    if (gy) gy[f] = or_tex_sample(gyi, w, h, sx, sy, mode);
  }
  return 1;
}

/* previous patch of a track at level position (u, v); 0 when its box leaves the image */
static int sample_previous(const float* img, int w, int h, float u, float v, int mode, float* p, float* sum) {
  const float xmin = (u - 4.5f) + 0.5f, ymin = (v - 4.5f) + 0.5f;
  if (xmin < 0.f || xmin + (float)PD >= (float)w || ymin < 0.f || ymin + (float)PD >= (float)h) return 0;
  for (int f = 0; f < PS; ++f) p[f] = or_tex_sample(img, w, h, xmin + (float)(f % PD), ymin + (float)(f / PD), mode);
  *sum = tap_sum(p, NULL);
  return 1;
}

typedef struct {
  float xy[2], map[4];
  int converged;
} st_state;

/* Gauss-Newton refinement of (xy, map) against the previous patch (st_tracker.cu:398-643): returns 0
 * when a patch leaves the image or a solve fails. */
static int refine(const float* img, const float* gxi, const float* gyi, int w, int h, const float* prev, float prev_sum,
                  int n_shift, int n_full, int mode, st_state* s) {
  float m[4], cx = s->xy[0], cy = s->xy[1];
  memcpy(m, s->map, sizeof(m));
  float p[PS], gx[PS], gy[PS], r[PS], wt[PS], t[PS];
  for (int f = 0; f < PS; ++f) wt[f] = kG9[f / PD] * kG9[f % PD];
  for (int it = 0; it < n_shift + n_full; ++it) {
    const int full = it >= n_shift;
    if (!in_image(cx, cy, w, h)) return 0;
    if (!sample_current(img, gxi, gyi, w, h, cx, cy, m, mode, p, gx, gy)) return 0;
    const float cs = tap_sum(p, NULL), gxs = tap_sum(gx, NULL), gys = tap_sum(gy, NULL);
    const float delta = (cs - prev_sum) / 81.f, gxm = gxs / 81.f, gym = gys / 81.f;
    for (int f = 0; f < PS; ++f) {
      gx[f] = gx[f] - gxm;
      gy[f] = gy[f] - gym;
      r[f] = (p[f] - prev[f]) - delta;
    }
#define SUM(expr) (({ for (int f = 0; f < PS; ++f) t[f] = (expr); }), tap_sum(t, NULL))
    const float sxx = SUM((wt[f] * gx[f]) * gx[f]), sxy = SUM((wt[f] * gx[f]) * gy[f]);
    const float syy = SUM((wt[f] * gy[f]) * gy[f]);
    const float rx = SUM((wt[f] * r[f]) * gx[f]), ry = SUM((wt[f] * r[f]) * gy[f]);
    const float det = sxx * syy - sxy * sxy;
    const float vx = (syy * rx - sxy * ry) / det, vy = (sxx * ry - sxy * rx) / det;
    s->converged = sqrtf(vx * vx + vy * vy) < 0.04f;
    if (s->converged) break;
    if (full) {
      /* moments of g g^T against 1, x, y, x^2, xy, y^2 over the window (x, y = tap offset from the centre) */
      float mm[6][3], rr[4];
      mm[0][0] = sxx;  /* the unweighted-by-position moments are the ones of the convergence test */
      mm[0][1] = sxy;
      mm[0][2] = syy;
      for (int k = 1; k < 6; ++k) {
        for (int c = 0; c < 3; ++c) {
          for (int f = 0; f < PS; ++f) {
            const float ox = (float)(f % PD - 4), oy = (float)(f / PD - 4);
            const float pw = k == 1 ? ox : k == 2 ? oy : k == 3 ? ox * ox : k == 4 ? ox * oy : oy * oy;
            const float g = c == 0 ? gx[f] * gx[f] : c == 1 ? gx[f] * gy[f] : gy[f] * gy[f];
            t[f] = (pw * wt[f]) * g;
          }
          mm[k][c] = tap_sum(t, NULL);
        }
      }
      for (int k = 0; k < 4; ++k) {
        for (int f = 0; f < PS; ++f) {
          const float ox = (float)(f % PD - 4), oy = (float)(f / PD - 4);
          const float pw = (k < 2 ? ox : oy) * wt[f];
          t[f] = (r[f] * pw) * (k % 2 == 0 ? gx[f] : gy[f]);
        }
        rr[k] = tap_sum(t, NULL);
      }
      /* normal equations of (dxx, dyx, dxy, dyy, dx, dy), the reference's layout */
      const float A[36] = {mm[3][0], mm[3][1], mm[4][0], mm[4][1], mm[1][0], mm[1][1],
                           mm[3][1], mm[3][2], mm[4][1], mm[4][2], mm[1][1], mm[1][2],
                           mm[4][0], mm[4][1], mm[5][0], mm[5][1], mm[2][0], mm[2][1],
                           mm[4][1], mm[4][2], mm[5][1], mm[5][2], mm[2][1], mm[2][2],
                           mm[1][0], mm[1][1], mm[2][0], mm[2][1], mm[0][0], mm[0][1],
                           mm[1][1], mm[1][2], mm[2][1], mm[2][2], mm[0][1], mm[0][2]};
      const float bvec[6] = {rr[0], rr[1], rr[2], rr[3], rx, ry};
      float z[6];
      if (!or_st_qr_solve(6, A, bvec, z)) return 0;
      m[0] = m[0] + z[0];
      m[1] = m[1] + z[1];
      m[2] = m[2] + z[2];
      m[3] = m[3] + z[3];
      cx = cx + z[4];
      cy = cy + z[5];
    } else {
      const float A[4] = {sxx, sxy, sxy, syy}, bvec[2] = {rx, ry};
      float z[2];
      if (!or_st_qr_solve(2, A, bvec, z)) return 0;
      cx = cx + z[0];
      cy = cy + z[1];
    }
#undef SUM
  }
  if (!in_image(cx, cy, w, h)) return 0;
  s->xy[0] = cx;
  s->xy[1] = cy;
  memcpy(s->map, m, sizeof(m));
  return 1;
}

/* 5x5 NCC of the final patch against the previous one (st_tracker.cu:744-790) */
static float ncc5(const float* cur, const float* prev) {
  uint8_t use[PS];
  float t[PS];
  for (int f = 0; f < PS; ++f) use[f] = f % PD >= 2 && f % PD < 7 && f / PD >= 2 && f / PD < 7;
  const float cs = tap_sum(cur, use), ps = tap_sum(prev, use);
  for (int f = 0; f < PS; ++f) t[f] = cur[f] * cur[f];
  const float css = tap_sum(t, use);
  for (int f = 0; f < PS; ++f) t[f] = prev[f] * prev[f];
  const float pss = tap_sum(t, use);
  for (int f = 0; f < PS; ++f) t[f] = cur[f] * prev[f];
  const float cps = tap_sum(t, use);
  const float cm = cs / 25.f, pm = ps / 25.f;
  const float cv = css / 25.f - cm * cm, pv = pss / 25.f - pm * pm, cov = cps / 25.f - cm * pm;
  const float d = cv * pv;
  return d < kEps ? 0.f : cov / sqrtf(d);
}

static void scale_up(float* v) {
  v[0] = v[0] * 2.f - 0.5f;
  v[1] = v[1] * 2.f - 0.5f;
}

/* One track; cache == NULL: st_track_kernel (previous patches from prev_img), else
 * st_track_with_cache_kernel (previous patches from the cache entry). */
static void st_one(int levels, const int* ws, const int* hs, const float* const* prev_img,
                   const float* const* cur_img, const float* const* cur_gx, const float* const* cur_gy,
                   const or_st_cache* cache, or_track_data* td, int n_shift, int n_full, int mode) {
  const or_st_cache* cd = NULL;
  if (cache) {
    if (td->cache_index == -1) {
      td->track_status = 0;
      return;
    }
    cd = &cache[td->cache_index];
  }
  if (td->search_radius_px < 0.f) {
    td->track_status = 0;
    return;
  }
  int top = (int)log1pf(td->search_radius_px);
  if (levels - 1 < top) top = levels - 1;
  if (!cache && !in_image(td->track[0], td->track[1], ws[0], hs[0])) {
    td->track_status = 0;
    return;
  }
  const float scale = 1.f / (float)(1 << top);
  float pu[2] = {(td->track[0] - 0.5f) * scale + 0.5f, (td->track[1] - 0.5f) * scale + 0.5f};
  st_state s;
  memcpy(s.map, td->initial_guess_map, sizeof(s.map));
  s.xy[0] = ((td->track[0] + td->offset[0]) - 0.5f) * scale + 0.5f;
  s.xy[1] = ((td->track[1] + td->offset[1]) - 0.5f) * scale + 0.5f;
  s.converged = 0;
  float prev[PS], cur[PS];
  for (int level = top; level >= 0; --level) {
    const int w = ws[level], h = hs[level];
    if (!cache && !in_image(pu[0], pu[1], w, h)) {
      td->track_status = 0;
      return;
    }
    if (!in_image(s.xy[0], s.xy[1], w, h)) {
      td->track_status = 0;
      return;
    }
    float prev_sum = 0.f;
    int have_prev;
    if (cache) {
      have_prev = (cd->level_mask >> level) & 1u;
      if (!have_prev && level > 0) {
        scale_up(s.xy);
        scale_up(pu);
        continue;
      }
      memcpy(prev, cd->patch + PS * level, sizeof(prev));
      prev_sum = cd->patch_sums[level];
      have_prev = 1;  /* level 0 uses the entry's level-0 patch whatever its mask says */
    } else {
      have_prev = sample_previous(prev_img[level], w, h, pu[0], pu[1], mode, prev, &prev_sum);
      if (!have_prev && level > 0) {
        scale_up(s.xy);
        scale_up(pu);
        continue;
      }
    }
    td->info[0] = 1.f / 9.f;
    td->info[1] = 0.f;
    td->info[2] = 0.f;
    td->info[3] = 1.f / 9.f;
    int ok = have_prev && refine(cur_img[level], cur_gx[level], cur_gy[level], w, h, prev, prev_sum, n_shift, n_full,
                                 mode, &s);
    if (!ok) {
      if (level > 0) {
        scale_up(s.xy);
        scale_up(pu);
        continue;
      }
      td->track_status = 0;
      return;
    }
    if (!sample_current(cur_img[level], NULL, NULL, w, h, s.xy[0], s.xy[1], s.map, mode, cur, NULL, NULL)) {
      td->track_status = 0;
      return;
    }
    if (level == 0) {
      const float c = ncc5(cur, prev);
      if (c <= td->ncc_threshold || !s.converged) {
        td->track_status = 0;
        return;
      }
      td->ncc = c;
    } else {
      scale_up(s.xy);
      scale_up(pu);
    }
  }
  td->track[0] = s.xy[0];
  td->track[1] = s.xy[1];
  td->track_status = in_image(s.xy[0], s.xy[1], ws[0], hs[0]);
}

void or_st_track(int levels, const int* ws, const int* hs, const float* const* prev_img, const float* const* cur_img,
                 const float* const* cur_gx, const float* const* cur_gy, or_track_data* td, int n, int n_shift,
                 int n_full, int mode) {
  for (int i = 0; i < n; ++i) st_one(levels, ws, hs, prev_img, cur_img, cur_gx, cur_gy, NULL, &td[i], n_shift, n_full, mode);
}

void or_st_track_cached(int levels, const int* ws, const int* hs, const float* const* cur_img,
                        const float* const* cur_gx, const float* const* cur_gy, const or_st_cache* cache,
                        or_track_data* td, int n, int n_shift, int n_full, int mode) {
  for (int i = 0; i < n; ++i) st_one(levels, ws, hs, NULL, cur_img, cur_gx, cur_gy, cache, &td[i], n_shift, n_full, mode);
}

/* st_build_cache_kernel (st_tracker.cu:1298-1371): each track's previous patches on every level whose
 * box lies inside the image, their sums, the level mask; cache_index = the track's index. */
void or_st_build_cache(int levels, const int* ws, const int* hs, const float* const* prev_img, or_track_data* td, int n,
                       or_st_cache* cache, int mode) {
  for (int i = 0; i < n; ++i) {
    or_st_cache* c = &cache[i];
    if (levels == 0) {
      td[i].cache_index = -1;
      continue;
    }
    int level = levels - 1;
    const float scale = 1.f / (float)(1 << level);
    float pu[2] = {(td[i].track[0] - 0.5f) * scale + 0.5f, (td[i].track[1] - 0.5f) * scale + 0.5f};
    c->level_mask = 0;
    for (;; --level) {
      if (in_image(pu[0], pu[1], ws[level], hs[level])) {
        float sum;
        if (sample_previous(prev_img[level], ws[level], hs[level], pu[0], pu[1], mode, c->patch + PS * level, &sum)) {
          c->patch_sums[level] = sum;
          c->level_mask |= 1u << level;
        }
      }
      if (level > 0) scale_up(pu);
      if (level == 0) break;
    }
    td[i].cache_index = i;
  }
}
