"""ctypes front for the CPU oracle (oracle/liboracle.so).  TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this module, as the
checker.  The product (cuvslam_b200) never imports it.
"""

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

P = ctypes.c_void_p
I = ctypes.c_int
F = ctypes.c_float

TEXTURE = 0
EXACT = 1
TEXTURE_WIDE = 2  # texture weights, each 4-tap sum rounded once (closest to the texture unit)


def build():
    subprocess.check_call(["make", "-s", "-C", HERE])


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        L.or_level_sizes.argtypes = [I, I, I, P, P]
        L.or_cast_u8.argtypes = [P, I, I, P]
        L.or_gauss_downscale.argtypes = [P, I, I, P, I, I]
        L.or_rgb_to_gray.argtypes = [P, I, I, ctypes.c_int64, P, I]
        L.or_finish_tracks.argtypes = [P, P, I, P, I, I, P, P, ctypes.c_int64, I]
        L.or_st_qr_solve.argtypes = [I, P, P, P]
        L.or_st_qr_solve.restype = I
        L.or_st_track.argtypes = [I, P, P, P, P, P, P, P, I, I, I, I]
        L.or_st_track_cached.argtypes = [I, P, P, P, P, P, P, P, I, I, I, I]
        L.or_st_build_cache.argtypes = [I, P, P, P, P, I, P, I]
        L.or_finish_tracks.restype = I
        L.or_box3.argtypes = [P, I, I, P]
        L.or_gradients.argtypes = [P, I, I, P, P]
        L.or_gftt_response.argtypes = [P, P, I, I, P]
        L.or_bins.argtypes = [P, I, I, P]
        L.or_select.argtypes = [P, I, I, P, I, I, I, I, I, I, P, P, P, P, P, P, P, P]
        L.or_select.restype = I
        L.or_tex_sample.argtypes = [P, I, I, F, F, I]
        L.or_tex_sample.restype = F
        L.or_lk_track.argtypes = [I, P, P, P, P, P, P, P, I, I]
        L.or_lk_track_horizontal.argtypes = [I, P, P, P, P, P, P, I, I]
        L.or_lk_track_f64.argtypes = [I, P, P, P, P, P, P, P, I]
        L.or_epipolar_candidates.argtypes = [I, I, F, P, P, F, F, P, I]
        L.or_epipolar_candidates.restype = I
        L.or_stereo_scan.argtypes = [I, P, P, P, P, P, P, P, P, I, P, P, F, F, F, I, I, P, P, P]
        for name, args, res in _CPU_SIGS:
            fn = getattr(L, name, None)
            if fn is None:
                continue
            fn.argtypes = args
            fn.restype = res
        _LIB = L
    return _LIB


# CPU-semantics (cuVSLAM use_gpu=false) entry points, see cpu_tracker.c
_CPU_SIGS = [
    ("cpu_cam_create", [I, I], P),
    ("cpu_cam_destroy", [P], None),
    ("cpu_cam_build", [P, P], None),
    ("cpu_cam_build_ex", [P, P, I], None),
    ("cpu_cam_patch", [P, I, F, F, P], I),
    ("cpu_cam_levels", [P], I),
    ("cpu_cam_level", [P, I, P, P, P, P, P], None),
    ("cpu_cam_track", [P, P, P, P, I, P, P], I),
    ("cpu_cam_select", [P, P, I, I, I, I, I, I, P], I),
    ("cpu_frame_step", [P, P, P, P, P, P, P, P, P, P, P, I, I], I),
    ("cpu_frame_step_features", [P, P, P, P, P, P, P, P, P, P, P, I, I], I),
]


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def level_sizes(w, h, max_levels=10):
    ws = np.zeros(10, np.int32)
    hs = np.zeros(10, np.int32)
    n = lib().or_level_sizes(w, h, max_levels, _p(ws), _p(hs))
    return list(zip(ws[:n].tolist(), hs[:n].tolist()))


def pyramid(img_u8, max_levels=10):
    """[(level image, gx, gy)] for the reference GPU pyramid + gradient pyramid."""
    img_u8 = np.ascontiguousarray(img_u8, np.uint8)
    h, w = img_u8.shape
    L = lib()
    out = []
    prev = np.zeros((h, w), np.float32)
    L.or_cast_u8(_p(img_u8), w, h, _p(prev))
    for i, (lw, lh) in enumerate(level_sizes(w, h, max_levels)):
        if i > 0:
            nxt = np.zeros((lh, lw), np.float32)
            L.or_gauss_downscale(_p(prev), prev.shape[1], prev.shape[0], _p(nxt), lw, lh)
            prev = nxt
        gx = np.zeros_like(prev)
        gy = np.zeros_like(prev)
        L.or_gradients(_p(prev), lw, lh, _p(gx), _p(gy))
        out.append((prev, gx, gy))
    return out


def pyramid_f32(img_f32, max_levels=10):
    """Same as `pyramid` but from a float32 base level."""
    prev = np.ascontiguousarray(img_f32, np.float32)
    h, w = prev.shape
    L = lib()
    out = []
    for i, (lw, lh) in enumerate(level_sizes(w, h, max_levels)):
        if i > 0:
            nxt = np.zeros((lh, lw), np.float32)
            L.or_gauss_downscale(_p(prev), prev.shape[1], prev.shape[0], _p(nxt), lw, lh)
            prev = nxt
        gx = np.zeros_like(prev)
        gy = np.zeros_like(prev)
        L.or_gradients(_p(prev), lw, lh, _p(gx), _p(gy))
        out.append((prev, gx, gy))
    return out


RGB_VARIANT = 2  # the reference kernel computes fma(0.114, b, fma(0.299, r, 0.587 g)) (pinned by the tests)


def rgb_to_gray(rgb, variant=None):
    """(h, w, 3) uint8 -> (h, w) float32 as cast_image_kernel_rgb computes it."""
    rgb = np.ascontiguousarray(rgb, np.uint8)
    h, w, _ = rgb.shape
    out = np.zeros((h, w), np.float32)
    lib().or_rgb_to_gray(_p(rgb), w, h, w * 3, _p(out), RGB_VARIANT if variant is None else variant)
    return out


def box3(img_f32):
    """The reference's box prefilter of a float32 level 0."""
    img = np.ascontiguousarray(img_f32, np.float32)
    h, w = img.shape
    out = np.zeros_like(img)
    lib().or_box3(_p(img), w, h, _p(out))
    return out


def level0(img, box=False):
    """The pyramid's level 0 from a (h, w) uint8 mono or (h, w, 3) uint8 RGB frame, optionally box
    prefiltered (ImageContext::build_gpu_image_pyramid + GaussianGPUImagePyramid::build)."""
    img = np.asarray(img)
    base = rgb_to_gray(img) if img.ndim == 3 else img.astype(np.float32)
    return box3(base) if box else base


def gftt(gx, gy):
    gx = np.ascontiguousarray(gx, np.float32)
    gy = np.ascontiguousarray(gy, np.float32)
    h, w = gx.shape
    r = np.zeros((h, w), np.float32)
    lib().or_gftt_response(_p(gx), _p(gy), w, h, _p(r))
    return r


def bins(resp):
    resp = np.ascontiguousarray(resp, np.float32)
    h, w = resp.shape
    b = np.zeros(64, np.float32)
    lib().or_bins(_p(resp), w, h, _p(b))
    return b


def select(resp, alive=None, num_desired=450, borders=(0, 0, 0, 0), mask=None):
    resp = np.ascontiguousarray(resp, np.float32)
    h, w = resp.shape
    cw, ch = w // 8, h // 8
    cap = max(cw * ch, 1)
    alive = np.zeros((0, 2), np.float32) if alive is None else np.ascontiguousarray(alive, np.float32).reshape(-1, 2)
    nms = np.zeros((h, w), np.float32)
    cmax = np.zeros(cap, np.float32)
    cidx = np.zeros(2 * cap, np.uint32)
    kp = np.zeros(3 * cap, np.float32)
    b = np.zeros(64, np.float32)
    sel = np.zeros(2 * max(num_desired, 1), np.float32)
    nkp = ctypes.c_int(0)
    m = None if mask is None else np.ascontiguousarray(mask, np.uint8)
    n = lib().or_select(_p(resp), w, h, _p(alive), len(alive), num_desired, borders[0], borders[1], borders[2],
                        borders[3], None if m is None else _p(m), _p(nms), _p(cmax), _p(cidx), _p(kp),
                        ctypes.byref(nkp), _p(b), _p(sel))
    return dict(nms=nms, cell_max=cmax[:cw * ch].reshape(ch, cw), cell_idx=cidx[:2 * cw * ch].reshape(ch, cw, 2),
                kp=kp[:3 * nkp.value].reshape(-1, 3), bins=b, sel=sel[:2 * n].reshape(-1, 2))


def tex_sample(img, xy, mode=TEXTURE):
    img = np.ascontiguousarray(img, np.float32)
    h, w = img.shape
    L = lib()
    return np.array([L.or_tex_sample(_p(img), w, h, float(x), float(y), mode) for x, y in np.asarray(xy)],
                    np.float32)


def _level_ptrs(arrs):
    arrs = [np.ascontiguousarray(a, np.float32) for a in arrs]
    ptrs = (ctypes.c_void_p * 10)(*[a.ctypes.data for a in arrs])
    return arrs, ptrs


def lk(prev_pyr, cur_pyr, tracks, mode=TEXTURE, horizontal=False, f64=False):
    """Run the LK oracle; prev_pyr/cur_pyr are lists of (img, gx, gy) per level.  Returns a copy of
    `tracks` (TRACK_DTYPE records) updated as the reference kernel would."""
    t = np.ascontiguousarray(tracks.copy())
    levels = len(prev_pyr)
    ws = np.array([p[0].shape[1] for p in prev_pyr] + [0] * (10 - levels), np.int32)
    hs = np.array([p[0].shape[0] for p in prev_pyr] + [0] * (10 - levels), np.int32)
    keep1, pgx = _level_ptrs([p[1] for p in prev_pyr])
    keep2, pgy = _level_ptrs([p[2] for p in prev_pyr])
    keep3, pim = _level_ptrs([p[0] for p in prev_pyr])
    keep4, cim = _level_ptrs([p[0] for p in cur_pyr[:levels]])
    L = lib()
    if f64:
        L.or_lk_track_f64(levels, _p(ws), _p(hs), pgx, pgy, pim, cim, _p(t), len(t))
    elif horizontal:
        L.or_lk_track_horizontal(levels, _p(ws), _p(hs), pgx, pim, cim, _p(t), len(t), mode)
    else:
        L.or_lk_track(levels, _p(ws), _p(hs), pgx, pgy, pim, cim, _p(t), len(t), mode)
    del keep1, keep2, keep3, keep4
    return t


def epipolar_candidates(cw, ch, inv_scale, offsets, xy, uv, valid=None):
    """Candidate lists of the points uv (n x 2) from an epipolar table (cw x ch corners, CSR
    offsets and x, y pairs), as (offsets (n + 1,) int32, xy (m, 2) float32); points with valid == 0
    get none."""
    L = lib()
    offsets = np.ascontiguousarray(offsets, np.int32)
    xy = np.ascontiguousarray(xy, np.float32)
    uv = np.ascontiguousarray(uv, np.float32).reshape(-1, 2)
    cap = int(max(np.diff(offsets).max(initial=0), 0))
    buf = np.zeros((max(cap, 1), 2), np.float32)
    out_off = [0]
    out_xy = []
    for i, (u, v) in enumerate(uv):
        n = 0
        if valid is None or valid[i]:
            n = L.or_epipolar_candidates(cw, ch, float(inv_scale), _p(offsets), _p(xy), float(u), float(v), _p(buf), cap)
        out_xy.append(buf[:n].copy())
        out_off.append(out_off[-1] + n)
    xy_all = np.concatenate(out_xy) if out_off[-1] else np.zeros((0, 2), np.float32)
    return np.array(out_off, np.int32), xy_all.astype(np.float32)


def lk_retrack(prev_pyr, cur_pyr, tracks, retrack_ncc=0.85, mode=TEXTURE):
    """MonoSOFGPU::launch's two passes merged as collect reads them: LK with each record's threshold,
    then the tracks it lost again from their inputs with retrack_ncc (the threshold field is kept)."""
    first = lk(prev_pyr, cur_pyr, tracks, mode)
    lost = first["track_status"] == 0
    if lost.any():
        again = tracks[lost].copy()
        again["ncc_threshold"] = retrack_ncc
        again = lk(prev_pyr, cur_pyr, again, mode)
        again["ncc_threshold"] = tracks[lost]["ncc_threshold"]
        first[lost] = again
    return first


def finish_tracks(tracks, age, width, height, border=(0, 0, 0, 0), pred=None, mask=None, collapse=True):
    """The finish filters (or_finish_tracks) on copies: returns (records, ages, alive count)."""
    t = np.ascontiguousarray(tracks.copy())
    a = np.ascontiguousarray(np.asarray(age, np.uint32).copy())
    pp = None
    if pred is not None:
        pred = np.ascontiguousarray(pred, np.float32).reshape(-1, 2)
        pp = _p(pred)
    mp, mpitch = None, 0
    if mask is not None:
        mask = np.ascontiguousarray(mask, np.uint8)
        mp, mpitch = _p(mask), mask.shape[1]
    b = np.ascontiguousarray(border, np.int32)
    alive = lib().or_finish_tracks(_p(t), _p(a), len(t), pp, int(width), int(height), _p(b), mp, mpitch,
                                   int(bool(collapse)))
    return t, a, alive


ST_CACHE_DTYPE = np.dtype([("patch", np.float32, (810,)), ("patch_sums", np.float32, (10,)),
                           ("level_mask", np.uint32)])


def _sizes(pyr):
    levels = len(pyr)
    ws = np.array([p[0].shape[1] for p in pyr] + [0] * (10 - levels), np.int32)
    hs = np.array([p[0].shape[0] for p in pyr] + [0] * (10 - levels), np.int32)
    return levels, ws, hs


def st_track(prev_pyr, cur_pyr, tracks, n_shift=0, n_full=20, mode=TEXTURE):
    """The affine tracker (or_st_track): previous patches from prev_pyr's images, current image and
    gradients from cur_pyr.  Returns updated copies of the TRACK_DTYPE records."""
    t = np.ascontiguousarray(tracks.copy())
    levels, ws, hs = _sizes(prev_pyr)
    k1, pim = _level_ptrs([p[0] for p in prev_pyr])
    k2, cim = _level_ptrs([p[0] for p in cur_pyr[:levels]])
    k3, cgx = _level_ptrs([p[1] for p in cur_pyr[:levels]])
    k4, cgy = _level_ptrs([p[2] for p in cur_pyr[:levels]])
    lib().or_st_track(levels, _p(ws), _p(hs), pim, cim, cgx, cgy, _p(t), len(t), n_shift, n_full, mode)
    del k1, k2, k3, k4
    return t


def st_build_cache(prev_pyr, tracks, mode=TEXTURE):
    """(tracks with cache_index set, cache entries) as st_build_cache_kernel makes them."""
    t = np.ascontiguousarray(tracks.copy())
    levels, ws, hs = _sizes(prev_pyr)
    k1, pim = _level_ptrs([p[0] for p in prev_pyr])
    cache = np.zeros(max(len(t), 1), ST_CACHE_DTYPE)
    lib().or_st_build_cache(levels, _p(ws), _p(hs), pim, _p(t), len(t), _p(cache), mode)
    del k1
    return t, cache[:len(t)]


def st_track_cached(cur_pyr, cache, tracks, n_shift=0, n_full=20, mode=TEXTURE):
    t = np.ascontiguousarray(tracks.copy())
    levels, ws, hs = _sizes(cur_pyr)
    k2, cim = _level_ptrs([p[0] for p in cur_pyr])
    k3, cgx = _level_ptrs([p[1] for p in cur_pyr])
    k4, cgy = _level_ptrs([p[2] for p in cur_pyr])
    cache = np.ascontiguousarray(cache, ST_CACHE_DTYPE)
    lib().or_st_track_cached(levels, _p(ws), _p(hs), cim, cgx, cgy, _p(cache), _p(t), len(t), n_shift, n_full, mode)
    del k2, k3, k4
    return t


def st_qr_solve(a, b):
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    x = np.zeros(len(b), np.float32)
    ok = lib().or_st_qr_solve(len(b), _p(a), _p(b), _p(x))
    return bool(ok), x


def stereo_scan(prim_pyr, sec_pyr, uv, cand_off, cand_xy, valid=None, search_radius=48.0, ncc_threshold=0.8,
                early_exit_fraction=0.8, mode=TEXTURE, horizontal=True):
    """The reference's left-to-right candidate scan (or_stereo_scan) on host pyramids [(img, gx, gy)]
    per level.  Returns (TRACK_DTYPE records, winner int32, stats int32[4])."""
    from cuvslam_b200.types import TRACK_DTYPE
    L = lib()
    uv = np.ascontiguousarray(uv, np.float32).reshape(-1, 2)
    n = len(uv)
    levels = len(prim_pyr)
    ws = np.array([p[0].shape[1] for p in prim_pyr] + [0] * (10 - levels), np.int32)
    hs = np.array([p[0].shape[0] for p in prim_pyr] + [0] * (10 - levels), np.int32)
    keep1, pgx = _level_ptrs([p[1] for p in prim_pyr])
    keep4, pgy = _level_ptrs([p[2] for p in prim_pyr])
    keep2, pim = _level_ptrs([p[0] for p in prim_pyr])
    keep3, sim = _level_ptrs([p[0] for p in sec_pyr[:levels]])
    cand_off = np.ascontiguousarray(cand_off, np.int32)
    cand_xy = np.ascontiguousarray(cand_xy, np.float32).reshape(-1, 2)
    if len(cand_xy) == 0:
        cand_xy = np.zeros((1, 2), np.float32)
    vp = None
    if valid is not None:
        valid = np.ascontiguousarray(valid, np.uint8)
        vp = _p(valid)
    out = np.zeros(max(n, 1), TRACK_DTYPE)
    win = np.zeros(max(n, 1), np.int32)
    stats = np.zeros(4, np.int32)
    L.or_stereo_scan(levels, _p(ws), _p(hs), pgx, pgy, pim, sim, _p(uv), vp, n, _p(cand_off), _p(cand_xy),
                     float(search_radius), float(ncc_threshold), float(early_exit_fraction), int(bool(horizontal)),
                     mode, _p(out), _p(win), _p(stats))
    del keep1, keep2, keep3, keep4
    return out[:n], win[:n], stats


class CpuCamera:
    """One camera of the restated reference CPU tracker (cpu_tracker.c)."""

    def __init__(self, width, height):
        self.w, self.h = int(width), int(height)
        self.h_ = lib().cpu_cam_create(self.w, self.h)

    def build(self, img_u8, box3=False):
        """ImagePyramidU8::build (image_pyramid_u8.cpp:24-57), box prefiltered when box3."""
        img = np.ascontiguousarray(img_u8, np.uint8)
        assert img.shape == (self.h, self.w)
        lib().cpu_cam_build_ex(self.h_, _p(img), int(bool(box3)))
        return self

    def patch(self, level, x, y):
        """computePatch's 9x9 exact-bilinear patch at (x, y) on a level's image, or None outside."""
        out = np.zeros((9, 9), np.float32)
        ok = lib().cpu_cam_patch(self.h_, int(level), ctypes.c_float(x), ctypes.c_float(y), _p(out))
        return out if ok else None

    def levels(self):
        return lib().cpu_cam_levels(self.h_)

    def level(self, l):
        w, h = ctypes.c_int(), ctypes.c_int()
        lib().cpu_cam_level(self.h_, l, ctypes.byref(w), ctypes.byref(h), None, None, None)
        out = [np.zeros((h.value, w.value), np.float32) for _ in range(3)]
        lib().cpu_cam_level(self.h_, l, ctypes.byref(w), ctypes.byref(h), _p(out[0]), _p(out[1]), _p(out[2]))
        return out

    def track_from(self, prev, xy, pred=None):
        xy = np.ascontiguousarray(xy, np.float32).reshape(-1, 2)
        out = np.zeros_like(xy)
        st = np.zeros(len(xy), np.uint8)
        pr = None if pred is None else np.ascontiguousarray(pred, np.float32).reshape(-1, 2)
        lib().cpu_cam_track(prev.h_, self.h_, _p(xy), None if pr is None else _p(pr), len(xy), _p(out), _p(st))
        return out, st

    def select(self, alive=None, num_desired=450, borders=(0, 0, 0, 0)):
        alive = np.zeros((0, 2), np.float32) if alive is None else np.ascontiguousarray(alive, np.float32).reshape(-1, 2)
        out = np.zeros((max(num_desired, 1), 2), np.float32)
        n = lib().cpu_cam_select(self.h_, _p(alive), len(alive), num_desired, *borders, _p(out))
        return out[:n]

    def __del__(self):
        try:
            lib().cpu_cam_destroy(self.h_)
        except Exception:
            pass


def cpu_frame_step(prev_cams, cur_cams, images, xy, pred, num_desired, nthreads, features_parallel=False):
    """One multi-camera frame step of the restated CPU tracker on `nthreads` threads: one camera per
    thread, or (features_parallel) the cameras in turn with each camera's tracking spread over the
    threads.  Returns (tracked positions, status, new features) per camera."""
    n = len(cur_cams)
    PA = ctypes.c_void_p * n
    imgs = [np.ascontiguousarray(i, np.uint8) for i in images]
    xys = [np.ascontiguousarray(a, np.float32).reshape(-1, 2) for a in xy]
    preds = None if pred is None else [np.ascontiguousarray(a, np.float32).reshape(-1, 2) for a in pred]
    outs = [np.zeros_like(a) for a in xys]
    sts = [np.zeros(len(a), np.uint8) for a in xys]
    news = [np.zeros((max(int(k), 1), 2), np.float32) for k in num_desired]
    counts = np.zeros(n, np.int32)
    ns = np.array([len(a) for a in xys], np.int32)
    nd = np.array(num_desired, np.int32)
    step = lib().cpu_frame_step_features if features_parallel else lib().cpu_frame_step
    step(PA(*[c.h_ for c in prev_cams]) if prev_cams is not None else None, PA(*[c.h_ for c in cur_cams]),
         PA(*[i.ctypes.data for i in imgs]), PA(*[a.ctypes.data for a in xys]),
         None if preds is None else PA(*[a.ctypes.data for a in preds]), _p(ns), _p(nd),
         PA(*[a.ctypes.data for a in outs]), PA(*[a.ctypes.data for a in sts]),
         PA(*[a.ctypes.data for a in news]), _p(counts), n, nthreads)
    return outs, sts, [a[:c] for a, c in zip(news, counts)]


# ---------------------------------------------------------------- FP64 differentiable LK (lk_adjoint64.c)
IMPLICIT = 0
UNROLLED = 1

_L64_SIGS = [
    ("or64_cam_create", [I, I, I], P),
    ("or64_cam_destroy", [P], None),
    ("or64_cam_levels", [P], I),
    ("or64_cam_set", [P, P, P], None),
    ("or64_cam_plane", [P, I, I, P], None),
    ("or64_track", [P, P, I, I, I, ctypes.c_double, P, P], None),
    ("or64_backward", [P, P, I, I, I, ctypes.c_double, P, P, P, P, P], None),
    ("or64_fd", [P, P, P, P, I, I, I, ctypes.c_double, P, P, I, P, P, ctypes.c_double, P, I], None),
]


def _l64():
    L = lib()
    if not getattr(L, "_l64_ready", False):
        for name, args, res in _L64_SIGS:
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        L._l64_ready = True
    return L


class Diff64:
    """FP64 differentiable LK on one camera: pyramids of a previous and a current level-0 image
    (float64), the forward tracker in both adjoint modes, its vector-Jacobian product, and
    central finite differences of the mean squared distance to ground truth."""

    def __init__(self, prev0, cur0, max_levels=10):
        self.prev = np.ascontiguousarray(prev0, np.float64)
        self.cur = np.ascontiguousarray(cur0, np.float64)
        self.h, self.w = self.prev.shape
        L = _l64()
        self.h_ = L.or64_cam_create(self.w, self.h, max_levels)
        L.or64_cam_set(self.h_, _p(self.prev), _p(self.cur))
        self.levels = L.or64_cam_levels(self.h_)

    def plane(self, level, plane):
        lw, lh = level_sizes(self.w, self.h)[level]
        out = np.zeros((lh, lw), np.float64)
        _l64().or64_cam_plane(self.h_, level, plane, _p(out))
        return out

    def track(self, tracks, mode, iters, tol=1e-13):
        tracks = np.ascontiguousarray(tracks)
        n = len(tracks)
        xy = np.zeros((n, 2), np.float64)
        st = np.zeros(n, np.uint8)
        _l64().or64_track(self.h_, _p(tracks), n, mode, iters, tol, _p(xy), _p(st))
        return xy, st

    def backward(self, tracks, mode, iters, grad_xy, tol=1e-13):
        tracks = np.ascontiguousarray(tracks)
        n = len(tracks)
        g = np.ascontiguousarray(grad_xy, np.float64).reshape(n, 2)
        gp = np.zeros((self.h, self.w), np.float64)
        gc = np.zeros((self.h, self.w), np.float64)
        gt = np.zeros((n, 2), np.float64)
        go = np.zeros((n, 2), np.float64)
        _l64().or64_backward(self.h_, _p(tracks), n, mode, iters, tol, _p(g), _p(gp), _p(gc), _p(gt), _p(go))
        return gp, gc, gt, go

    def fd(self, tracks, mode, iters, gt_xy, mask, which, index, h=1e-3, tol=1e-13, strict=False):
        """Central differences; NaN where a perturbation changed a counted track's success or, with
        strict, any of its discrete decisions (levels set up and accepted, steps per level)."""
        tracks = np.ascontiguousarray(tracks)
        n = len(tracks)
        gt = np.ascontiguousarray(gt_xy, np.float64).reshape(n, 2)
        m = np.ascontiguousarray(mask, np.uint8)
        wh = np.ascontiguousarray(which, np.int32)
        ix = np.ascontiguousarray(index, np.int64)
        out = np.zeros(len(wh), np.float64)
        _l64().or64_fd(self.h_, _p(self.prev), _p(self.cur), _p(tracks), n, mode, iters, tol, _p(gt), _p(m), len(wh),
                       _p(wh), _p(ix), h, _p(out), int(bool(strict)))
        return out

    def __del__(self):
        try:
            _l64().or64_cam_destroy(self.h_)
        except Exception:
            pass
