"""ctypes front for oracle/_ref/libcuvslam_ref.so: the reference's own CUDA kernels (compiled from the
cuVSLAM sources by oracle/build_ref.sh) driven by oracle/ref_harness.cu's restatement of the
reference wrappers' launch sequences.  TEST INFRASTRUCTURE ONLY: the golden-fixture script, the
GPU parity tests and bench.py's parity checker (outside its timed regions) use it to compare this
library's results with the reference's; the product never loads it.

Every call takes and returns host arrays and synchronises (a checker, not fast).
"""

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libcuvslam_ref.so")
_LIB = None

P, I, F = ctypes.c_void_p, ctypes.c_int, ctypes.c_float


def available():
    return os.path.exists(LIB_PATH)


def lib():
    """Loads the harness (raises if oracle/_ref was not built: it needs the reference sources)."""
    global _LIB
    if _LIB is None:
        L = ctypes.CDLL(LIB_PATH)
        L.ref_pyramid.argtypes = [P, I, I, I, P, P, P, P]
        L.ref_pyramid_ex.argtypes = [P, I, I, I, I, I, P, P, P, P]
        L.ref_select.argtypes = [P, I, I, P, I, I, I, I, I, I, P, P, P, P, P, P, P, P, P]
        L.ref_lk.argtypes = [P, P, I, I, I, P, I, I]
        L.ref_tex_probe.argtypes = [P, I, I, P, I, P]
        L.ref_stereo_scan.argtypes = [P, P, I, I, I, P, P, I, P, P, F, F, F, I, P, P, P]
        L.ref_st_track.argtypes = [P, P, I, I, I, P, I, I, I, I, P]
        _LIB = L
    return _LIB


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def level_sizes(w, h, max_levels=10):
    """GPUImagePyramid::prepare_levels (image_pyramid.h:136-151): (d+1)/2 while both sides >= 15."""
    out = []
    while len(out) < max_levels:
        out.append((w, h))
        w, h = (w + 1) // 2, (h + 1) // 2
        if w < 15 or h < 15:
            break
    return out


def pyramid(img, max_levels=10):
    """ImageCast::cast + GaussianGPUImagePyramid::build + GPUGradientPyramid::set on a uint8 frame:
    [(level, grad_x, grad_y)] per level."""
    h, w = img.shape
    sizes = level_sizes(w, h, max_levels)
    total = sum(a * b for a, b in sizes)
    lv, gx, gy = (np.zeros(total, np.float32) for _ in range(3))
    n = ctypes.c_int(0)
    img = np.ascontiguousarray(img)
    rc = lib().ref_pyramid(_ptr(img), w, h, max_levels, ctypes.byref(n), _ptr(lv), _ptr(gx), _ptr(gy))
    assert rc == 0 and n.value == len(sizes), (rc, n.value)
    out, off = [], 0
    for (a, b) in sizes:
        out.append((lv[off:off + a * b].reshape(b, a), gx[off:off + a * b].reshape(b, a),
                    gy[off:off + a * b].reshape(b, a)))
        off += a * b
    return out


def select(img, alive, num_desired, borders=(0, 0, 0, 0)):
    """GPUSelection::computeGFTTAndSelectFeatures (selection_v2.cpp:27-184) on a uint8 frame's level 0,
    with its host quota loop: dict of the response and NMS maps, cell maxima, sorted keypoints, bin
    sums and the selected features (sel, n x 2)."""
    h, w = img.shape
    cw, ch = w // 8, h // 8
    cap = max(cw * ch, 1)
    gftt = np.zeros((h, w), np.float32)
    nms = np.zeros((h, w), np.float32)
    cmax = np.zeros(cap, np.float32)
    cidx = np.zeros(cap * 2, np.uint32)
    kp = np.zeros(cap * 3, np.float32)
    bins = np.zeros(64, np.float32)
    sel = np.zeros(max(num_desired, 1) * 2, np.float32)
    nkp, nsel = ctypes.c_int(0), ctypes.c_int(0)
    alive = np.ascontiguousarray(alive, np.float32).reshape(-1, 2)
    img = np.ascontiguousarray(img)
    rc = lib().ref_select(_ptr(img), w, h, _ptr(alive), len(alive), num_desired, *borders, _ptr(gftt), _ptr(nms),
                          _ptr(cmax), _ptr(cidx), _ptr(kp), ctypes.byref(nkp), _ptr(bins), _ptr(sel),
                          ctypes.byref(nsel))
    assert rc == 0, rc
    return dict(gftt=gftt, nms=nms, cell_max=cmax[:cw * ch].reshape(ch, cw),
                cell_idx=cidx[:2 * cw * ch].reshape(ch, cw, 2), kp=kp[:3 * nkp.value].reshape(-1, 3), bins=bins,
                sel=sel[:2 * nsel.value].reshape(-1, 2))


def lk(prev, nxt, tracks, max_levels=10, horizontal=False):
    """GPULKFeatureTracker::track_points (cuda_modules/lk_tracker.cpp:24-73) -> lk_track_kernel on the
    two frames' pyramids: a copy of the TrackData records, tracked."""
    h, w = prev.shape
    t = np.ascontiguousarray(tracks.copy())
    rc = lib().ref_lk(_ptr(np.ascontiguousarray(prev)), _ptr(np.ascontiguousarray(nxt)), w, h, max_levels, _ptr(t),
                      len(t), int(horizontal))
    assert rc == 0, rc
    return t


def tex_probe(img, xy):
    """Linear-filtered texture fetches of an FP32 image at xy (the texture unit's own arithmetic)."""
    h, w = img.shape
    out = np.zeros(len(xy), np.float32)
    rc = lib().ref_tex_probe(_ptr(np.ascontiguousarray(img, np.float32)), w, h,
                             _ptr(np.ascontiguousarray(xy, np.float32)), len(xy), _ptr(out))
    assert rc == 0, rc
    return out


def lk_deviation(got, want):
    """Per-track agreement of two TrackData arrays from the same inputs: status agreement over all
    tracks, and the distance between positions of the tracks both keep (median, p99, max)."""
    sg, sw = got["track_status"] != 0, want["track_status"] != 0
    both = sg & sw
    d = np.linalg.norm(got["track"][both].astype(np.float64) - want["track"][both].astype(np.float64), axis=1)
    return {"n": int(len(got)), "kept_both": int(both.sum()), "status_agree": float((sg == sw).mean()) if len(got) else 1.0,
            "median_px": float(np.median(d)) if len(d) else 0.0,
            "p99_px": float(np.percentile(d, 99)) if len(d) else 0.0, "max_px": float(d.max()) if len(d) else 0.0}


def same_features(a, b, tol=1e-4):
    """Selected feature sets equal as sets (the reference orders exact strength ties arbitrarily)."""
    a, b = np.asarray(a, np.float64).reshape(-1, 2), np.asarray(b, np.float64).reshape(-1, 2)
    if a.shape != b.shape:
        return False
    ka, kb = a[np.lexsort((a[:, 0], a[:, 1]))], b[np.lexsort((b[:, 0], b[:, 1]))]
    return bool(len(a) == 0 or np.abs(ka - kb).max() <= tol)
