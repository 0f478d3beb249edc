"""Generates the golden fixtures under tests/golden/.

Step 1 (any machine, no GPU):   python tests/golden/make_golden.py inputs
    Draws the seeded synthetic input frames and writes tests/golden/inputs.npz.
    (`stereo-inputs` likewise writes tests/golden/stereo_inputs.npz: a rectified right image of the
    c1 scene, primary points and their candidate lists for the left-to-right scan.)
Step 2 (a B200, after oracle/build_ref.sh built oracle/_ref/libcuvslam_ref.so):
    python tests/golden/make_golden.py reference --out DIR
    Runs the reference's own CUDA kernels (compiled unchanged from cuVSLAM by oracle/build_ref.sh)
    on those inputs and writes DIR/reference.npz (compact: hashes of every pyramid/gradient level,
    the sorted keypoints, the selected features, the LK results and a texture-sampling probe) and
    DIR/reference_full.npz (every intermediate array, for debugging; not committed).
The committed tests/golden/reference.npz is the step-2 output.
`input-reference --out DIR` runs the reference's cast_image_rgb and box prefilter ahead of its pyramid
(oracle/ref_harness.cu ref_pyramid_ex) and writes DIR/input_reference.npz.
`stereo-reference --out DIR` runs the reference's multi-launch left-to-right scan
(lk_track_horizontal per candidate round, oracle/ref_harness.cu) on stereo_inputs.npz and writes
DIR/stereo_reference.npz.
`st-reference --out DIR` runs the reference's affine tracker (st_track, st_build_cache +
st_track_with_cache; oracle/ref_harness.cu ref_st_track) and writes DIR/st_reference.npz.
`headline-reference --out DIR` runs the reference's selection and LK at the batched workload's
camera sizes (1280x720 and 1920x1200, 3000 features each; frames drawn from their seeds, hashed so
a test can check it regenerated the same ones) and writes DIR/headline_reference.npz.
"""

import argparse
import ctypes
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from cuvslam_b200 import synthetic  # noqa: E402
from cuvslam_b200.types import TRACK_DTYPE, level_sizes, make_tracks  # noqa: E402
from oracle import ref as REF  # noqa: E402

# name -> (width, height, camera id)
CASES = {
    "c1": (752, 480, 0),  # the 752x480 stereo-pair configuration
    "half": (376, 240, 1),
    "odd": (97, 61, 2),
    "tiny": (31, 17, 3),
}


def make_inputs(path):
    arrays = {}
    for name, (w, h, cam) in CASES.items():
        prev, nxt, warp = synthetic.frame_pair(cam, w, h)
        arrays[f"{name}/prev"] = prev
        arrays[f"{name}/next"] = nxt
        arrays[f"{name}/warp"] = np.array([warp.theta, warp.scale, warp.tx, warp.ty, warp.cx, warp.cy])
    np.savez_compressed(path, **arrays)


def _lib():
    return REF.lib()


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def ref_pyramid(lib, img, max_levels=10):
    return REF.pyramid(img, max_levels)


def ref_select(lib, img, alive, num_desired, borders=(0, 0, 0, 0)):
    return REF.select(img, alive, num_desired, borders)


def ref_lk(lib, prev, nxt, tracks, max_levels=10, horizontal=False):
    return REF.lk(prev, nxt, tracks, max_levels, horizontal)


def ref_tex_probe(lib, img, xy):
    return REF.tex_probe(img, xy)


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def tex_probe_inputs():
    rng = np.random.default_rng(99)
    img = rng.uniform(-300.0, 300.0, (40, 48)).astype(np.float32)
    # 1) fractional sweep across one texel step of a 0/1 image reveals the weight quantisation
    step = np.zeros((40, 48), np.float32)
    step[:, 25:] = 1.0
    fr = (np.arange(8192, dtype=np.float64) / 8192.0)
    sweep = np.stack([24.5 + fr, np.full_like(fr, 10.5)], 1).astype(np.float32)
    # 2) random sub-texel coordinates on a random image, including clamped edges
    xy = np.stack([rng.uniform(-1.0, 49.0, 20000), rng.uniform(-1.0, 41.0, 20000)], 1).astype(np.float32)
    return img, step, sweep, xy


def make_reference(out_dir):
    lib = _lib()
    inp = np.load(os.path.join(HERE, "inputs.npz"))
    compact, full = {}, {}
    for name in CASES:
        prev, nxt = inp[f"{name}/prev"], inp[f"{name}/next"]
        for tag, img in (("prev", prev), ("next", nxt)):
            for l, (lv, gx, gy) in enumerate(ref_pyramid(lib, img)):
                for q, arr in (("img", lv), ("gx", gx), ("gy", gy)):
                    compact[f"{name}/{tag}/L{l}/{q}/sha"] = np.array(_sha(arr))
                    full[f"{name}/{tag}/L{l}/{q}"] = arr
        # 4-level pyramids (the stereo-pair workload caps levels at 4)
        for l, (lv, gx, gy) in enumerate(ref_pyramid(lib, prev, 4)):
            compact[f"{name}/prev4/L{l}/img/sha"] = np.array(_sha(lv))
        h, w = prev.shape
        s1 = ref_select(lib, prev, np.zeros((0, 2), np.float32), 450)
        alive = s1["sel"][::2].copy()
        s2 = ref_select(lib, prev, alive, 450 - len(alive), borders=(3, 4, 5, 6))
        for tag, s in (("sel0", s1), ("sel1", s2)):
            compact[f"{name}/{tag}/kp"] = s["kp"]
            compact[f"{name}/{tag}/sel"] = s["sel"]
            compact[f"{name}/{tag}/bins"] = s["bins"]
            compact[f"{name}/{tag}/gftt/sha"] = np.array(_sha(s["gftt"]))
            compact[f"{name}/{tag}/nms/sha"] = np.array(_sha(s["nms"]))
            for k, v in s.items():
                full[f"{name}/{tag}/{k}"] = v
        compact[f"{name}/sel1/alive"] = alive
        pts = s1["sel"]
        if len(pts) == 0:
            continue
        wp = inp[f"{name}/warp"]
        warp = synthetic.Similarity(*[float(v) for v in wp])
        gt = synthetic.flow_texture(warp, pts.astype(np.float64)).astype(np.float32)
        rng = np.random.default_rng(5)
        pred = gt + rng.normal(0.0, 0.7, gt.shape).astype(np.float32)
        runs = {
            "lk_zero": make_tracks(pts, None, float(w), 0.8),
            "lk_pred": make_tracks(pts, pred - pts, float(w), 0.8),
            "lk_retrack": make_tracks(pts, None, float(w), 0.85),
        }
        for tag, t in runs.items():
            out = ref_lk(lib, prev, nxt, t)
            compact[f"{name}/{tag}/in"] = t
            compact[f"{name}/{tag}/out"] = out
        out4 = ref_lk(lib, prev, nxt, runs["lk_pred"], max_levels=4)
        compact[f"{name}/lk_pred4/out"] = out4
        outh = ref_lk(lib, prev, nxt, runs["lk_zero"], horizontal=True)
        compact[f"{name}/lk_horiz/out"] = outh
        compact[f"{name}/gt"] = gt
    img, step, sweep, xy = tex_probe_inputs()
    compact["tex/sweep"] = ref_tex_probe(lib, step, sweep)
    compact["tex/random"] = ref_tex_probe(lib, img, xy)
    os.makedirs(out_dir, exist_ok=True)
    np.savez_compressed(os.path.join(out_dir, "reference.npz"), **compact)
    np.savez_compressed(os.path.join(out_dir, "reference_full.npz"), **full)
    print("wrote", out_dir)


# Left-to-right scan fixtures: the c1 scene (left: inputs.npz c1/prev) and its rectified right view (disparity 5-40 px), 4-level
# pyramids (top level 3), primary points, and two candidate sets: the epipolar table of a pinhole
# pair (fx 458, baseline 0.11 m) and random lists of 0-12 candidates left of each point.
STEREO_LEVELS = 4
STEREO_RUNS = {  # name -> (candidate set, early-exit fraction, horizontal tracker)
    "curves": ("curves", 0.8, True),
    "random": ("random", 0.8, True),
    "random_full": ("random", 1.0, True),
    "random_low": ("random", 0.3, True),
    "curves_2d": ("curves", 0.8, False),
    "random_2d": ("random", 0.3, False),
}


def make_stereo_inputs(path):
    from cuvslam_b200 import stereo
    from oracle import oracle

    w, h, cam = CASES["c1"]
    left = np.load(os.path.join(HERE, "inputs.npz"))["c1/prev"]
    right = synthetic.stereo_right(cam, w, h)
    rng = np.random.default_rng(61)
    n = 700
    uv = np.stack([rng.uniform(6.0, w - 6.0, n), rng.uniform(6.0, h - 6.0, n)], 1).astype(np.float32)
    uv[:6] = [[0.5, 0.5], [w - 0.5, h - 0.5], [w - 1.0, 10.0], [3.0, h / 2], [w / 2, 0.0], [w / 2, h - 1.0]]
    valid = (rng.uniform(size=n) > 0.03).astype(np.uint8)
    sizes = level_sizes(w, h, STEREO_LEVELS)
    top = len(sizes) - 1
    k = (458.0, 458.0, 367.0, 248.0)
    curves = stereo.pinhole_curves(k, k, (np.eye(3), (-0.11, 0.0, 0.0)), top, sizes[top][0], sizes[top][1])
    cw, ch, c_off, c_xy = stereo.curves_csr(curves)
    inv_scale = 1.0 / float(1 << top)
    off_c, xy_c = oracle.epipolar_candidates(cw, ch, inv_scale, c_off, c_xy, uv, valid)
    counts = rng.integers(0, 13, n)
    off_r = np.zeros(n + 1, np.int32)
    np.cumsum(counts, out=off_r[1:])
    xs = np.repeat(uv[:, 0], counts) - rng.uniform(0.0, 80.0, off_r[-1])
    ys = np.repeat(uv[:, 1], counts) + rng.normal(0.0, 0.5, off_r[-1])
    xy_r = np.stack([xs, ys], 1).astype(np.float32)
    np.savez_compressed(path, right=right, uv=uv, valid=valid, top=np.int32(top),
                        curves_wh=np.array([cw, ch], np.int32), curves_inv_scale=np.float32(inv_scale),
                        curves_offsets=c_off, curves_xy=c_xy, curves_cand_off=off_c, curves_cand_xy=xy_c,
                        random_cand_off=off_r, random_cand_xy=xy_r)


def make_stereo_reference(out_dir):
    lib = _lib()
    P, I, F = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
    lib.ref_stereo_scan.argtypes = [P, P, I, I, I, P, P, I, P, P, F, F, F, I, P, P, P]
    inp = np.load(os.path.join(HERE, "stereo_inputs.npz"))
    left = np.ascontiguousarray(np.load(os.path.join(HERE, "inputs.npz"))["c1/prev"])
    right = np.ascontiguousarray(inp["right"])
    h, w = left.shape
    uv = np.ascontiguousarray(inp["uv"], np.float32)
    valid = np.ascontiguousarray(inp["valid"], np.uint8)
    n = len(uv)
    radius = 3.0 * float(1 << (int(inp["top"]) + 1))
    compact = {}
    for run, (cset, frac, horizontal) in STEREO_RUNS.items():
        off = np.ascontiguousarray(inp[f"{cset}_cand_off"], np.int32)
        xy = np.ascontiguousarray(inp[f"{cset}_cand_xy"], np.float32)
        out = np.zeros(n, TRACK_DTYPE)
        win = np.zeros(n, np.int32)
        stats = np.zeros(2, np.int32)
        rc = lib.ref_stereo_scan(_ptr(left), _ptr(right), w, h, STEREO_LEVELS, _ptr(uv), _ptr(valid), n, _ptr(off),
                                 _ptr(xy), radius, 0.8, frac, int(horizontal), _ptr(out), _ptr(win), _ptr(stats))
        assert rc == 0, rc
        compact[f"{run}/out"] = out
        compact[f"{run}/winner"] = win
        compact[f"{run}/stats"] = stats
        print(run, "matched", stats[0], "rounds", stats[1])
    os.makedirs(out_dir, exist_ok=True)
    np.savez_compressed(os.path.join(out_dir, "stereo_reference.npz"), **compact)


# Input-stage fixtures: the pyramid from an RGB8 frame (cast_image_rgb) and with the box prefilter,
# by the reference's kernels (oracle/ref_harness.cu ref_pyramid_ex), on frames built from inputs.npz.
INPUT_CASES = ("c1", "odd", "tiny")
INPUT_MODES = {"mono_box3": (0, 1), "rgb": (1, 0), "rgb_box3": (1, 1)}


def input_frame(inp, name, rgb):
    prev = inp[f"{name}/prev"]
    if not rgb:
        return np.ascontiguousarray(prev)
    return np.ascontiguousarray(np.stack([prev, inp[f"{name}/next"], np.roll(prev, 7, axis=1)], -1))


def make_input_reference(out_dir):
    lib = _lib()
    P, I = ctypes.c_void_p, ctypes.c_int
    lib.ref_pyramid_ex.argtypes = [P, I, I, I, I, I, P, P, P, P]
    inp = np.load(os.path.join(HERE, "inputs.npz"))
    compact = {}
    for name in INPUT_CASES:
        for mode, (rgb, box) in INPUT_MODES.items():
            img = input_frame(inp, name, rgb)
            h, w = img.shape[:2]
            sizes = level_sizes(w, h, 10)
            total = sum(a * b for a, b in sizes)
            lv, gx, gy = (np.zeros(total, np.float32) for _ in range(3))
            n = ctypes.c_int(0)
            rc = lib.ref_pyramid_ex(_ptr(img), w, h, rgb, box, 10, ctypes.byref(n), _ptr(lv), _ptr(gx), _ptr(gy))
            assert rc == 0 and n.value == len(sizes), (rc, n.value)
            off = 0
            for l, (a, b) in enumerate(sizes):
                for q, arr in (("img", lv), ("gx", gx), ("gy", gy)):
                    compact[f"{name}/{mode}/L{l}/{q}/sha"] = np.array(_sha(arr[off:off + a * b].reshape(b, a)))
                if l == 0 and name != "c1":
                    compact[f"{name}/{mode}/level0"] = lv[:a * b].reshape(b, a).copy()
                off += a * b
    os.makedirs(out_dir, exist_ok=True)
    np.savez_compressed(os.path.join(out_dir, "input_reference.npz"), **compact)
    print("wrote input_reference.npz")


# Affine (Shi-Tomasi) tracker fixtures: the reference's st_track / st_build_cache +
# st_track_with_cache (oracle/ref_harness.cu ref_st_track) on the inputs.npz pairs, from the
# selected points of reference.npz, and on one strongly rotated and scaled pair drawn here
# (st_frames, "rot").
ST_CASES = ("c1", "half", "odd")
ST_ROT_WARP = (0.12, 1.08, 3.0, -2.0)  # theta, scale, tx, ty about the frame centre
ST_CACHE_KEEP = 8  # cache entries stored whole per case


def st_frames(name, inp=None):
    """(prev, next, Similarity) of an affine-tracker case."""
    if name == "rot":
        w, h = 376, 240
        scene = synthetic.Scene.draw(1101, w, h)
        warp = synthetic.Similarity(*ST_ROT_WARP, cx=(w - 1) / 2.0, cy=(h - 1) / 2.0)
        prev = synthetic.quantise(scene.render())
        nxt = synthetic.quantise(scene.render(warp), np.random.default_rng(3101), 2.0)
        return prev, nxt, warp
    wp = inp[f"{name}/warp"]
    return inp[f"{name}/prev"], inp[f"{name}/next"], synthetic.Similarity(*[float(v) for v in wp])


def st_points(name, ref, prev):
    if name == "rot":
        h, w = prev.shape
        rng = np.random.default_rng(44)
        return np.stack([rng.uniform(12, w - 12, 300), rng.uniform(12, h - 12, 300)], 1).astype(np.float32)
    return ref[f"{name}/sel0/sel"].astype(np.float32)


def st_runs(name, prev, warp, pts):
    """name -> (records, n_shift, n_full, cached)."""
    h, w = prev.shape
    gt = synthetic.flow_texture(warp, pts.astype(np.float64)).astype(np.float32)
    rng = np.random.default_rng(6)
    pred = gt + rng.normal(0.0, 0.7, gt.shape).astype(np.float32)
    lin = warp._mat().astype(np.float32).reshape(-1)
    mapped = make_tracks(pts, pred - pts, float(w), 0.8)
    mapped["initial_guess_map"] = lin
    runs = {
        "st_pred": (make_tracks(pts, pred - pts, float(w), 0.8), 0, 20, 0),
        "st_map": (mapped, 0, 20, 0),
        "st_cached": (make_tracks(pts, pred - pts, float(w), 0.8), 0, 20, 1),
    }
    if name != "rot":
        runs["st_zero"] = (make_tracks(pts, None, float(w), 0.8), 0, 20, 0)
        runs["st_mixed"] = (make_tracks(pts, pred - pts, 7.0, 0.8), 10, 10, 0)
    return runs, gt


def make_st_reference(out_dir):
    lib = _lib()
    P, I = ctypes.c_void_p, ctypes.c_int
    lib.ref_st_track.argtypes = [P, P, I, I, I, P, I, I, I, I, P]
    inp = np.load(os.path.join(HERE, "inputs.npz"))
    ref = np.load(os.path.join(HERE, "reference.npz"))
    compact = {}
    for name in ST_CASES + ("rot",):
        prev, nxt, warp = st_frames(name, inp)
        h, w = prev.shape
        pts = st_points(name, ref, prev)
        runs, gt = st_runs(name, prev, warp, pts)
        compact[f"{name}/gt"] = gt
        for tag, (t, ns, nf, cached) in runs.items():
            out = np.ascontiguousarray(t.copy())
            cache = np.zeros((max(len(t), 1), 3284), np.uint8)
            rc = lib.ref_st_track(_ptr(np.ascontiguousarray(prev)), _ptr(np.ascontiguousarray(nxt)), w, h, 10,
                                  _ptr(out), len(out), ns, nf, cached, _ptr(cache))
            assert rc == 0, rc
            compact[f"{name}/{tag}/in"] = t
            compact[f"{name}/{tag}/out"] = out
            if cached:
                c = cache[:len(t)]
                compact[f"{name}/{tag}/cache_head"] = c[:ST_CACHE_KEEP].copy()
                compact[f"{name}/{tag}/patch_sums"] = c[:, 3240:3280].copy().view(np.float32)
                compact[f"{name}/{tag}/level_mask"] = c[:, 3280:3284].copy().view(np.uint32).reshape(-1)
        if name == "rot":
            compact["rot/prev"] = prev
            compact["rot/next"] = nxt
        print(name, {k: int((v[0]["track_status"] != 0).sum()) for k, v in runs.items()})
    os.makedirs(out_dir, exist_ok=True)
    np.savez_compressed(os.path.join(out_dir, "st_reference.npz"), **compact)
    print("wrote st_reference.npz")


# Headline-size fixtures: one camera of each large size of the batched 32-camera workload (its camera
# index gives the scene seed), 3000 Shi-Tomasi features selected by the reference on the previous
# frame, LK with zero and with predicted offsets, and the selection on the next frame with the zero-
# offset run's survivors alive (the batched step's selection).
HEADLINE_CASES = {"hd": (1280, 720, 12), "fhd": (1920, 1200, 24)}  # name -> (width, height, camera)
HEADLINE_FEATURES = 3000


def headline_frames(name):
    w, h, cam = HEADLINE_CASES[name]
    return synthetic.frame_pair(cam, w, h)


def headline_runs(pts, gt, w):
    """name -> input TrackData records of the headline fixtures' LK runs."""
    rng = np.random.default_rng(17)
    pred = gt + rng.normal(0.0, 0.7, gt.shape).astype(np.float32)
    return {"lk_zero": make_tracks(pts, None, float(w), 0.8), "lk_pred": make_tracks(pts, pred - pts, float(w), 0.8)}


def make_headline_reference(out_dir):
    compact = {}
    for name, (w, h, cam) in HEADLINE_CASES.items():
        prev, nxt, warp = headline_frames(name)
        compact[f"{name}/prev/sha"] = np.array(_sha(prev))
        compact[f"{name}/next/sha"] = np.array(_sha(nxt))
        s0 = REF.select(prev, np.zeros((0, 2), np.float32), HEADLINE_FEATURES)
        pts = s0["sel"].astype(np.float32)
        compact[f"{name}/sel0"] = pts
        gt = synthetic.flow_texture(warp, pts.astype(np.float64)).astype(np.float32)
        compact[f"{name}/gt"] = gt
        for tag, t in headline_runs(pts, gt, w).items():
            out = REF.lk(prev, nxt, t)
            compact[f"{name}/{tag}/offset"] = t["offset"].copy()
            compact[f"{name}/{tag}/track"] = out["track"].copy()
            compact[f"{name}/{tag}/status"] = out["track_status"].copy()
            if tag == "lk_zero":
                alive = out["track"][out["track_status"] != 0].astype(np.float32)
                s1 = REF.select(nxt, alive, HEADLINE_FEATURES - len(alive))
                compact[f"{name}/sel1/alive"] = alive
                compact[f"{name}/sel1/sel"] = s1["sel"]
        print(name, "features", len(pts), "tracked", int((compact[f"{name}/lk_zero/status"] != 0).sum()),
              "new", len(compact[f"{name}/sel1/sel"]))
    os.makedirs(out_dir, exist_ok=True)
    np.savez_compressed(os.path.join(out_dir, "headline_reference.npz"), **compact)
    print("wrote headline_reference.npz")


# CPU-path pinning: the reference's GPU pyramid of a 512x512 random uint8 frame (levels 0-3 are what
# the reference's own test compares with its CPU uint8 pyramid, image_pyramid_test.cpp:143-227), plain
# and box prefiltered (ref_pyramid_ex), as SHA-256 hashes of every level.
CPU_PYR_SIZE = 512


def cpu_pyramid_frame():
    """Random uint8 frame as the reference's test draws it (ImageMatrix<uint8_t>::Random * 100, which
    wraps modulo 256), from a fixed seed."""
    rng = np.random.default_rng(143)
    return ((rng.integers(0, 256, (CPU_PYR_SIZE, CPU_PYR_SIZE)) * 100) % 256).astype(np.uint8)


def make_cpu_pyramid_reference(out_dir):
    img = cpu_pyramid_frame()
    compact = {"frame/sha": np.array(_sha(img))}
    lib = _lib()
    for box in (0, 1):
        sizes = level_sizes(CPU_PYR_SIZE, CPU_PYR_SIZE, 10)
        total = sum(a * b for a, b in sizes)
        lv, gx, gy = (np.zeros(total, np.float32) for _ in range(3))
        n = ctypes.c_int(0)
        rc = lib.ref_pyramid_ex(_ptr(img), CPU_PYR_SIZE, CPU_PYR_SIZE, 0, box, 10, ctypes.byref(n), _ptr(lv), _ptr(gx),
                                _ptr(gy))
        assert rc == 0 and n.value == len(sizes), (rc, n.value)
        off = 0
        for l, (a, b) in enumerate(sizes):
            compact[f"box{box}/L{l}/sha"] = np.array(_sha(lv[off:off + a * b].reshape(b, a)))
            off += a * b
    os.makedirs(out_dir, exist_ok=True)
    np.savez_compressed(os.path.join(out_dir, "cpu_pyramid_reference.npz"), **compact)
    print("wrote cpu_pyramid_reference.npz")


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("step", choices=["inputs", "reference", "stereo-inputs", "stereo-reference", "input-reference",
                                        "st-reference", "headline-reference", "cpu-pyramid-reference"])
    ap.add_argument("--out", default=HERE)
    a = ap.parse_args()
    if a.step == "inputs":
        make_inputs(os.path.join(HERE, "inputs.npz"))
    elif a.step == "stereo-inputs":
        make_stereo_inputs(os.path.join(HERE, "stereo_inputs.npz"))
    elif a.step == "stereo-reference":
        make_stereo_reference(a.out)
    elif a.step == "input-reference":
        make_input_reference(a.out)
    elif a.step == "st-reference":
        make_st_reference(a.out)
    elif a.step == "headline-reference":
        make_headline_reference(a.out)
    elif a.step == "cpu-pyramid-reference":
        make_cpu_pyramid_reference(a.out)
    else:
        make_reference(a.out)
