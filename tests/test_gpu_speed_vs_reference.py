"""Device time of this library's stages against the reference's own GPU kernels (compiled from the
cuVSLAM sources for sm_100a into oracle/_ref by oracle/build_ref.sh) on the same inputs: one
1920x1200 frame pair (seeded scene, similarity warp), 8192 Shi-Tomasi features with predicted
offsets.  Stages: the current frame's pyramid + gradients (uint8 in device memory -> every level),
pyramidal LK (the default sampling, the texture unit's own filtering as the reference samples, and
the FP32 restatement of that filtering, FE_SAMPLE_TEXTURE; 8191 tracks and the same features seven
times over, 57 337), the affine tracker (0 shift + 20 full steps) and its cached variant.  Both
sides are timed with CUDA events around the stage alone (records reset before each run, outside the
timed interval, and the host's enqueue time hidden behind a spin kernel), mean of 20 runs after 3
warm-up runs.  Prints one JSON line.
Asserts that the pyramid, LK in the default sampling (both track counts) and the affine tracker are
faster than the reference's kernels.  The FP32 restatement is reported, not asserted: it computes
the texture unit's weight rule in FP32 from shared-memory windows (the price of bit-identical
results with the oracle) and is slower than the reference's kernel on one camera (about 0.85x)."""

import ctypes
import json
import os

import numpy as np
import pytest
import torch

from conftest import ROOT

pytestmark = pytest.mark.gpu

REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libcuvslam_ref.so")
W, H, N, REPS = 1920, 1200, 8192, 20


def _ref_stage(lib, prev, nxt, tracks, which):
    ms = ctypes.c_float(0.0)
    rc = lib.ref_time_stage(prev.ctypes.data_as(ctypes.c_void_p), nxt.ctypes.data_as(ctypes.c_void_p), W, H, 10,
                            tracks.ctypes.data_as(ctypes.c_void_p), len(tracks), which, 0, 20, REPS,
                            ctypes.byref(ms))
    assert rc == 0, rc
    return ms.value


def _ours(fn, reset=None):
    """Device time of fn: the stream is kept busy by a short spin kernel while the host enqueues fn
    (so the Python call's host time is not counted, as the reference's C harness counts none)."""
    stream = torch.cuda.current_stream()
    tot = 0.0
    for r in range(REPS + 3):
        if reset is not None:
            reset()
        torch.cuda._sleep(1_000_000)
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        fn()
        e.record(stream)
        torch.cuda.synchronize()
        if r >= 3:
            tot += s.elapsed_time(e)
    return tot / REPS


def test_stages_vs_reference_kernels(ctx):
    if not os.path.exists(REF_LIB):
        pytest.skip("oracle/_ref/libcuvslam_ref.so not built (needs the reference sources)")
    from cuvslam_b200 import _lib, synthetic
    from cuvslam_b200.frontend import (ImagePyramid, LKFeatureTracker, Selection, STFeatureTracker,
                                       STFeatureTrackerWithCache)
    from cuvslam_b200.types import make_tracks

    lib = ctypes.CDLL(REF_LIB)
    lib.ref_time_stage.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_int, ctypes.POINTER(ctypes.c_float)]
    prev, nxt, warp = synthetic.frame_pair(5, W, H)
    dev = torch.device("cuda", 0)
    pp = ImagePyramid(W, H, 10, device=dev).build(ctx, torch.from_numpy(prev).to(dev))
    cp = ImagePyramid(W, H, 10, device=dev)
    cur_u8 = torch.from_numpy(nxt).to(dev)
    cp.build(ctx, cur_u8)
    uv = Selection(ctx).compute_gftt_and_select_features(pp, 0, 0, 0, 0, None, None, N)
    pts = uv.cpu().numpy().astype(np.float32)
    gt = synthetic.flow_texture(warp, pts.astype(np.float64)).astype(np.float32)
    rec = make_tracks(pts, (gt - pts) + np.float32(0.5), 64.0, 0.8)
    src = torch.from_numpy(rec.view(np.uint8).reshape(len(rec), 80).copy()).to(dev)
    d = src.clone()
    torch.cuda.synchronize()

    ours, ref = {}, {}
    ours["pyramid"] = _ours(lambda: cp.build(ctx, cur_u8))
    ref["pyramid"] = _ref_stage(lib, prev, nxt, rec, 0)
    lk = LKFeatureTracker(ctx)  # the default sampling
    ours["lk"] = _ours(lambda: lk.track_points(pp, cp, d), lambda: d.copy_(src))
    ref["lk"] = _ref_stage(lib, prev, nxt, rec, 1)
    lk_fp32 = LKFeatureTracker(ctx, False, _lib.FE_SAMPLE_TEXTURE)
    ours["lk_texture"] = _ours(lambda: lk_fp32.track_points(pp, cp, d), lambda: d.copy_(src))
    ref["lk_texture"] = ref["lk"]
    # the same features seven times over: 57 337 tracks, the 32-camera step's track count
    rec7 = np.tile(rec, 7)
    src7 = torch.from_numpy(rec7.view(np.uint8).reshape(len(rec7), 80).copy()).to(dev)
    d7 = src7.clone()
    ours["lk_57k"] = _ours(lambda: lk.track_points(pp, cp, d7), lambda: d7.copy_(src7))
    ours["lk_texture_57k"] = _ours(lambda: lk_fp32.track_points(pp, cp, d7), lambda: d7.copy_(src7))
    ref["lk_57k"] = _ref_stage(lib, prev, nxt, rec7, 1)
    ref["lk_texture_57k"] = ref["lk_57k"]
    st = STFeatureTracker(ctx, 0, 20)
    ours["affine"] = _ours(lambda: st.track_points(pp, cp, d), lambda: d.copy_(src))
    ref["affine"] = _ref_stage(lib, prev, nxt, rec, 2)
    stc = STFeatureTrackerWithCache(ctx, 0, 20)
    d.copy_(src)
    cache = stc.build_points_cache(pp, d)
    torch.cuda.synchronize()
    src_c = d.clone()
    ours["affine_cached"] = _ours(lambda: stc.track_points(cp, cache, d), lambda: d.copy_(src_c))
    ref["affine_cached"] = _ref_stage(lib, prev, nxt, rec, 3)
    line = {"workload": f"{W}x{H} pair, {len(rec)} Shi-Tomasi features (lk_57k: {len(rec7)} tracks)", "ours_ms": ours, "reference_ms": ref,
            "speedup": {k: ref[k] / ours[k] for k in ours}}
    print(json.dumps(line))
    for k in ("pyramid", "lk", "lk_57k", "affine", "affine_cached"):
        assert ours[k] <= ref[k], (k, ours[k], ref[k])
    assert all(v > 0 for v in ours.values()) and all(v > 0 for v in ref.values())


def test_multicam_frame_vs_reference_path(ctx):
    """The 32-camera frame step (bench.py's workload: 12 x 640x480, 12 x 1280x720, 8 x 1920x1200,
    300-3000 features each) through the reference's GPU path, one camera after another on one stream
    as MonoSOFGPU runs it (pyramid, lk_track, GPUSelection with its read-backs and host quota loop;
    ref_time_frame, host clock), against this library's batched step (one CUDA graph, CUDA events).
    Prints one JSON line; asserts the batched step is faster."""
    if not os.path.exists(REF_LIB):
        pytest.skip("oracle/_ref/libcuvslam_ref.so not built (needs the reference sources)")
    import bench
    from cuvslam_b200.frontend import Batch, CameraFrame, ImagePyramid, Selection, tracks_to_device
    from cuvslam_b200.types import make_tracks

    lib = ctypes.CDLL(REF_LIB)
    lib.ref_time_frame.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   ctypes.POINTER(ctypes.c_float)]
    shapes, counts, prevs, nexts = bench.workload()
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream()
    sel = Selection(ctx)
    frames, pristine, hosts = [], [], []
    for (w, h), p, nx, n in zip(shapes, prevs, nexts, counts):
        pp = ImagePyramid(w, h, device=dev).build(ctx, torch.from_numpy(p).to(dev))
        xy = sel.compute_gftt_and_select_features(pp, 0, 0, 0, 0, None, None, n).cpu().numpy()
        t = make_tracks(xy, None, float(w), 0.8)
        hosts.append(t)
        td = tracks_to_device(t, dev)
        pristine.append(td.clone())
        frames.append(CameraFrame(torch.from_numpy(nx).to(dev), ImagePyramid(w, h, device=dev), pp, td, n, (0, 0, 0, 0)))
    batch = Batch(ctx, frames)  # the default sampling
    batch.autotune(reps=10, stream=stream)

    def restore():
        for f, p0 in zip(frames, pristine):
            f.tracks.copy_(p0)

    ours_ms = _ours(lambda: batch.run(stream), restore)
    batch.close()
    ref_ms = []
    for (w, h), p, nx, n, t in zip(shapes, prevs, nexts, counts, hosts):
        ms = ctypes.c_float(0.0)
        rc = lib.ref_time_frame(np.ascontiguousarray(p).ctypes.data_as(ctypes.c_void_p),
                                np.ascontiguousarray(nx).ctypes.data_as(ctypes.c_void_p), w, h, 10,
                                t.ctypes.data_as(ctypes.c_void_p), len(t), n, 5, ctypes.byref(ms))
        assert rc == 0, rc
        ref_ms.append(ms.value)
    tracks = sum(len(t) for t in hosts)
    line = {"workload": "multicam32 frame step", "tracks": tracks, "ours_batched_ms": ours_ms,
            "reference_path_ms": float(sum(ref_ms)), "speedup": float(sum(ref_ms)) / ours_ms,
            "reference_per_camera_ms": {"640x480": float(np.mean(ref_ms[:12])), "1280x720": float(np.mean(ref_ms[12:24])),
                                        "1920x1200": float(np.mean(ref_ms[24:]))}}
    print(json.dumps(line))
    assert ours_ms < sum(ref_ms)
