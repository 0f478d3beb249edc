"""The restated reference CPU tracker (the timed CPU baseline) behaves like cuVSLAM's CPU path."""

import numpy as np

from cuvslam_b200 import synthetic


def test_u8_pyramid_rule(oracle):
    img = np.random.default_rng(0).integers(0, 256, (480, 752), dtype=np.uint8)
    cam = oracle.CpuCamera(752, 480).build(img)
    # d/2 sizes while >= 15: 752x480 -> ... -> 23x15
    sizes = [cam.level(l)[0].shape[::-1] for l in range(cam.levels())]
    assert sizes == [(752, 480), (376, 240), (188, 120), (94, 60), (47, 30), (23, 15)]
    # binomial with rounding: level 1 of a constant image is that constant
    c = oracle.CpuCamera(64, 48).build(np.full((48, 64), 77, np.uint8))
    assert np.all(c.level(1)[0] == 77)
    # gradients: zero 3-px border
    gx = cam.level(0)[1]
    assert np.all(gx[:, :3] == 0) and np.all(gx[:, -3:] == 0)


def test_tracks_known_motion():
    from oracle import oracle as O

    prev, nxt, warp = synthetic.frame_pair(0, 752, 480)
    a, b = O.CpuCamera(752, 480).build(prev), O.CpuCamera(752, 480).build(nxt)
    sel = a.select(None, 450)
    assert 300 <= len(sel) <= 450
    out, st = b.track_from(a, sel)
    gt = synthetic.flow_texture(warp, sel.astype(np.float64))
    ok = st == 1
    assert ok.mean() > 0.5
    assert np.median(np.linalg.norm(out[ok] - gt[ok], axis=1)) < 0.3


def test_frame_step_threads_agree():
    from oracle import oracle as O

    cams = [(160, 120), (200, 150), (320, 240)]
    prevs, curs, imgs, xys = [], [], [], []
    for i, (w, h) in enumerate(cams):
        p, n, _ = synthetic.frame_pair(i, w, h)
        prevs.append(O.CpuCamera(w, h).build(p))
        curs.append(O.CpuCamera(w, h))
        imgs.append(n)
        xys.append(prevs[-1].select(None, 100))
    r1 = O.cpu_frame_step(prevs, curs, imgs, xys, None, [50] * 3, 1)
    r4 = O.cpu_frame_step(prevs, curs, imgs, xys, None, [50] * 3, 4)
    for a, b in zip(r1, r4):
        for x, y in zip(a, b):
            np.testing.assert_array_equal(x, y)


def test_box_prefilter_equals_the_gpu_rule(oracle):
    """BoxBlur3Cpu (sof/box_blur.cpp:25-55) and the reference's GPU box prefilter give the same level 0
    on uint8 input (both are the exact integer rule)."""
    img = np.random.default_rng(3).integers(0, 256, (61, 97), dtype=np.uint8)
    cam = oracle.CpuCamera(97, 61).build(img, box3=True)
    np.testing.assert_array_equal(cam.level(0)[0], oracle.level0(img, box=True))


def test_u8_pyramid_within_one_percent_of_the_reference_gpu_pyramid(oracle):
    """The reference's CPU/GPU relation (image_pyramid_test.cpp:143-227, ImagePyramidU8 and
    ImagePyramidU8Prefilter): on a 512x512 random frame, levels 0-3 of the CPU uint8 pyramid are within
    1% (relative Frobenius norm, Eigen's isApprox) of the GPU pyramid, with and without the box
    prefilter.  The GPU pyramid here is the oracle's, which equals the reference kernels' output bit
    for bit on this frame (hashes in tests/golden/cpu_pyramid_reference.npz, made on a B200)."""
    import hashlib
    import os
    import sys

    import pytest

    from conftest import ROOT

    path = os.path.join(ROOT, "tests", "golden", "cpu_pyramid_reference.npz")
    if not os.path.exists(path):
        pytest.skip("cpu_pyramid_reference.npz not generated")
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import make_golden as MG

    ref = np.load(path)
    img = MG.cpu_pyramid_frame()
    sha = lambda a: hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()
    assert sha(img) == str(ref["frame/sha"])
    n = MG.CPU_PYR_SIZE
    for box in (False, True):
        gpu = oracle.pyramid_f32(oracle.level0(img, box))
        for l, (lv, _, _) in enumerate(gpu):
            assert sha(lv) == str(ref[f"box{int(box)}/L{l}/sha"]), (box, l)
        cam = oracle.CpuCamera(n, n).build(img, box3=box)
        assert cam.levels() == len(gpu)
        for l in range(4):
            a, b = cam.level(l)[0].astype(np.float64), gpu[l][0].astype(np.float64)
            assert np.linalg.norm(a - b) <= 0.01 * min(np.linalg.norm(a), np.linalg.norm(b)), (box, l)


def test_patch_ramp_known_answer(oracle):
    """interpolation_test.cpp:24-72: on a vertical (then horizontal) linear ramp, the exact-bilinear
    patch centred at (10.75, 10.75) holds row (column) index + 10.75 - half - 0.5 exactly; half = 4
    for the tracker's 9x9 patch (2 for the test's 5x5)."""
    n = 240  # ramp values stay within uint8
    ramp = np.tile(np.arange(n, dtype=np.uint8)[:, None], (1, n))
    expected_first = 10.75 - 4 - 0.5
    for img, axis in ((ramp, 0), (np.ascontiguousarray(ramp.T), 1)):
        p = oracle.CpuCamera(n, n).build(img).patch(0, 10.75, 10.75)
        assert p is not None
        idx = np.arange(9, dtype=np.float32)
        want = (idx[:, None] if axis == 0 else idx[None, :]) + np.float32(expected_first)
        np.testing.assert_array_equal(p, np.broadcast_to(want, (9, 9)))
    # a patch whose box leaves the image is refused
    assert oracle.CpuCamera(n, n).build(ramp).patch(0, 3.0, 3.0) is None


def test_features_parallel_step_equals_serial():
    """The features-parallel variant (cameras in turn, each camera's tracking over the threads) gives
    the single-threaded results."""
    from oracle import oracle as O

    cams = [(200, 150), (320, 240)]
    prevs, curs, imgs, xys = [], [], [], []
    for i, (w, h) in enumerate(cams):
        p, n, _ = synthetic.frame_pair(i + 5, w, h)
        prevs.append(O.CpuCamera(w, h).build(p))
        curs.append(O.CpuCamera(w, h))
        imgs.append(n)
        xys.append(prevs[-1].select(None, 150))
    r1 = O.cpu_frame_step(prevs, curs, imgs, xys, None, [60] * 2, 1)
    r4 = O.cpu_frame_step(prevs, curs, imgs, xys, None, [60] * 2, 4, features_parallel=True)
    for a, b in zip(r1, r4):
        for x, y in zip(a, b):
            np.testing.assert_array_equal(x, y)
