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
