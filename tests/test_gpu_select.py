"""Selection on the GPU: response within __logf's error of the oracle, the selected features equal
to the oracle's selection run on the GPU's own response map, and equal to the reference's."""

import os

import numpy as np
import pytest
import torch

from conftest import gpu_pyramid

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dctx():
    os.environ["CUVSLAM_FE_DEBUG_MAPS"] = "1"
    from cuvslam_b200.frontend import Context

    c = Context(0)
    del os.environ["CUVSLAM_FE_DEBUG_MAPS"]
    yield c
    c.close()


def _select(ctx, pyr, alive, nd, borders=(0, 0, 0, 0), mask=None):
    from cuvslam_b200.frontend import Selection

    s = Selection(ctx)
    out = s.compute_gftt_and_select_features(pyr, *borders, mask, alive, nd)
    w, h = pyr.level_size(0)
    resp, nms = s.debug_maps(w, h)
    return out.cpu().numpy(), resp.cpu().numpy(), nms.cpu().numpy()


def _same_selection(a, b, tol=1e-4):
    assert a.shape == b.shape, (a.shape, b.shape)
    if len(a):
        np.testing.assert_allclose(a, b, rtol=0, atol=tol)


@pytest.mark.parametrize("name", ["c1", "half", "odd", "tiny"])
def test_golden_frames(dctx, oracle, golden, name):
    inp, ref = golden
    img = inp[f"{name}/prev"]
    pyr = gpu_pyramid(dctx, img)
    for tag, borders in (("sel0", (0, 0, 0, 0)), ("sel1", (3, 4, 5, 6))):
        alive = ref[f"{name}/sel1/alive"] if tag == "sel1" else np.zeros((0, 2), np.float32)
        nd = 450 - len(alive)
        sel, resp, nms = _select(dctx, pyr, alive, nd, borders)
        o = oracle.pyramid(img)
        oresp = oracle.gftt(o[0][1], o[0][2])
        assert np.abs(resp - oresp).max() < 1e-5  # __logf vs logf
        s = oracle.select(resp, alive, nd, borders)
        np.testing.assert_array_equal(nms, s["nms"])
        _same_selection(sel, s["sel"], 2e-4)
        # the reference: same set (the order of exactly equal strengths is arbitrary there)
        rsel = ref[f"{name}/{tag}/sel"]
        assert len(sel) == len(rsel)
        if len(sel):
            key = lambda a: a[np.lexsort((a[:, 0], a[:, 1]))]
            np.testing.assert_allclose(key(sel), key(rsel), rtol=0, atol=1e-5)


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_random_configurations(dctx, oracle, seed):
    from cuvslam_b200 import synthetic

    rng = np.random.default_rng(seed)
    w, h = [(640, 480), (1280, 720), (1241, 376)][seed]
    img, _, _ = synthetic.frame_pair(seed + 20, w, h)
    pyr = gpu_pyramid(dctx, img)
    alive = np.stack([rng.uniform(0, w - 1, 300), rng.uniform(0, h - 1, 300)], 1).astype(np.float32)
    mask = np.zeros((h, w), np.uint8)
    mask[: h // 5, : w // 3] = 1
    # 10000 wanted: more kept candidates than the headline's, up to the whole 1280x720 frame's cells
    for nd, a, m, borders in ((1000, None, None, (0, 0, 0, 0)), (600, alive, mask, (10, 20, 30, 40)),
                              (0, alive, None, (0, 0, 0, 0)), (5, None, None, (0, 0, 0, 0)),
                              (10000, None, None, (0, 0, 0, 0))):
        sel, resp, _ = _select(dctx, pyr, a, nd, borders, m)
        s = oracle.select(resp, a, nd, borders, m)
        _same_selection(sel, s["sel"], 2e-4)
        assert len(sel) <= nd


def test_flat_image_selects_nothing(dctx):
    img = np.full((64, 80), 100, np.uint8)
    pyr = gpu_pyramid(dctx, img)
    sel, resp, _ = _select(dctx, pyr, None, 50)
    assert len(sel) == 0
    assert np.all(resp == 0)


def test_deterministic_across_runs(dctx):
    from cuvslam_b200 import synthetic

    img, _, _ = synthetic.frame_pair(9, 1280, 720)
    pyr = gpu_pyramid(dctx, img)
    a = _select(dctx, pyr, None, 2000)[0]
    for _ in range(3):
        b = _select(dctx, pyr, None, 2000)[0]
        np.testing.assert_array_equal(a, b)
