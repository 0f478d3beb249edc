"""The compiled drop-in shim (include/cuvslam_fe_shim.hpp) on the GPU: one MonoSOFGPU-style frame
through the restated wrapper classes (tests/shim_frame.cpp) equals the same steps through the Python
binding bit for bit: the previous frame's selection (with and without a mask), the LK records (2-D
and horizontal tracker), and the next frame's selection with the tracked features alive, appended to
a vector that already holds an entry (the reference counts it against the limit)."""

import ctypes

import numpy as np
import pytest
import torch

import shim_lib
from conftest import assert_tracks_equal
from cuvslam_b200 import synthetic
from cuvslam_b200.frontend import ImagePyramid, LKFeatureTracker, Selection, tracks_from_device, tracks_to_device
from cuvslam_b200.types import TRACK_DTYPE, make_tracks

pytestmark = pytest.mark.gpu

W, H, K = 752, 480, 450


@pytest.fixture(scope="module")
def shim(tmp_path_factory):
    if shim_lib.compile_args() is None:
        pytest.skip("g++ not available")
    lib = ctypes.CDLL(shim_lib.build(str(tmp_path_factory.mktemp("shim"))))
    P, I = ctypes.c_void_p, ctypes.c_int
    lib.shim_frame.argtypes = [P, P, I, I, I, P, I, P, P, P, P, P]
    lib.shim_last_error.restype = ctypes.c_char_p
    return lib


def _shim_frame(lib, prev, nxt, mask, horizontal):
    sel0 = np.zeros((K, 2), np.float32)
    sel1 = np.zeros((K, 2), np.float32)
    tracks = np.zeros(K, TRACK_DTYPE)
    n0, n1 = ctypes.c_int(0), ctypes.c_int(0)
    m = None if mask is None else np.ascontiguousarray(mask, np.uint8)
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    rc = lib.shim_frame(P(prev), P(nxt), W, H, K, None if m is None else P(m), int(horizontal), P(sel0),
                        ctypes.byref(n0), P(tracks), P(sel1), ctypes.byref(n1))
    assert rc == 0, lib.shim_last_error().decode()
    return sel0[:n0.value], tracks[:n0.value], sel1[:n1.value]


def _python_frame(ctx, prev, nxt, mask, horizontal):
    pp = ImagePyramid(W, H).build(ctx, torch.from_numpy(prev).cuda())
    cp = ImagePyramid(W, H).build(ctx, torch.from_numpy(nxt).cuda())
    sel = Selection(ctx)
    m = None if mask is None else torch.from_numpy(mask).cuda()
    s0 = sel.compute_gftt_and_select_features(pp, 0, 0, 0, 0, m, None, K).cpu().numpy()
    d = tracks_to_device(make_tracks(s0, None, float(W), 0.8))
    LKFeatureTracker(ctx, horizontal=horizontal).track_points(pp, cp, d)
    torch.cuda.synchronize()
    t = tracks_from_device(d)
    alive = t["track"][t["track_status"] != 0].astype(np.float32)
    k1 = max(0, K - len(alive))
    s1 = sel.compute_gftt_and_select_features(cp, 2, 3, 4, 5, None, torch.from_numpy(alive).cuda(), k1).cpu().numpy()
    return s0, t, s1[:max(0, k1 - 1)]  # one slot of the shim's vector was taken before the call


@pytest.mark.parametrize("masked,horizontal", [(False, False), (True, False), (False, True)])
def test_shim_frame_equals_python_binding(ctx, shim, masked, horizontal):
    prev, nxt, _ = synthetic.frame_pair(3, W, H)
    mask = None
    if masked:
        mask = np.zeros((H, W), np.uint8)
        mask[100:260, 200:500] = 1
    s0, t, s1 = _shim_frame(shim, prev, nxt, mask, horizontal)
    w0, wt, w1 = _python_frame(ctx, prev, nxt, mask, horizontal)
    assert len(s0) > 100
    np.testing.assert_array_equal(s0, w0)
    assert_tracks_equal(t, wt)
    np.testing.assert_array_equal(s1, w1)
    if masked:
        assert not mask[s0[:, 1].astype(int), s0[:, 0].astype(int)].any()


def test_unset_gradient_pyramid_is_refused(shim):
    assert shim.shim_unset_gradients_throws() == 1
