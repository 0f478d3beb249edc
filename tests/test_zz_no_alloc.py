"""fe_select_noalloc: selection for callers that cannot allocate device memory while they run (a
tracking loop that reserves everything at start-up, or a process whose device memory belongs to its
own pool allocator).  Its scratch is a static array inside the library; the results must equal
fe_select's, call after call, although every call reuses (and must first clear) the same scratch.

This file is collected last on purpose, so a run that stops at the first failure has run every other
test first; it also passes on its own in a fresh process."""

import ctypes

import numpy as np
import pytest
import torch

from cuvslam_b200 import _lib, synthetic
from cuvslam_b200.frontend import ImagePyramid

pytestmark = pytest.mark.gpu


def _call(fn, ctx, pyr, alive, num_desired, borders=(0, 0, 0, 0)):
    out = torch.zeros((max(num_desired, 1), 2), dtype=torch.float32, device="cuda")
    cnt = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    a = None if alive is None else torch.from_numpy(np.ascontiguousarray(alive, np.float32)).cuda()
    n_alive = 0 if alive is None else len(alive)
    args = [ctypes.byref(pyr.desc), *borders, None, 0, None if a is None else ctypes.c_void_p(a.data_ptr()), n_alive,
            num_desired, ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(cnt.data_ptr()),
            ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)]
    lib = _lib.load()
    rc = lib.fe_select(ctx.handle, *args) if fn == "fe_select" else lib.fe_select_noalloc(*args)
    assert rc == 0, lib.fe_status_string(rc)
    torch.cuda.synchronize()
    n = int(cnt.item())
    return out[:n].cpu().numpy()


def test_matches_fe_select_on_consecutive_calls(ctx):
    # call 1: 1280x720, no alive features; call 2: 640x480 with alive features and borders.  The
    # second call starts on the scratch the first one left behind.
    img1, _, _ = synthetic.frame_pair(31, 1280, 720)
    img2, _, _ = synthetic.frame_pair(32, 640, 480)
    p1 = ImagePyramid(1280, 720).build(ctx, torch.from_numpy(img1).cuda())
    p2 = ImagePyramid(640, 480).build(ctx, torch.from_numpy(img2).cuda())
    rng = np.random.default_rng(4)
    alive = np.stack([rng.uniform(0, 639, 200), rng.uniform(0, 479, 200)], 1).astype(np.float32)
    cases = [(p1, None, 1500, (0, 0, 0, 0)), (p2, alive, 400, (4, 5, 6, 7))]
    for pyr, a, nd, borders in cases:
        got = _call("fe_select_noalloc", ctx, pyr, a, nd, borders)
        want = _call("fe_select", ctx, pyr, a, nd, borders)
        assert len(got) > 0
        assert got.shape == want.shape
        np.testing.assert_allclose(got, want, rtol=0, atol=2e-4)
    # and the first case again, after the second one used the scratch
    got = _call("fe_select_noalloc", ctx, p1, None, 1500)
    want = _call("fe_select", ctx, p1, None, 1500)
    np.testing.assert_allclose(got, want, rtol=0, atol=2e-4)


def test_rejects_sizes_beyond_the_static_scratch(ctx):
    lib = _lib.load()
    big = ImagePyramid(2112, 64)  # wider than the 2048-pixel limit; no kernel runs
    out = torch.zeros((10, 2), dtype=torch.float32, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = lib.fe_select_noalloc(ctypes.byref(big.desc), 0, 0, 0, 0, None, 0, None, 0, 10,
                               ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(cnt.data_ptr()), None)
    assert rc == 4  # FE_ERR_CAPACITY
    small = ImagePyramid(64, 64)
    rc = lib.fe_select_noalloc(ctypes.byref(small.desc), 0, 0, 0, 0, None, 0, None, 0, 16400,
                               ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(cnt.data_ptr()), None)
    assert rc == 4
