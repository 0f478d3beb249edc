"""fe_select_noalloc: selection for callers that cannot allocate device memory while they run (a
tracking loop that reserves everything at start-up, or a process whose device memory belongs to its
own pool allocator).  Its scratch is a static array inside the library; the results must equal
fe_select's bit for bit, call after call, although every call reuses (and must first clear) the same
scratch.

This file is collected last on purpose, so a run that stops at the first failure has run every other
test first; it also passes on its own in a fresh process."""

import ctypes
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest
import torch

from cuvslam_b200 import _lib, synthetic
from cuvslam_b200.frontend import ImagePyramid

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _call(fn, ctx, pyr, alive, num_desired, borders=(0, 0, 0, 0), mask=None):
    out = torch.zeros((max(num_desired, 1), 2), dtype=torch.float32, device="cuda")
    cnt = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    a = None if alive is None else torch.from_numpy(np.ascontiguousarray(alive, np.float32)).cuda()
    n_alive = 0 if alive is None else len(alive)
    m = None if mask is None else torch.from_numpy(np.ascontiguousarray(mask, np.uint8)).cuda()
    args = [ctypes.byref(pyr.desc), *borders, None if m is None else ctypes.c_void_p(m.data_ptr()),
            0 if m is None else m.shape[1], None if a is None else ctypes.c_void_p(a.data_ptr()), n_alive,
            num_desired, ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(cnt.data_ptr()),
            ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)]
    lib = _lib.load()
    rc = lib.fe_select(ctx.handle, *args) if fn == "fe_select" else lib.fe_select_noalloc(*args)
    assert rc == 0, lib.fe_status_string(rc)
    torch.cuda.synchronize()
    n = int(cnt.item())
    return out[:n].cpu().numpy()


def _same(got, want):
    assert got.shape == want.shape, (got.shape, want.shape)
    assert np.array_equal(got, want), np.abs(got - want).max()


def _blob_mask(w, h, seed):
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:h, 0:w]
    m = np.zeros((h, w), np.uint8)
    for _ in range(6):
        cx, cy, r = rng.uniform(0, w), rng.uniform(0, h), rng.uniform(20, 90)
        m[(xx - cx) ** 2 + (yy - cy) ** 2 < r * r] = 255
    return m


def test_matches_fe_select_on_consecutive_calls(ctx):
    # call 1: 1280x720, no alive features; call 2: 640x480 with alive features, borders and a mask.
    # The second call starts on the scratch the first one left behind.
    img1, _, _ = synthetic.frame_pair(31, 1280, 720)
    img2, _, _ = synthetic.frame_pair(32, 640, 480)
    p1 = ImagePyramid(1280, 720).build(ctx, torch.from_numpy(img1).cuda())
    p2 = ImagePyramid(640, 480).build(ctx, torch.from_numpy(img2).cuda())
    rng = np.random.default_rng(4)
    alive = np.stack([rng.uniform(0, 639, 200), rng.uniform(0, 479, 200)], 1).astype(np.float32)
    mask = _blob_mask(640, 480, 5)
    cases = [(p1, None, 1500, (0, 0, 0, 0), None), (p2, alive, 400, (4, 5, 6, 7), mask)]
    for pyr, a, nd, borders, m in cases:
        got = _call("fe_select_noalloc", ctx, pyr, a, nd, borders, m)
        want = _call("fe_select", ctx, pyr, a, nd, borders, m)
        assert len(got) > 0
        _same(got, want)
    # the mask took effect: no feature on a masked pixel
    got = _call("fe_select_noalloc", ctx, p2, alive, 400, (4, 5, 6, 7), mask)
    xi, yi = np.clip(got[:, 0].astype(int), 0, 639), np.clip(got[:, 1].astype(int), 0, 479)
    assert not mask[yi, xi].any()
    # and the first case again, after the second one used the scratch
    _same(_call("fe_select_noalloc", ctx, p1, None, 1500), _call("fe_select", ctx, p1, None, 1500))


def test_largest_frame_that_fits(ctx):
    # 2048x2048, the largest layout the static array holds: twice in a row, with alive features
    img, _, _ = synthetic.frame_pair(33, 2048, 2048)
    p = ImagePyramid(2048, 2048).build(ctx, torch.from_numpy(img).cuda())
    rng = np.random.default_rng(8)
    alive = np.stack([rng.uniform(0, 2047, 3000), rng.uniform(0, 2047, 3000)], 1).astype(np.float32)
    for _ in range(2):
        got = _call("fe_select_noalloc", ctx, p, alive, 8000, (2, 3, 4, 5))
        want = _call("fe_select", ctx, p, alive, 8000, (2, 3, 4, 5))
        assert len(got) > 0
        _same(got, want)


def test_small_frame_large_request_is_accepted(ctx):
    # kept candidates are bounded by the frame's cells, as in fe_select: 64x64 has 64 cells
    img, _, _ = synthetic.frame_pair(34, 64, 64)
    p = ImagePyramid(64, 64).build(ctx, torch.from_numpy(img).cuda())
    _same(_call("fe_select_noalloc", ctx, p, None, 16000), _call("fe_select", ctx, p, None, 16000))


def test_rejects_sizes_beyond_the_static_scratch(ctx):
    lib = _lib.load()
    big = ImagePyramid(2112, 64)  # wider than the 2048-pixel limit; no kernel runs
    out = torch.zeros((10, 2), dtype=torch.float32, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = lib.fe_select_noalloc(ctypes.byref(big.desc), 0, 0, 0, 0, None, 0, None, 0, 10,
                               ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(cnt.data_ptr()), None)
    assert rc == _lib.FE_ERR_CAPACITY
    small = ImagePyramid(64, 64)
    rc = lib.fe_select_noalloc(ctypes.byref(small.desc), 0, 0, 0, 0, None, 0, None, 0, 16400,
                               ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(cnt.data_ptr()), None)
    assert rc == _lib.FE_ERR_CAPACITY


def test_rejects_misaligned_planes(ctx):
    # a level-0 gradient plane off a 16-byte boundary is refused before any launch
    lib = _lib.load()
    p = ImagePyramid(640, 480)
    d = _lib.FePyramid.from_buffer_copy(p.desc)
    d.grad_x[0] = d.grad_x[0] + 4
    out = torch.zeros((10, 2), dtype=torch.float32, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = lib.fe_select_noalloc(ctypes.byref(d), 0, 0, 0, 0, None, 0, None, 0, 10, ctypes.c_void_p(out.data_ptr()),
                               ctypes.c_void_p(cnt.data_ptr()), None)
    assert rc == _lib.FE_ERR_INVALID_ARGUMENT


_CAPTURE_SCRIPT = textwrap.dedent("""
    import ctypes, sys, torch
    sys.path.insert(0, %r)
    from cuvslam_b200 import _lib
    from cuvslam_b200.frontend import Context, ImagePyramid
    ctx = Context(0)
    p = ImagePyramid(320, 240).build(ctx, torch.zeros((240, 320), dtype=torch.uint8, device="cuda"))
    out = torch.zeros((10, 2), dtype=torch.float32, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
    lib = _lib.load()
    s = torch.cuda.Stream()
    def call():
        return lib.fe_select_noalloc(ctypes.byref(p.desc), 0, 0, 0, 0, None, 0, None, 0, 10,
                                     ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(cnt.data_ptr()),
                                     ctypes.c_void_p(s.cuda_stream))
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        inside = call()
    del g
    after = call()
    torch.cuda.synchronize()
    print("RESULT", inside, after)
""")


def test_first_call_inside_a_capture_is_refused():
    # in a fresh process (the device is not set up yet): refused inside the capture, fine after it
    r = subprocess.run([sys.executable, "-c", _CAPTURE_SCRIPT % ROOT], capture_output=True, text=True, timeout=600)
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("RESULT")]
    assert r.returncode == 0 and lines, r.stdout + r.stderr
    inside, after = (int(v) for v in lines[0].split()[1:])
    assert inside == _lib.FE_ERR_INVALID_ARGUMENT
    assert after == _lib.FE_OK
