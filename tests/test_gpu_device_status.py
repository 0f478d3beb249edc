"""Device-side failure reporting: the pyramid's bounded waits give up, the kernel still finishes, and
the context reports the fault (fe_device_status), without a GPU fault, trap or hang.

A wait limit of 0 makes every bounded wait give up at once (the tile's staging copy is then drained
with the full bound before the CTA exits, so nothing lands in a retired CTA).  After the limit is
restored the same context builds correct pyramids again: the item counters the failed launch left
are returned to zero by that launch's last CTA."""

import numpy as np
import pytest
import torch

from conftest import assert_tracks_equal
from cuvslam_b200 import _lib, synthetic
from cuvslam_b200.frontend import Batch, CameraFrame, Context, ImagePyramid, tracks_from_device, tracks_to_device
from cuvslam_b200.types import make_tracks

pytestmark = pytest.mark.gpu


def _levels(p):
    torch.cuda.synchronize()
    return [x.copy() for lv in p.to_numpy() for x in lv]


def test_wait_that_runs_out_is_reported(ctx):
    img, _, _ = synthetic.frame_pair(71, 1280, 720)
    dimg = torch.from_numpy(img).cuda()
    want = _levels(ImagePyramid(1280, 720).build(ctx, dimg))
    c = Context(0)
    try:
        assert c.device_status() == 0
        c.set_wait_limit(0)
        ImagePyramid(1280, 720).build(c, dimg)
        with pytest.raises(_lib.FeError, match="device fault"):
            c.device_status()
        # the flags were read and cleared; the kernel that gave up finished, the context still works
        assert c.device_status() == 0
        # raw call: both wait kinds gave up (tile staging: bit 0, deeper-level items: bit 1)
        ImagePyramid(1280, 720).build(c, dimg)
        import ctypes
        flags = ctypes.c_int32(0)
        rc = c.lib.fe_device_status(c.handle, None, ctypes.byref(flags))
        assert rc == _lib.FE_ERR_DEVICE_FAULT and flags.value == 3
        c.set_wait_limit(_lib.FE_DEFAULT_WAIT_LIMIT)
        for _ in range(3):  # every counter slot the failed builds used is clean again
            got = _levels(ImagePyramid(1280, 720).build(c, dimg))
            assert c.device_status() == 0
            for x, y in zip(got, want):
                assert np.array_equal(x, y)
    finally:
        c.close()


def test_batch_reports_and_recovers(ctx):
    c = Context(0)
    try:
        shapes = [(640, 480), (1280, 720)]
        frames, host = [], []
        for i, (w, h) in enumerate(shapes):
            p, n, _ = synthetic.frame_pair(80 + i, w, h)
            pp = ImagePyramid(w, h).build(c, torch.from_numpy(p).cuda())
            xy = np.stack([np.linspace(20, w - 20, 200), np.linspace(20, h - 20, 200)], 1).astype(np.float32)
            t = make_tracks(xy, None, float(w), 0.8)
            host.append(t)
            frames.append(CameraFrame(torch.from_numpy(n).cuda(), ImagePyramid(w, h), pp, tracks_to_device(t), 300,
                                      (0, 0, 0, 0)))
        good = Batch(c, frames)
        good.run()
        torch.cuda.synchronize()
        want = [(tracks_from_device(f.tracks), _levels(f.cur)) for f in frames]
        assert c.device_status() == 0
        c.set_wait_limit(0)
        bad = Batch(c, frames)  # plans with the limit in force
        for f, t in zip(frames, host):
            f.tracks.copy_(tracks_to_device(t))
        bad.run()
        import ctypes
        flags = ctypes.c_int32(0)
        rc = c.lib.fe_device_status(c.handle, None, ctypes.byref(flags))
        # the pyramid's staging (bit 0) and the response tiles' TMA staging (bit 2) gave up
        assert rc == _lib.FE_ERR_DEVICE_FAULT and (flags.value & 1) and (flags.value & 4), flags.value
        bad.close()
        c.set_wait_limit(_lib.FE_DEFAULT_WAIT_LIMIT)
        for _ in range(2):
            for f, t in zip(frames, host):
                f.tracks.copy_(tracks_to_device(t))
            good.run()
            assert c.device_status() == 0
            for f, (wt, wl) in zip(frames, want):
                assert_tracks_equal(tracks_from_device(f.tracks), wt)
                for x, y in zip(_levels(f.cur), wl):
                    assert np.array_equal(x, y)
        good.close()
    finally:
        c.close()
