"""LK with the texture unit's own filtering (FE_SAMPLE_HARDWARE, lk_hw.cu), the default sampling of
the LK wrappers.

Its samples are the reference's (the same hardware filtering at the same coordinates), its
arithmetic is written as the reference writes it and its window sums pair lanes as the reference's
warp reduction does, so it equals the reference kernels' outputs bit for bit:
  - against the reference kernels' outputs (tests/golden/reference.npz): every record field
    identical, for the 2-D, predicted, NCC-0.85, horizontal and 4-level runs;
  - against the oracle's wide texture mode (an FP64 restatement of the texture unit's filtering):
    statuses agree on >= 99% of tracks, positions within 0.01 px (max);
  - the batched step in this mode equals its per-camera calls bit for bit (same kernel).
"""

import ctypes

import numpy as np
import pytest
import torch

from conftest import assert_tracks_equal, gpu_pyramid
from cuvslam_b200 import _lib, synthetic
from cuvslam_b200.frontend import (Batch, CameraFrame, ImagePyramid, LKFeatureTracker, Selection, TrackFinish,
                                   track_mono, tracks_from_device, tracks_to_device)
from cuvslam_b200.types import make_tracks

pytestmark = pytest.mark.gpu
HW = _lib.FE_SAMPLE_HARDWARE


def _run(ctx, pp, cp, tracks, horizontal=False):
    d = tracks_to_device(tracks)
    LKFeatureTracker(ctx, horizontal, HW).track_points(pp, cp, d)
    torch.cuda.synchronize()
    return tracks_from_device(d)


def _agree(got, want, max_flips, max_px, med_px):
    flips = int((got["track_status"] != want["track_status"]).sum())
    assert flips <= max_flips, flips
    ok = (got["track_status"] == 1) & (want["track_status"] == 1)
    if ok.any():
        d = np.linalg.norm(got["track"][ok] - want["track"][ok], axis=1)
        assert d.max() <= max_px and np.median(d) <= med_px, (d.max(), np.median(d))
    return flips


@pytest.mark.parametrize("name", ["c1", "half", "odd"])
@pytest.mark.parametrize("run", ["lk_zero", "lk_pred", "lk_retrack", "lk_horiz", "lk_pred4"])
def test_matches_reference(ctx, golden, name, run):
    inp, ref = golden
    src = {"lk_horiz": "lk_zero", "lk_pred4": "lk_pred"}.get(run, run)
    tin, tout = ref[f"{name}/{src}/in"], ref[f"{name}/{run}/out"]
    ml = 4 if run == "lk_pred4" else 10
    pp, cp = gpu_pyramid(ctx, inp[f"{name}/prev"], ml), gpu_pyramid(ctx, inp[f"{name}/next"])
    assert_tracks_equal(_run(ctx, pp, cp, tin, run == "lk_horiz"), tout)


@pytest.mark.parametrize("name", ["c1", "half"])
def test_matches_oracle_wide(ctx, oracle, golden, name):
    inp, ref = golden
    tin = ref[f"{name}/lk_pred/in"]
    pp, cp = gpu_pyramid(ctx, inp[f"{name}/prev"]), gpu_pyramid(ctx, inp[f"{name}/next"])
    got = _run(ctx, pp, cp, tin)
    want = oracle.lk(oracle.pyramid(inp[f"{name}/prev"]), oracle.pyramid(inp[f"{name}/next"]), tin,
                     mode=oracle.TEXTURE_WIDE)
    _agree(got, want, max(1, len(tin) // 100), 0.01, 1e-3)


def test_retrack_and_full_size(ctx, oracle):
    """The retrack pass (fe_track_mono) on a 1280x720 pair with 2000 features, against the oracle's
    two passes in the wide mode."""
    p, nx, _ = synthetic.frame_pair(41, 1280, 720)
    pp = ImagePyramid(1280, 720).build(ctx, torch.from_numpy(p).cuda())
    cp = ImagePyramid(1280, 720).build(ctx, torch.from_numpy(nx).cuda())
    xy = Selection(ctx).compute_gftt_and_select_features(pp, 0, 0, 0, 0, None, None, 2000).cpu().numpy()
    t = make_tracks(xy, None, 1280.0, 0.8)
    d = tracks_to_device(t)
    track_mono(ctx, pp, cp, d, 0.85, sampling=HW)
    got = tracks_from_device(d)
    want = oracle.lk_retrack(oracle.pyramid(p), oracle.pyramid(nx), t, 0.85, mode=oracle.TEXTURE_WIDE)
    _agree(got, want, len(t) // 100, 0.01, 1e-3)
    assert got["track_status"].sum() > len(t) // 4


def test_batched_equals_per_camera(ctx):
    shapes = [(640, 480), (1280, 720), (97, 61)]
    frames, hosts = [], []
    for i, (w, h) in enumerate(shapes):
        p, nx, _ = synthetic.frame_pair(i + 80, w, h)
        pp = ImagePyramid(w, h).build(ctx, torch.from_numpy(p).cuda())
        xy = Selection(ctx).compute_gftt_and_select_features(pp, 0, 0, 0, 0, None, None, 500).cpu().numpy()
        t = make_tracks(xy, None, float(w), 0.8)
        hosts.append(t)
        fin = TrackFinish(torch.ones(len(t), dtype=torch.int32, device="cuda"), 0.85)
        frames.append(CameraFrame(torch.from_numpy(nx).cuda(), ImagePyramid(w, h), pp, tracks_to_device(t), 300,
                                  (0, 0, 0, 0), finish=fin))
    b = Batch(ctx, frames, HW)
    b.run()
    torch.cuda.synchronize()
    batched = [(tracks_from_device(f.tracks), f.finish.age.cpu().numpy().copy(),
                f.new_xy[:int(f.new_count.item())].cpu().numpy().copy()) for f in frames]
    for f, t in zip(frames, hosts):
        f.tracks.copy_(tracks_to_device(t))
        f.finish.age.fill_(1)
    b.run_plain()
    torch.cuda.synchronize()
    for f, (tb, ab, nb) in zip(frames, batched):
        assert_tracks_equal(tracks_from_device(f.tracks), tb)
        np.testing.assert_array_equal(f.finish.age.cpu().numpy(), ab)
        np.testing.assert_array_equal(f.new_xy[:int(f.new_count.item())].cpu().numpy(), nb)
    b.close()


def test_edge_cases(ctx):
    rng = np.random.default_rng(11)
    img = rng.integers(0, 256, (120, 160), dtype=np.uint8)
    img[40:80, 40:80] = 128
    nxt = np.roll(img, (1, 2), (0, 1))
    xy = np.array([[0, 0], [159.9, 119.9], [-1, 5], [60, 60], [4.5, 4.5], [80, 20], [150, 100], [160, 50]], np.float32)
    t = make_tracks(xy, np.full_like(xy, 0.5), 160.0, 0.8)
    t["search_radius_px"][5] = -1.0
    t["ncc"] = 5.0
    pp, cp = gpu_pyramid(ctx, img), gpu_pyramid(ctx, nxt)
    got = _run(ctx, pp, cp, t)
    assert got["track_status"][2] == 0 and got["track_status"][5] == 0 and got["track_status"][7] == 0
    lost = got["track_status"] == 0
    np.testing.assert_array_equal(got["track"][lost], t["track"][lost])  # positions only written when tracked
    np.testing.assert_array_equal(got["ncc"], t["ncc"])
    assert _run(ctx, pp, cp, t[:0]).size == 0


def test_misaligned_planes_rejected(ctx):
    """Texture objects need plane addresses on the device's texture alignment."""
    h = w = 20
    buf = torch.zeros(8192, dtype=torch.float32, device="cuda")
    base = buf.data_ptr() + 16  # 16-byte aligned only
    desc = _lib.FePyramid()
    desc.levels = 1
    desc.width[0], desc.height[0], desc.pitch_bytes[0] = w, h, 80  # a multiple of 16 bytes, not of 32
    desc.image[0], desc.grad_x[0], desc.grad_y[0] = base, base + 8192, base + 16384
    d = tracks_to_device(make_tracks(np.array([[10, 10]], np.float32)))
    rc = ctx.lib.fe_track(ctx.handle, ctypes.byref(desc), ctypes.byref(desc), ctypes.c_void_p(d.data_ptr()), 1, 0,
                          HW, None)
    assert rc == _lib.FE_ERR_INVALID_ARGUMENT
