"""The batched frame step (one graph over all cameras) equals the plain per-camera sequence and the
single-camera entry points, camera by camera, bit for bit."""

import numpy as np
import pytest
import torch

from conftest import assert_tracks_equal
from cuvslam_b200 import _lib, synthetic
from cuvslam_b200.frontend import (Batch, CameraFrame, ImagePyramid, LKFeatureTracker, Selection, tracks_from_device,
                                   tracks_to_device)
from cuvslam_b200.types import make_tracks

pytestmark = pytest.mark.gpu

SHAPES = [(640, 480), (97, 61), (1280, 720), (31, 17), (752, 480)]


def _setup(ctx, shapes, seed=0):
    frames, prevs, host = [], [], []
    rng = np.random.default_rng(seed)
    for i, (w, h) in enumerate(shapes):
        p, n, _ = synthetic.frame_pair(i + 50, w, h)
        pp = ImagePyramid(w, h).build(ctx, torch.from_numpy(p).cuda())
        budget = int(rng.integers(50, 600))
        xy = Selection(ctx).compute_gftt_and_select_features(pp, 0, 0, 0, 0, None, None, budget).cpu().numpy()
        t = make_tracks(xy, None, float(w), 0.8)
        host.append(t)
        prevs.append(pp)
        frames.append(CameraFrame(torch.from_numpy(n).cuda(), ImagePyramid(w, h), pp,
                                  tracks_to_device(t) if len(t) else None, budget, (1, 2, 3, 4)))
    return frames, prevs, host


def _results(frames):
    torch.cuda.synchronize()
    out = []
    for f in frames:
        tr = tracks_from_device(f.tracks) if f.tracks is not None else None
        n = int(f.new_count.item())
        out.append((tr, f.new_xy[:n].cpu().numpy().copy(), [x.copy() for lv in f.cur.to_numpy() for x in lv]))
    return out


def test_batched_equals_plain_and_single(ctx):
    frames, prevs, host = _setup(ctx, SHAPES)
    b = Batch(ctx, frames)
    assert b.kernel_count() > 0
    b.run()
    got_batch = _results(frames)
    for f, t in zip(frames, host):
        if f.tracks is not None:
            f.tracks.copy_(tracks_to_device(t))
    b.run_plain()
    got_plain = _results(frames)
    for (ta, na, pa), (tb, nb, pb) in zip(got_batch, got_plain):
        if ta is not None:
            assert_tracks_equal(ta, tb)
        np.testing.assert_array_equal(na, nb)
        for x, y in zip(pa, pb):
            np.testing.assert_array_equal(x, y)
    # single-camera entry points
    for f, t, (ta, na, pa) in zip(frames, host, got_batch):
        cur = ImagePyramid(f.cur.width, f.cur.height).build(ctx, f.image)
        for x, y in zip([x for lv in cur.to_numpy() for x in lv], pa):
            np.testing.assert_array_equal(x, y)
        if f.tracks is not None:
            d = tracks_to_device(t)
            LKFeatureTracker(ctx).track_points(f.prev, cur, d)
            torch.cuda.synchronize()
            assert_tracks_equal(tracks_from_device(d), ta)


def test_batch_graph_relaunch_is_deterministic(ctx):
    frames, _, host = _setup(ctx, SHAPES[:3], seed=3)
    b = Batch(ctx, frames)
    runs = []
    for _ in range(3):
        for f, t in zip(frames, host):
            f.tracks.copy_(tracks_to_device(t))
        b.run()
        runs.append(_results(frames))
    for r in runs[1:]:
        for (ta, na, _), (tb, nb, _) in zip(runs[0], r):
            assert_tracks_equal(ta, tb)
            np.testing.assert_array_equal(na, nb)


def test_new_features_respect_budget_and_borders(ctx):
    frames, _, host = _setup(ctx, SHAPES[:3], seed=5)
    b = Batch(ctx, frames)
    b.run()
    torch.cuda.synchronize()
    for f in frames:
        alive = int((tracks_from_device(f.tracks)["track_status"] == 1).sum())
        n = int(f.new_count.item())
        assert n <= max(f.num_desired - alive, 0)
        xy = f.new_xy[:n].cpu().numpy()
        w, h = f.cur.width, f.cur.height
        if n:
            assert xy[:, 0].min() >= 3 and xy[:, 0].max() <= w - 1 - 4
            assert xy[:, 1].min() >= 1 and xy[:, 1].max() <= h - 1 - 2


def test_autotuned_batch_gives_the_same_results(ctx):
    """Every shape the autotuner can pick computes the same step: results after fe_batch_autotune
    equal the default shapes' bit for bit, and the tracks are restored by the tuner."""
    frames, prevs, host = _setup(ctx, SHAPES, seed=3)
    b = Batch(ctx, frames)
    b.run()
    ref = _results(frames)
    for f, t in zip(frames, host):
        if f.tracks is not None:
            f.tracks.copy_(tracks_to_device(t))
    torch.cuda.synchronize()
    tuned = b.autotune(reps=2)
    assert tuned["lk_block"] in ("8x4", "8x3", "4x8", "12x2") and tuned["stage_tile"] in (8, 16)
    assert tuned["response_overlap"] in Batch.OVERLAP and tuned["l012_ctas_per_sm"] in (2, 3)
    for f, t in zip(frames, host):  # restored by the tuner
        if f.tracks is not None:
            assert_tracks_equal(tracks_from_device(f.tracks), t)
    b.run()
    got = _results(frames)
    for (ta, na, pa), (tb, nb, pb) in zip(ref, got):
        if ta is not None:
            assert_tracks_equal(ta, tb)
        np.testing.assert_array_equal(na, nb)
        for x, y in zip(pa, pb):
            np.testing.assert_array_equal(x, y)
    # every combination of shapes, set directly
    for block in ("8x4", "8x3", "4x8", "12x2"):
        for overlap in Batch.OVERLAP:
            for tile, ctas in ((8, 2), (16, 3)):
                b.set_tuning(block, overlap, tile, ctas)
                for f, t in zip(frames, host):
                    if f.tracks is not None:
                        f.tracks.copy_(tracks_to_device(t))
                b.run()
                for (ta, na, pa), (tb, nb, pb) in zip(ref, _results(frames)):
                    if ta is not None:
                        assert_tracks_equal(ta, tb)
                    np.testing.assert_array_equal(na, nb)
                    for x, y in zip(pa, pb):
                        np.testing.assert_array_equal(x, y)


@pytest.mark.parametrize("sampling", ["texture", "hardware"])
def test_lk_work_counters(ctx, sampling):
    """The kernel's work counters (fe_batch_lk_work) change no result, repeat exactly from the same
    inputs, and bound the work: every kept track was set up, stepped and NCC-checked at least at level
    0, and no level takes more than the 11 steps of the reference rule.  Both LK kernels (the
    texture-weight emulation and the texture unit) count."""
    frames, prevs, host = _setup(ctx, SHAPES[:3], seed=3)
    b = Batch(ctx, frames, _lib.FE_SAMPLE_TEXTURE if sampling == "texture" else _lib.FE_SAMPLE_HARDWARE)

    def restore():
        for f, t in zip(frames, host):
            if f.tracks is not None:
                f.tracks.copy_(tracks_to_device(t))

    restore()
    b.run_part(0)
    b.run_part(1)
    plain = [tracks_from_device(f.tracks) for f in frames if f.tracks is not None]
    restore()
    c1 = b.lk_work()
    counted = [tracks_from_device(f.tracks) for f in frames if f.tracks is not None]
    for x, y in zip(plain, counted):
        assert_tracks_equal(x, y)
    restore()
    assert b.lk_work() == c1
    levels, steps, ncc = c1
    kept = sum(int((t["track_status"] != 0).sum()) for t in counted)
    assert kept > 0 and levels >= kept and steps >= kept and ncc >= kept
    assert steps <= 11 * levels
    b.close()
