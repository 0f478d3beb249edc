"""MonoSOFGPU's retrack pass and finish filters on the device: fe_track_mono and fe_finish_tracks
bit-identical to the oracle's restatement, and the batched frame step with the filters between LK
and selection equal to the plain per-camera sequence."""

import numpy as np
import pytest
import torch

from conftest import assert_tracks_equal, gpu_pyramid
from cuvslam_b200 import _lib, synthetic
from cuvslam_b200.frontend import (Batch, CameraFrame, ImagePyramid, Selection, TrackFinish, finish_tracks,
                                   track_mono, tracks_from_device, tracks_to_device)
from cuvslam_b200.types import make_tracks

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["c1", "half", "odd"])
def test_retrack_matches_oracle(ctx, oracle, golden, name):
    inp, ref = golden
    tin = ref[f"{name}/lk_pred/in"]
    pp, cp = gpu_pyramid(ctx, inp[f"{name}/prev"]), gpu_pyramid(ctx, inp[f"{name}/next"])
    d = tracks_to_device(tin)
    track_mono(ctx, pp, cp, d, 0.85, sampling=_lib.FE_SAMPLE_TEXTURE)
    got = tracks_from_device(d)
    want = oracle.lk_retrack(oracle.pyramid(inp[f"{name}/prev"]), oracle.pyramid(inp[f"{name}/next"]), tin, 0.85)
    assert_tracks_equal(got, want)
    # the retrack pass can only add tracks to the first pass's
    first = oracle.lk(oracle.pyramid(inp[f"{name}/prev"]), oracle.pyramid(inp[f"{name}/next"]), tin)
    assert np.all(got["track_status"] >= first["track_status"])


def _finish_case(seed, n, w, h, clustered=True):
    rng = np.random.default_rng(seed)
    xy = np.stack([rng.uniform(-3, w + 3, n), rng.uniform(-3, h + 3, n)], 1).astype(np.float32)
    if clustered:  # many tracks in few 3x3 cells, to exercise collapse's age and index rules
        k = n // 3
        xy[:k] = (np.floor(xy[:k] / 3) * 3 + rng.uniform(0, 2.9, (k, 2))).astype(np.float32)
        xy[k:2 * k] = xy[:k] + rng.uniform(-1, 1, (k, 2)).astype(np.float32)
    t = make_tracks(xy, None, float(w), 0.8)
    t["track_status"] = (rng.uniform(size=n) < 0.85).astype(np.uint8)
    age = rng.integers(0, 6, n).astype(np.uint32)
    pred = (xy + rng.normal(0, 2.0, xy.shape) * rng.choice([1.0, 4.0], (n, 1))).astype(np.float32)
    pred[rng.uniform(size=n) < 0.2] = np.nan
    mask = (rng.uniform(size=(h, w)) < 0.02).astype(np.uint8)
    return t, age, pred, mask


@pytest.mark.parametrize("opts", [dict(), dict(pred=True), dict(mask=True), dict(pred=True, mask=True, border=(3, 4, 5, 6)),
                                  dict(collapse=False, pred=True), dict(border=(0, 0, 2000, 0))])
def test_finish_matches_oracle(ctx, oracle, opts):
    w, h, n = 640, 480, 3000
    t, age, pred, mask = _finish_case(17 + len(opts), n, w, h)
    border = opts.get("border", (0, 0, 0, 0))
    collapse = opts.get("collapse", True)
    d = tracks_to_device(t)
    age_d = torch.from_numpy(age.astype(np.int32)).cuda()
    fin = TrackFinish(age_d, predicted=torch.from_numpy(pred).cuda() if opts.get("pred") else None,
                      mask=torch.from_numpy(mask).cuda() if opts.get("mask") else None, collapse=collapse)
    finish_tracks(ctx, d, fin, w, h, border)
    torch.cuda.synchronize()
    want, wage, walive = oracle.finish_tracks(t, age, w, h, border, pred if opts.get("pred") else None,
                                              mask if opts.get("mask") else None, collapse)
    assert_tracks_equal(tracks_from_device(d), want)
    np.testing.assert_array_equal(age_d.cpu().numpy().astype(np.uint32), wage)
    assert int(fin.alive_count.item()) == walive
    # the collapse cells are cleared: a second identical call gives the same result
    d2 = tracks_to_device(t)
    age2 = torch.from_numpy(age.astype(np.int32)).cuda()
    fin2 = TrackFinish(age2, predicted=fin.predicted, mask=fin.mask, collapse=collapse)
    finish_tracks(ctx, d2, fin2, w, h, border)
    torch.cuda.synchronize()
    assert_tracks_equal(tracks_from_device(d2), want)


def test_batched_step_with_finish_equals_plain_and_oracle(ctx, oracle):
    shapes = [(640, 480), (1280, 720), (97, 61)]
    frames, hosts, ages, prevs, nexts = [], [], [], [], []
    for i, (w, h) in enumerate(shapes):
        p, nx, _ = synthetic.frame_pair(i + 70, w, h)
        pp = ImagePyramid(w, h).build(ctx, torch.from_numpy(p).cuda())
        xy = Selection(ctx).compute_gftt_and_select_features(pp, 0, 0, 0, 0, None, None, 400).cpu().numpy()
        t = make_tracks(xy, None, float(w), 0.8)
        age = np.random.default_rng(i).integers(1, 9, len(t)).astype(np.uint32)
        hosts.append(t)
        ages.append(age)
        prevs.append(p)
        nexts.append(nx)
        fin = TrackFinish(torch.from_numpy(age.astype(np.int32)).cuda(), 0.85)
        frames.append(CameraFrame(torch.from_numpy(nx).cuda(), ImagePyramid(w, h), pp, tracks_to_device(t), 450,
                                  (2, 2, 2, 2), finish=fin))
    b = Batch(ctx, frames, _lib.FE_SAMPLE_TEXTURE)  # compared with the oracle bit for bit
    b.run()
    torch.cuda.synchronize()
    batched = [(tracks_from_device(f.tracks), f.finish.age.cpu().numpy().copy(),
                f.new_xy[:int(f.new_count.item())].cpu().numpy().copy()) for f in frames]
    for f, t, a in zip(frames, hosts, ages):
        f.tracks.copy_(tracks_to_device(t))
        f.finish.age.copy_(torch.from_numpy(a.astype(np.int32)))
    b.run_plain()
    torch.cuda.synchronize()
    for f, (tb, ab, nb), t, a, p, nx, (w, h) in zip(frames, batched, hosts, ages, prevs, nexts, shapes):
        assert_tracks_equal(tracks_from_device(f.tracks), tb)
        np.testing.assert_array_equal(f.finish.age.cpu().numpy(), ab)
        np.testing.assert_array_equal(f.new_xy[:int(f.new_count.item())].cpu().numpy(), nb)
        lk = oracle.lk_retrack(oracle.pyramid(p), oracle.pyramid(nx), t, 0.85)
        want, wage, _ = oracle.finish_tracks(lk, a, w, h, (2, 2, 2, 2))
        assert_tracks_equal(tb, want)
        np.testing.assert_array_equal(ab.astype(np.uint32), wage)


def test_finish_known_answers(ctx):
    """The CUDA filters on the hand-computed known answers of each rule (tests/finish_cases.py)."""
    import finish_cases as FC

    for name, (xy, st, age, w, h, border, pred, mask, collapse, want) in FC.cases().items():
        t = FC.tracks_of(xy, st)
        d = tracks_to_device(t)
        age_d = torch.from_numpy(np.asarray(age, np.int32)).cuda()
        fin = TrackFinish(age_d, predicted=None if pred is None else torch.from_numpy(np.asarray(pred, np.float32)).cuda(),
                          mask=None if mask is None else torch.from_numpy(mask).cuda(), collapse=collapse)
        finish_tracks(ctx, d, fin, w, h, border)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(age_d.cpu().numpy().astype(np.uint32), np.asarray(want, np.uint32), err_msg=name)
        got = tracks_from_device(d)
        np.testing.assert_array_equal(got["track_status"] != 0, np.asarray(want) != 0, err_msg=name)


def test_finish_scratch_survives_stereo_scratch_growth(oracle):
    """One context's scratch buffers are independent: growing the left-to-right matching scratch
    (twice) leaves the finish filters' collapse cells allocated and correct, and no CUDA error is
    left pending for the next call to report."""
    import os

    from conftest import ROOT
    from cuvslam_b200.frontend import Context
    from cuvslam_b200.stereo import StereoMatcher, StereoPair

    c = Context(0)
    try:
        w, h, n = 640, 480, 3000
        t, age, pred, mask = _finish_case(29, n, w, h)
        want, wage, _ = oracle.finish_tracks(t, age, w, h, (0, 0, 0, 0), None, None, True)

        def finish_once():
            d = tracks_to_device(t)
            a = torch.from_numpy(age.astype(np.int32)).cuda()
            finish_tracks(c, d, TrackFinish(a), w, h, (0, 0, 0, 0))
            torch.cuda.synchronize()
            assert_tracks_equal(tracks_from_device(d), want)
            np.testing.assert_array_equal(a.cpu().numpy().astype(np.uint32), wage)

        finish_once()
        inp = np.load(os.path.join(ROOT, "tests", "golden", "stereo_inputs.npz"))
        left = np.load(os.path.join(ROOT, "tests", "golden", "inputs.npz"))["c1/prev"]
        pp, sp = gpu_pyramid(c, left, 4), gpu_pyramid(c, inp["right"], 4)
        uv = torch.from_numpy(inp["uv"]).cuda()
        for k in (40, 400):  # a larger candidate list each time: the scratch grows twice
            off = torch.from_numpy((np.arange(len(inp["uv"]) + 1) * 2).astype(np.int32)).cuda()
            xy = torch.from_numpy(np.repeat(inp["uv"], 2, axis=0) - np.float32(k / 40)).cuda()
            m = StereoMatcher(c)
            m.track_primary_to_secondary([StereoPair(pp, sp, uv, None, cand_offsets=off, cand_xy=xy,
                                                     max_candidates=2 * k // 40)])
            torch.cuda.synchronize()
        finish_once()
    finally:
        c.close()
