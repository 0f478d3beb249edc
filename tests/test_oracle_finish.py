"""CPU checks of the oracle's finish filters against a plain-Python restatement of the reference's
host loops (MonoSOFGPU::collect and finish, sof_mono_gpu.cpp:80-104,144-170,249-280;
MonoSOFBase::filterByPredictionError / IncrementTracksAge / KillTracksWithinMask,
sof_mono_base.cpp:51-133; KillTracksOnBorder, selector_stereo.cpp:109-125)."""

import numpy as np
import pytest

from cuvslam_b200.types import make_tracks


def _reference_loops(tracks, age, w, h, border, pred, mask, collapse):
    """The reference's loops over a Python list of tracks, step by step."""
    f32 = np.float32
    n = len(tracks)
    age = [int(a) for a in age]
    pos = [(f32(x), f32(y)) for x, y in tracks["track"]]
    for k in range(n):  # collect + IncrementTracksAge
        if age[k]:
            age[k] = age[k] + 1 if tracks["track_status"][k] else 0
    if pred is not None:
        deltas = []
        for k in range(n):
            if age[k] and not np.isnan(pred[k][0]):
                dx, dy = f32(pred[k][0]) - pos[k][0], f32(pred[k][1]) - pos[k][1]
                deltas.append(f32(np.sqrt(f32(f32(dx * dx) + f32(dy * dy)))))
        if len(deltas) >= 3:
            thr = max(f32(3), f32(2) * sorted(deltas)[len(deltas) // 2])
            it = iter(deltas)
            for k in range(n):
                if age[k] and not np.isnan(pred[k][0]):
                    if next(it) > thr:
                        age[k] = 0
    top, bottom, left, right = border
    xr = f32((w - 1 - right) % 2**64)
    yb = f32((h - 1 - bottom) % 2**64)
    for k in range(n):
        if age[k]:
            x, y = pos[k]
            if not (f32(left) <= x <= xr and f32(top) <= y <= yb):
                age[k] = 0
    if mask is not None:
        for k in range(n):
            if age[k]:
                x, y = pos[k]
                if mask[int(y), int(x)]:
                    age[k] = 0
    if collapse:
        cells = {}
        for k in range(n):
            if age[k]:
                c = (int(pos[k][0] / f32(3)), int(pos[k][1] / f32(3)))
                cells[c] = max(cells.get(c, 0), age[k])
        for k in range(n):
            if age[k]:
                c = (int(pos[k][0] / f32(3)), int(pos[k][1] / f32(3)))
                if age[k] == cells[c]:
                    cells[c] = 0
                else:
                    age[k] = 0
    return np.array(age, np.uint32)


@pytest.mark.parametrize("seed", [1, 2, 3])
@pytest.mark.parametrize("opts", [dict(), dict(pred=True), dict(mask=True, border=(3, 4, 5, 6)), dict(collapse=False)])
def test_oracle_finish_equals_reference_loops(oracle, seed, opts):
    rng = np.random.default_rng(seed)
    w, h, n = 160, 120, 900
    xy = np.stack([rng.uniform(-2, w + 2, n), rng.uniform(-2, h + 2, n)], 1).astype(np.float32)
    xy[: n // 2] = (np.floor(xy[: n // 2] / 3) * 3 + 1).astype(np.float32)  # crowded cells
    t = make_tracks(xy)
    t["track_status"] = (rng.uniform(size=n) < 0.8).astype(np.uint8)
    age = rng.integers(0, 5, n).astype(np.uint32)
    pred = (xy + rng.normal(0, 3, xy.shape)).astype(np.float32) if opts.get("pred") else None
    if pred is not None:
        pred[rng.uniform(size=n) < 0.3] = np.nan
    mask = (rng.uniform(size=(h, w)) < 0.05).astype(np.uint8) if opts.get("mask") else None
    border = opts.get("border", (0, 0, 0, 0))
    collapse = opts.get("collapse", True)
    got, gage, alive = oracle.finish_tracks(t, age, w, h, border, pred, mask, collapse)
    want = _reference_loops(t, age, w, h, border, pred, mask, collapse)
    np.testing.assert_array_equal(gage, want)
    np.testing.assert_array_equal(got["track_status"], ((want != 0) & (t["track_status"] != 0)).astype(np.uint8))
    assert alive == int((want != 0).sum())


def test_oracle_finish_known_answers(oracle):
    """Hand-computed known answers of each filter rule (tests/finish_cases.py)."""
    import finish_cases as FC

    for name, (xy, st, age, w, h, border, pred, mask, collapse, want) in FC.cases().items():
        t = FC.tracks_of(xy, st)
        p = None if pred is None else np.asarray(pred, np.float32)
        _, gage, alive = oracle.finish_tracks(t, np.asarray(age, np.uint32), w, h, border, p, mask, collapse)
        np.testing.assert_array_equal(gage, np.asarray(want, np.uint32), err_msg=name)
        assert alive == int((np.asarray(want) != 0).sum()), name
