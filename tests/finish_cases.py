"""Hand-computed known answers of MonoSOFGPU::finish's filters, one rule per case, written from the
reference's scalar code (the numbers below are worked out by hand from those rules, not produced by
any implementation):
  collect + IncrementTracksAge   sof_mono_gpu.cpp:80-104, sof_mono_base.cpp:111-118
  filterByPredictionError        sof_mono_base.cpp:40-92: with >= 3 alive predicted tracks, the
                                 median distance m (nth_element at size/2) sets max(3, 2 m); farther
                                 tracks die
  KillTracksOnBorder             selector_stereo.cpp:109-125: alive iff left <= x <= w-1-right and
                                 top <= y <= h-1-bottom (sizes unsigned)
  KillTracksWithinMask           sof_mono_base.cpp:121-133: mask(int y, int x) != 0 kills
  collapseTracks                 sof_mono_gpu.cpp:249-280: per 3x3 cell (position / 3 truncated) the
                                 first track with the cell's largest age survives
Each case: (xy, status, age_in, w, h, border, pred, mask, collapse, expected ages out)."""

import numpy as np

NAN = np.nan


def cases():
    out = {}
    # collect + age: a dead track stays dead; an alive tracked one ages; an alive lost one dies
    out["age"] = (
        [[10, 10], [20, 20], [30, 30], [40, 40]], [1, 1, 0, 0], [3, 0, 5, 0], 64, 64, (0, 0, 0, 0), None, None,
        False, [4, 0, 0, 0])
    # prediction filter: distances 1, 2, 10, 0.5, 2.5 (alive, predicted) -> sorted 0.5 1 2 2.5 10, the
    # element at 5 // 2 = 2 is 2 -> threshold max(3, 4) = 4: only the 10 px track dies.  The track
    # without a prediction (NaN) is not counted and survives.
    out["median"] = (
        [[10, 10], [20, 10], [30, 10], [40, 10], [50, 10], [60, 10]], [1] * 6, [1] * 6, 80, 40, (0, 0, 0, 0),
        [[11, 10], [20, 12], [30, 20], [40.5, 10], [50, 12.5], [NAN, NAN]], None, False, [2, 2, 0, 2, 2, 2])
    # prediction filter with small errors: distances 0.1 0.2 3.5 -> median 0.2 -> threshold max(3, 0.4)
    # = 3: the 3.5 px track dies (the floor of 3 px applies)
    out["median_floor"] = (
        [[10, 10], [20, 10], [30, 10]], [1] * 3, [1] * 3, 64, 32, (0, 0, 0, 0), [[10.1, 10], [20, 10.2], [33.5, 10]],
        None, False, [2, 2, 0])
    # fewer than 3 predicted alive tracks: no prediction filtering at all
    out["median_few"] = (
        [[10, 10], [20, 10], [30, 10]], [1, 1, 0], [1, 1, 1], 64, 32, (0, 0, 0, 0), [[10, 10], [40, 40], [30, 10]],
        None, False, [2, 2, 0])
    # border (top 2, bottom 3, left 4, right 5) on 40x30: alive iff 4 <= x <= 34 and 2 <= y <= 26
    out["border"] = (
        [[4, 2], [34, 26], [3.99, 10], [34.01, 10], [10, 1.99], [10, 26.01], [20, 15]], [1] * 7, [1] * 7, 40, 30,
        (2, 3, 4, 5), None, None, False, [2, 2, 0, 0, 0, 0, 2])
    # mask: pixel (int x, int y) = (7, 5) is masked: (7.9, 5.9) dies, (8.0, 5.0) lives
    m = np.zeros((16, 16), np.uint8)
    m[5, 7] = 1
    out["mask"] = ([[7.9, 5.9], [8.0, 5.0], [7.0, 4.99]], [1] * 3, [1] * 3, 16, 16, (0, 0, 0, 0), None, m, False,
                   [0, 2, 2])
    # collapse: cell (3, 3) holds tracks aged 2, 5, 5 (after ageing 3, 6, 6): the first of the two
    # oldest survives; (11.9, 9) is in the same cell (11.9 / 3 = 3.97); (12, 9) is in cell (4, 3)
    out["collapse"] = (
        [[9.5, 9.5], [10, 11], [11.9, 9], [12, 9]], [1] * 4, [2, 5, 5, 1], 32, 32, (0, 0, 0, 0), None, None, True,
        [0, 6, 0, 2])
    return out


def tracks_of(xy, status):
    from cuvslam_b200.types import make_tracks

    t = make_tracks(np.asarray(xy, np.float32))
    t["track_status"] = np.asarray(status, np.uint8)
    return t
