"""The per-cell argmax of the response tiles (select.cu, phase E) against the reference's warp rule
(downsample_gftt_x8_kernel, selection_v2.cu:107-178), as step-for-step models of both reductions on
tie-heavy 8x8 cells.

Reference: lane l holds pixels l and l + 32 (the second replaces the first only when strictly
greater, starting from 0), then a shfl_down tree over d = 1, 2, 4, 8, 16 in which lane i takes lane
i + d's pair only when strictly greater (lanes past 31 return their own value).
select.cu: eight threads per cell, thread g scanning lanes 4g .. 4g+3 in (lane, element) order with
the same strict rule, then a shfl_down merge over d = 1, 2, 4 within the eight threads.
Both must give the same (value, pixel) for every cell, ties included."""

import numpy as np


def _shfl_down_tree(vals, idxs, width, steps):
    vals, idxs = list(vals), list(idxs)
    for d in steps:
        nv, ni = vals[:], idxs[:]
        for i in range(len(vals)):
            src = i + d
            if (i % width) + d < width:  # source inside the segment, else the lane keeps its own
                if vals[src] > vals[i]:
                    nv[i], ni[i] = vals[src], idxs[src]
        vals, idxs = nv, ni
    return vals[0], idxs[0]


def reference_cell(cell):
    flat = cell.reshape(64)
    m, idx = [0.0] * 32, [0] * 32
    for lane in range(32):
        for e in range(2):
            f = lane + 32 * e
            if flat[f] > m[lane]:
                m[lane], idx[lane] = flat[f], f
    return _shfl_down_tree(m, idx, 32, (1, 2, 4, 8, 16))


def tile_cell(cell):
    flat = cell.reshape(64)
    m, idx = [0.0] * 8, [0] * 8
    for g in range(8):
        for k in range(8):
            f = 4 * g + (k >> 1) + 32 * (k & 1)
            if flat[f] > m[g]:
                m[g], idx[g] = flat[f], f
    return _shfl_down_tree(m, idx, 8, (1, 2, 4))


def test_same_pixel_on_tie_heavy_cells():
    rng = np.random.default_rng(5)
    for trial in range(3000):
        levels = rng.integers(1, 5)
        cell = rng.integers(0, levels + 1, size=(8, 8)).astype(np.float32) * np.float32(0.25)
        if trial % 3 == 0:
            cell[rng.random((8, 8)) < 0.7] = 0.0  # NMS leaves mostly zeros
        assert tile_cell(cell) == reference_cell(cell), cell


def test_all_zero_and_single_maximum():
    z = np.zeros((8, 8), np.float32)
    assert tile_cell(z) == reference_cell(z) == (0.0, 0)
    for f in range(64):
        c = np.zeros(64, np.float32)
        c[f] = 1.0
        assert tile_cell(c.reshape(8, 8)) == reference_cell(c.reshape(8, 8)) == (1.0, f)


def test_first_maximum_in_lane_order():
    # maxima at pixels 35 (lane 3, second element) and 5 (lane 5): the lower lane wins
    c = np.zeros(64, np.float32)
    c[35] = c[5] = 2.0
    assert reference_cell(c.reshape(8, 8)) == tile_cell(c.reshape(8, 8)) == (2.0, 35)
