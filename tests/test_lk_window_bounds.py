"""Window bounds of the LK tracker's bilinear taps (lk_track.cuh, lk_common.cuh), restated on the CPU
in FP32 (numpy's float32 operations round to nearest even, as __fadd_rn / __fsub_rn do).

A 9x9 patch whose first sample is at xmin takes, for column i, the texels floor(fl(fl(xmin + i) -
0.5)) and +1 (the same in y).  The 12-texel span of the previous-frame patch starts at
bx = floor(fl(xmin - 0.5)) - 1; its window is staged from the aligned column ax = bx rounded down to
a multiple of 4, 16 texels wide.  The current-frame window is restaged, 20 texels wide from the
aligned column (nbx - 2) rounded down to a multiple of 4, whenever the 12-texel span would leave it.
Rounding may move a column's texel by one against base + i, so the 12-texel span leaves one texel on
each side.  This test checks that every tap lies inside its window for coordinates from 0 to
65536 px."""

import numpy as np

F = np.float32
PW = 12           # the patch's texel span
PA, CA = 16, 20   # staged widths of the previous and current windows


def texel_range(xmin):
    """First and last texel that the nine columns of a patch starting at xmin read."""
    i = np.arange(9, dtype=F)
    p = (F(xmin) + i).astype(F)
    base = np.floor((p - F(0.5)).astype(F)).astype(np.int64)
    return int(base.min()), int(base.max()) + 1


def window_origin(xmin):
    return int(np.floor(F(F(xmin) - F(0.5)))) - 1


def samples(rng):
    vals = list(rng.uniform(0, 4096, 20000).astype(F)) + list(rng.uniform(4096, 65536, 5000).astype(F))
    for k in list(range(0, 64)) + list(range(4000, 4096)) + list(rng.integers(0, 65536, 400)):
        for frac in (0.0, 0.5):
            c = F(k + frac)
            vals += [c, np.nextafter(c, F(-1)), np.nextafter(c, F(1e9))]
    return [v for v in vals if v >= 0]


def test_previous_window_holds_every_tap():
    rng = np.random.default_rng(3)
    for xmin in samples(rng):
        bx = window_origin(xmin)
        ax = bx & ~3
        lo, hi = texel_range(xmin)
        assert bx <= lo and hi < bx + PW, (float(xmin), bx, lo, hi)
        assert ax % 4 == 0 and ax <= lo and hi < ax + PA, (float(xmin), ax, lo, hi)


def test_current_window_rule_holds_every_tap():
    """A walk of iterates (steps below the search radius): the window is restaged only when the
    12-texel span leaves it, and every tap stays inside the 20 staged texels."""
    rng = np.random.default_rng(4)
    for start in rng.uniform(8, 4088, 2000).astype(F):
        wbx = None
        x = F(start)
        for _ in range(12):
            nbx = window_origin(x)
            if wbx is None or nbx < wbx or nbx + PW > wbx + CA:
                wbx = (nbx - 2) & ~3
            lo, hi = texel_range(x)
            assert wbx % 4 == 0 and wbx <= lo and hi < wbx + CA, (float(x), wbx, lo, hi)
            x = F(x + F(rng.normal(0, 1.5)))
            if not (0 <= x < 4090):
                break
