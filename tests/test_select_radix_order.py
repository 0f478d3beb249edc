"""The final selection order's radix sort (select.cu, final_radix_kernel), restated on the CPU.

Keys are (~strength bits) << 32 | cell, padded to S x 1024 slots with all-ones keys.  Each pass takes
a 4-bit digit (the cell bits of the low word, then the 32 bits of the high word); a warp's key of
slot s and lane l is ranked among the lanes of its warp with the same digit; the per-(digit, slot,
warp) counts are scanned in (digit, slot, warp) order; each key moves to its offset plus rank.  This
checks that the passes leave the real keys sorted ascending and the padding last, for camera sizes
whose cell count is and is not a power of 16."""

import numpy as np
import pytest


def radix_order(keys, n, slots, cells):
    src = np.full(slots * 1024, np.uint64(0xFFFFFFFFFFFFFFFF), np.uint64)
    src[:n] = keys
    cb = 0
    while (1 << cb) < cells:
        cb += 4
    shifts = list(range(0, cb, 4)) + list(range(32, 64, 4))
    idx = np.arange(slots * 1024)
    s_of, w_of, l_of = idx // 1024, (idx % 1024) // 32, idx % 32
    for sh in shifts:
        dig = ((src >> np.uint64(sh)) & np.uint64(15)).astype(np.int64)
        # rank among the lanes of the same warp (slot, warp) with the same digit
        group = (s_of * 32 + w_of) * 16 + dig
        rank = np.zeros_like(idx)
        counts = np.zeros(16 * slots * 32, np.int64)
        for g in np.unique(group):
            members = np.nonzero(group == g)[0]  # ascending lanes
            rank[members] = np.arange(len(members))
            d, sw = g % 16, g // 16
            counts[(d * slots + sw // 32) * 32 + sw % 32] = len(members)
        offsets = np.concatenate([[0], np.cumsum(counts)[:-1]])
        dst = np.empty_like(src)
        dst[offsets[(dig * slots + s_of) * 32 + w_of] + rank] = src
        src = dst
    return src


@pytest.mark.parametrize("n,cells", [(1, 4800), (300, 4800), (1024, 14400), (2500, 36000), (4096, 65536), (3000, 36001)])
def test_radix_passes_sort_the_kept_keys(n, cells):
    rng = np.random.default_rng(n + cells)
    strength = rng.uniform(0.0101, 4.0, n).astype(np.float32)
    strength[: n // 5] = strength[0]  # ties in strength, broken by the cell index
    cell = rng.permutation(cells)[:n].astype(np.uint64)
    keys = ((~strength.view(np.uint32)).astype(np.uint64) << np.uint64(32)) | cell
    slots = max(1, (n + 1023) // 1024)
    out = radix_order(keys, n, slots, cells)
    np.testing.assert_array_equal(out[:n], np.sort(keys))
    assert (out[n:] == np.uint64(0xFFFFFFFFFFFFFFFF)).all()
