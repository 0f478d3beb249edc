"""Index arithmetic of the levels 0-2 tile kernel (pyramid.cu, namespace l012), restated on the CPU.

For each frame size, the tiles on the frame's edges and one interior tile are modelled (interior
tiles are translations of one another).  For each modelled tile the test checks that every
shared-memory read is inside its region (the uint8 tile, 163 x 176 bytes; the level-1 region,
79 rows of 80 floats; the level-2 region, 38 rows of 40 floats).  Every value that reaches an
output must also come from a cell that holds data:
  - for the uint8 tile, a pixel of the frame;
  - for the level-1 and level-2 regions, a cell that the strips or the corner fixes wrote.

The kernel runs for frames with at least three levels (level 2 at least 15 px, so the frame is at
least 57 px), where one reflection of `mirror_index` always lands inside the frame.  Everything
here is restated from the kernel's source; it checks bounds, not pixel values, which the GPU parity
tests compare with the oracle.

The generic stage kernel (pyramid_stage_kernel: FP32 sources, frames with fewer than three levels)
is restated the same way below: each level's staged region holds every tap of the levels and
gradients computed from it, mirrored taps included."""

import numpy as np
import pytest

from cuvslam_b200.types import level_sizes

T2, S0W, S0H, S1, S1S, S2, S2S = 32, 176, 163, 79, 80, 38, 40


def mirror(i, n):
    i = i if i >= 0 else -i - 1
    return i if i < n else 2 * n - i - 1


def tiles(w2, h2):
    tx, ty = -(-w2 // T2), -(-h2 // T2)
    xs = sorted({0, 1, tx // 2, tx - 2, tx - 1} & set(range(tx)))
    ys = sorted({0, 1, ty // 2, ty - 2, ty - 1} & set(range(ty)))
    return [(x * T2, y * T2) for y in ys for x in xs]


def check_tile(sizes, X2, Y2):
    (w0, h0), (w1, h1), (w2, h2) = sizes[:3]
    a0x, a0y = 4 * X2 - 32, 4 * Y2 - 19
    a1x, a1y = 2 * X2 - 8, 2 * Y2 - 8
    a2x, a2y = X2 - 4, Y2 - 3

    def b0(row, col):  # a read of the uint8 tile at tile coordinates whose value is used
        assert 0 <= row < S0H and 0 <= col < S0W, (row, col)
        assert 0 <= a0y + row < h0 and 0 <= a0x + col < w0, "read outside the frame"

    # level 1: column pairs (c, c + 1) over bands of 7 rows, 40 pairs x 12 bands; away from the edges
    # both columns' taps are bytes 4 pp + 14 .. 4 pp + 20 of the three words at 4 pp + 12
    done1 = np.zeros((S1, S1S), bool)
    for tid in range(40 * 12):
        pp, band = tid % 40, tid // 40
        c = 2 * pp
        x1 = a1x + c
        ys, ye = max(a1y + band * 7, 0), min(a1y + min(band * 7 + 7, S1), h1)
        if ys >= ye:
            continue
        if 2 * x1 - 2 >= 0 and 2 * x1 + 4 < w0 and c + 1 < S1 and 2 * ys - 2 >= 0 and 2 * ye < h0:
            assert 4 * pp + 12 + 12 <= S0W  # the three words of a row
            for r in range(2 * ys - 2, 2 * ye + 1):
                for col in range(4 * pp + 14, 4 * pp + 21):
                    b0(r - a0y, col)
            for y in range(ys, ye):
                done1[y - a1y, c] = done1[y - a1y, c + 1] = True
            continue
        for k in range(2):
            cc, xx = c + k, x1 + k
            if cc >= S1 or not (0 <= xx < w1):
                continue
            cols = [mirror(2 * xx - 2 + l, w0) - a0x for l in range(5)]
            for r in range(2 * ys - 2, 2 * (ye - 1) + 3):
                for col in cols:
                    b0(mirror(r, h0) - a0y, col)
            for y in range(ys, ye):
                done1[y - a1y, cc] = True
    for tid in range(4):  # corners redone with the 25-tap rule
        x1, y1 = (w1 - 1 if tid & 1 else 0), (h1 - 1 if tid & 2 else 0)
        if a1x <= x1 < a1x + S1 and a1y <= y1 < a1y + S1:
            for k in range(5):
                for l in range(5):
                    xc, yc = 2 * x1 - 2 + l, 2 * y1 - 2 + k
                    if (xc < 0 or xc >= w0) and (yc < 0 or yc >= h0):
                        continue
                    b0(mirror(yc, h0) - a0y, mirror(xc, w0) - a0x)
            done1[y1 - a1y, x1 - a1x] = True

    # level 2: column pairs over bands of 3 rows, 19 pairs x 13 bands; away from the edges both
    # columns' taps are the level-1 values 4 pp .. 4 pp + 6 of a row (two 16-byte loads)
    done2 = np.zeros((S2, S2S), bool)
    for tid in range(19 * 13):
        pp, band = tid % 19, tid // 19
        c = 2 * pp
        x2 = X2 - 3 + c
        ys, ye = max(a2y + band * 3, 0), min(a2y + min(band * 3 + 3, S2), h2)
        if ys >= ye:
            continue
        if 2 * x2 - 2 >= 0 and 2 * x2 + 4 < w1 and 2 * ys - 2 >= 0 and 2 * ye < h1:
            assert 4 * pp + 8 <= S1S  # the two 16-byte loads of a row
            for r in range(2 * ys - 2, 2 * ye + 1):
                rr = r - a1y
                for cc in range(4 * pp, 4 * pp + 7):
                    assert 0 <= rr < S1 and done1[rr, cc], (rr, cc)
            for y in range(ys, ye):
                assert x2 + 1 - a2x < S2S
                done2[y - a2y, x2 - a2x] = done2[y - a2y, x2 + 1 - a2x] = True
            continue
        for k in range(2):
            xx = x2 + k
            if not (0 <= xx < w2):
                continue
            cols = [mirror(2 * xx - 2 + l, w1) - a1x for l in range(5)]
            for r in range(2 * ys - 2, 2 * (ye - 1) + 3):
                rr = mirror(r, h1) - a1y
                for cc in cols:
                    assert 0 <= rr < S1 and 0 <= cc < S1S and done1[rr, cc], (rr, cc)
            for y in range(ys, ye):
                assert 0 <= xx - a2x < S2S
                done2[y - a2y, xx - a2x] = True

    def l2_taps(x, y, sw, sh, ax, ay, done, rows, stride):  # downscale_px on a region
        x0, y0 = 2 * x - 2, 2 * y - 2
        for k in range(5):
            for l in range(5):
                xc, yc = x0 + l, y0 + k
                if (xc < 0 or xc >= sw) and (yc < 0 or yc >= sh):
                    continue
                rr, cc = mirror(yc, sh) - ay, mirror(xc, sw) - ax
                assert 0 <= rr < rows and 0 <= cc < stride and done[rr, cc], (rr, cc)

    for tid in range(4):
        x2, y2 = (w2 - 1 if tid & 1 else 0), (h2 - 1 if tid & 2 else 0)
        if X2 - 3 <= x2 < X2 + 35 and a2y <= y2 < a2y + S2:
            l2_taps(x2, y2, w1, h1, a1x, a1y, done1, S1, S1S)
            done2[y2 - a2y, x2 - a2x] = True

    # level 3's image on the tile's 16x16 core (when the pyramid has a level 3)
    if len(sizes) > 3:
        w3, h3 = sizes[3]
        for tid in range(256):
            x3, y3 = (X2 >> 1) + (tid & 15), (Y2 >> 1) + (tid >> 4)
            if x3 < w3 and y3 < h3:
                l2_taps(x3, y3, w2, h2, a2x, a2y, done2, S2, S2S)

    # level-0 outputs.  (a) image and grad_y: a pixel pair's column over a strip of 16 rows, 64
    # pairs x 8 strips, its 7-row window sliding down (rows y0 - 3 .. y0 + 18 loaded)
    for tid in range(512):
        pc, strip = tid & 63, tid >> 6
        x, y0 = 4 * X2 + 2 * pc, 4 * Y2 + 16 * strip
        if x >= w0 or y0 >= h0:
            continue
        c = x - a0x
        assert 0 <= c and c + 1 < S0W
        for k in range(22):
            assert 0 <= y0 - a0y - 3 + k < S0H  # every 2-byte load
        two = x + 1 < w0
        for i in range(16):
            y = y0 + i
            if y >= h0:
                continue
            for px in ((0, 1) if two else (0,)):
                b0(y - a0y, c + px)  # the image value
                if 2 < y < h0 - 3:
                    for j in range(-3, 4):
                        b0(y - a0y + j, c + px)
    # (b) grad_x: four pixels of a row per item from the words at x - 4, x, x + 4
    for q in range(128 * 32):
        y, x = 4 * Y2 + (q >> 5), 4 * X2 + (q & 31) * 4
        if y >= h0 or x >= w0:
            continue
        r, c = y - a0y, x - a0x
        assert 0 <= r < S0H and c >= 4 and c + 8 <= S0W  # every word read
        for i in range(4):
            if x + i < w0 and 2 < x + i < w0 - 3:
                for j in range(-3, 4):
                    b0(r, c + i + j)

    # level-1 and level-2 outputs: four pixels per item
    for q in range(64 * 16 + 32 * 8):
        lev1 = q < 64 * 16
        qq = q if lev1 else q - 64 * 16
        qpr = 16 if lev1 else 8
        lw, lh = (w1, h1) if lev1 else (w2, h2)
        y = (2 * Y2 if lev1 else Y2) + qq // qpr
        x = (2 * X2 if lev1 else X2) + (qq % qpr) * 4
        if y >= lh or x >= lw:
            continue
        rows, stride, done = (S1, S1S, done1) if lev1 else (S2, S2S, done2)
        r, c = y - (a1y if lev1 else a2y), x - (a1x if lev1 else a2x)
        assert r >= 3 and r + 3 < rows and c >= 4 and c + 8 <= stride  # every 16-byte read

        def used(rr, cc):
            assert done[rr, cc], (lev1, rr, cc)

        for i in range(4):
            if x + i >= lw:
                continue
            used(r, c + i)
            if 2 < x + i < lw - 3:
                for j in range(-3, 4):
                    used(r, c + i + j)
            if 2 < y < lh - 3:
                for j in range(-3, 4):
                    used(r + j, c + i)


SIZES = [(57, 57), (58, 61), (63, 120), (97, 61), (130, 57), (640, 480), (752, 480), (1241, 376),
         (1280, 720), (1920, 1200), (2047, 1535), (4096, 4096)]


@pytest.mark.parametrize("w,h", SIZES)
def test_tile_reads_stay_inside_and_use_written_cells(w, h):
    sizes = level_sizes(w, h)
    assert len(sizes) >= 3
    (w2, h2) = sizes[2]
    for X2, Y2 in tiles(w2, h2):
        check_tile(sizes, X2, Y2)


def test_smallest_frame_of_the_kernel():
    assert len(level_sizes(57, 57)) >= 3 and len(level_sizes(56, 57)) == 2


# ---------------------------------------------------------------- generic stages
# pyramid_stage_kernel<InT, NL, KT>: a CTA owns a KT x KT core of the deepest produced level NL and
# stages, per level k, the region [a_k, a_k + S_k) in x (the same in y): a_NL = X - 3,
# a_k = 2 a_{k+1} - 2, S_NL = KT + 6, S_k = 2 S_{k+1} + 3.  Level 0 of the stage is its source.

def region_size(kt, nl, k):
    return kt + 6 if k == nl else 2 * region_size(kt, nl, k + 1) + 3


def check_stage(dims, nl, kt, write_level0, X, Y):
    a, ay = [0] * (nl + 1), [0] * (nl + 1)
    a[nl], ay[nl] = X - 3, Y - 3
    for k in range(nl - 1, -1, -1):
        a[k], ay[k] = 2 * a[k + 1] - 2, 2 * ay[k + 1] - 2
    S = [region_size(kt, nl, k) for k in range(nl + 1)]
    valid = []
    w, h = dims[0]
    rr, cc = np.meshgrid(np.arange(S[0]), np.arange(S[0]), indexing="ij")
    valid.append((a[0] + cc >= 0) & (ay[0] + rr >= 0) & (a[0] + cc < w) & (ay[0] + rr < h))
    for k in range(1, nl + 1):
        (sw, sh), (w, h) = dims[k - 1], dims[k]
        v = np.zeros((S[k], S[k]), bool)
        for r in range(S[k]):
            for c in range(S[k]):
                gx, gy = a[k] + c, ay[k] + r
                if not (0 <= gx < w and 0 <= gy < h):
                    continue
                x0, y0 = 2 * gx - 2, 2 * gy - 2
                for kk in range(5):
                    for l in range(5):
                        xc, yc = x0 + l, y0 + kk
                        if (xc < 0 or xc >= sw) and (yc < 0 or yc >= sh):
                            continue
                        r2, c2 = mirror(yc, sh) - ay[k - 1], mirror(xc, sw) - a[k - 1]
                        assert 0 <= r2 < S[k - 1] and 0 <= c2 < S[k - 1], (k, r2, c2)
                        assert valid[k - 1][r2, c2], (k, r2, c2)
                v[r, c] = True
        valid.append(v)
    for k in range(0 if write_level0 else 1, nl + 1):
        w, h = dims[k]
        C = kt << (nl - k)
        cx0, cy0 = X << (nl - k), Y << (nl - k)
        for r in range(C):
            for c in range(C):
                x, y = cx0 + c, cy0 + r
                if x >= w or y >= h:
                    continue
                pr, pc = y - ay[k], x - a[k]
                taps = [(pr, pc)]
                if 2 < x < w - 3:
                    taps += [(pr, pc + j) for j in range(-3, 4)]
                if 2 < y < h - 3:
                    taps += [(pr + j, pc) for j in range(-3, 4)]
                for tr, tc in taps:
                    assert 0 <= tr < S[k] and 0 <= tc < S[k] and valid[k][tr, tc], (k, tr, tc)


def halvings(w, h, n):
    dims = [(w, h)]
    for _ in range(n):
        w, h = (w + 1) // 2, (h + 1) // 2
        dims.append((w, h))
    return dims


STAGE_SOURCES = [(1, 1), (5, 7), (15, 15), (16, 29), (29, 29), (30, 31), (57, 57), (97, 61), (130, 57),
                 (640, 480), (1241, 376)]


@pytest.mark.parametrize("nl", [0, 1, 2])
@pytest.mark.parametrize("kt", [8, 16])
def test_stage_regions_hold_every_tap(nl, kt):
    for w, h in STAGE_SOURCES:
        dims = halvings(w, h, nl)
        if any(dw < 15 or dh < 15 for dw, dh in dims[1:]):
            continue  # the planner never produces a level below 15 px
        dw, dh = dims[nl]
        tx, ty = -(-dw // kt), -(-dh // kt)
        xs = sorted({0, 1, tx // 2, tx - 2, tx - 1} & set(range(tx)))
        ys = sorted({0, 1, ty // 2, ty - 2, ty - 1} & set(range(ty)))
        for ty_ in ys:
            for tx_ in xs:
                check_stage(dims, nl, kt, True, tx_ * kt, ty_ * kt)
