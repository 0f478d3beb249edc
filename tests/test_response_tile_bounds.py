"""Shared-memory indices of the response tile kernel (select.cu, tile_kernel), restated on the CPU.

One CTA per 64x32 tile.  Regions, in floats:
  - three planes of horizontal sums, 40 rows of 68, from offset 0;
  - two gradient planes, 40 rows of 76, after them;
  - the response (34 rows of 68) aliases the gradient planes once the horizontal pass is done;
  - the NMS map (32 rows of 64) aliases the first sums plane once the vertical pass is done.
For every phase this checks that each read is inside its region and falls on a cell that an
earlier phase wrote.  Each write must stay inside its region and must not touch a region that the
same phase reads.  The geometry does not depend on the frame (edge tiles differ only in which
global pixels are staged), so one tile is modelled."""

import numpy as np

TW, TH = 64, 32
RW = TW + 2
GW, GH = TW + 10, TH + 8
GS, HS, RS = 76, 68, 68
THREADS = 256
OFF_H = 0
OFF_G = OFF_H + 3 * GH * HS
SMEM_FLOATS = OFF_G + 2 * GH * GS


def test_regions_fit_and_alias_as_stated():
    assert SMEM_FLOATS * 4 == 56960  # the kernel's dynamic shared memory (kSmem)
    assert (OFF_G * 4) % 16 == 0 and (GS * 4) % 16 == 0 and (HS * 4) % 16 == 0 and (RS * 4) % 16 == 0
    assert (TH + 2) * RS <= 2 * GH * GS  # the response fits in the gradient planes it replaces
    assert TH * TW <= GH * HS  # the NMS map fits in the first sums plane


def test_tma_staging_box():
    """Interior tiles of batches stage each gradient plane with one TMA copy of a GS x GH box at
    (X - 4, Y - 4): the box fills its plane exactly, the planes start 128-byte aligned in the
    dynamic shared memory, and the copy's x coordinate and row bytes meet TMA's 16-byte rule for
    every tile origin X (a multiple of TW); the box's last GS - GW columns are never read (phase
    B reads columns below GW)."""
    box_w, box_h = GS, GH
    assert box_w <= 256 and box_h <= 256 and (box_w * 4) % 16 == 0
    for plane in range(2):
        start = (OFF_G + plane * GH * GS) * 4
        assert start % 128 == 0 and start + box_w * box_h * 4 <= SMEM_FLOATS * 4
    for X in range(TW, 4096, TW):
        assert ((X - 4) * 4) % 16 == 0
    assert max(q0 + 9 for q0 in range(0, HS, 4)) < GW


def test_phases_read_written_cells():
    grads = np.zeros((GH, GS), bool)  # either plane
    # A (interior tiles): per row 18 copies of 16 bytes and one of 8 -> columns 0..73
    for i in range(GH * 19 * 2):
        k = i % (GH * 19)
        r, v = k // 19, k % 19
        cols = range(4 * v, 4 * v + 4) if v < 18 else range(72, 74)
        for c in cols:
            assert c < GS
            grads[r, c] = True
    assert grads[:, :GW].all()  # edge tiles load the same GW columns one float at a time

    # B: horizontal 7-tap sums, four columns per item, reading columns q0 .. q0+9
    sums = np.zeros((GH, HS), bool)
    for qd in range(GH * (HS // 4)):
        r, q0 = qd // (HS // 4), (qd % (HS // 4)) * 4
        for m in range(5):
            for c in (q0 + 2 * m, q0 + 2 * m + 1):
                assert grads[r, c], (r, c)
        for c in range(q0, q0 + 4):
            assert c < HS
            sums[r, c] = True

    # C: vertical 7-tap, a column pair and a strip of five rows per thread
    resp = np.zeros((TH + 2, RS), bool)
    strip, strips = 5, -(-(TH + 2) // 5)
    assert strips * (RW // 2) <= THREADS
    for tid in range(strips * (RW // 2)):
        s, q = tid // (RW // 2), (tid % (RW // 2)) * 2
        r0 = min(s * strip, TH + 2 - strip)
        keep = s * strip - r0
        for k in range(strip + 6):
            assert sums[r0 + k, q] and sums[r0 + k, q + 1], (r0 + k, q)
        for o in range(keep, strip):
            assert not resp[r0 + o, q], "two threads write one response pair"
            resp[r0 + o, q] = resp[r0 + o, q + 1] = True
        # the response (offset OFF_G) does not overlap the sums this phase reads
        assert OFF_G + (r0 + strip - 1) * RS + q + 1 >= 3 * GH * HS
    assert resp[:, :RW].all()

    # D: NMS, four pixels per item: rows r .. r+2, columns q .. q+5 of the response
    nms = np.zeros((TH, TW), bool)
    for i in range(TW * TH // 4):
        r, q = i // (TW // 4), (i % (TW // 4)) * 4
        for k in range(3):
            for c in range(q, q + 6):
                assert resp[r + k, c], (r + k, c)
        # the clamped path: neighbours (y + dy, x + p + dx) of in-frame pixels stay in rows 0..33,
        # columns 0..65 (clamping only moves them towards the tile's own pixels)
        for p in range(4):
            for dy in (-1, 0, 1):
                for dx in (-1, 0, 1):
                    assert 0 <= r + 1 + dy < TH + 2 and 0 <= q + p + 1 + dx < RW
        nms[r, q:q + 4] = True
    assert nms.all()

    # E: eight threads per cell; refinement reads the response around the cell's pixel
    for tid in range(THREADS):
        cc, g = tid >> 3, tid & 7
        ccx, ccy = cc & 7, cc >> 3
        for k in range(8):
            f = 4 * g + (k >> 1) + 32 * (k & 1)
            assert 0 <= f < 64
            assert nms[ccy * 8 + (f >> 3), ccx * 8 + (f & 7)]
    for py in range(TH):
        for px in range(TW):
            for dy, dx in ((0, 0), (0, -1), (0, 1), (-1, 0), (1, 0)):
                assert resp[py + 1 + dy, px + 1 + dx]

    # F: sub-tile sums read the response's core
    for wid in range(THREADS // 32):
        for lane in range(32):
            for s8 in range(8):
                si, sj = s8 >> 2, s8 & 3
                ty, tx = 2 * wid + (lane >> 4), lane & 15
                assert resp[si * 16 + ty + 1, sj * 16 + tx + 1]
