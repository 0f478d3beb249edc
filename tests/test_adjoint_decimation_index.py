"""CPU restatement of pyramid_adjoint_kernel's transposed decimation (lk_adjoint.cu): for every pixel
(x, y) of a level, the outputs (X, Y) of the next level whose 5x5 taps read it, directly or through
the mirror, each with its weight.  The restated operator must be the exact transpose of the forward
filter-and-decimate (the oracle's restatement of gaussian_scaling_kernel, image_pyramid.cu:56-102),
weight for weight, on even and odd sizes down to the 15-pixel minimum.

The pixels that receive a mirrored tap are rows and columns 0 and 1 (virtual coordinates -1, -2)
and n-2, n-1 (virtual n+1, n, reached on odd and even sizes); both branches of the kernel (the
interior fast path and the general path) are restated, the fast path only where the kernel takes it."""

import numpy as np
import pytest


def _binom5(k):
    return (1.0, 4.0, 6.0, 4.0, 1.0)[k] / 16.0


def _sources(c, n):
    """Virtual coordinates whose mirror image is c: the kernel's a / b cases."""
    out = [c]
    if c <= 1:
        out.append(-c - 1)
    if c >= n - 2:
        out.append(2 * n - c - 1)
    return out


def _transposed(w, h, uw, uh):
    """The kernel's transposed decimation as a dense (h*w, uh*uw) matrix of weights."""
    T = np.zeros((h * w, uh * uw))
    for y in range(h):
        for x in range(w):
            row = T[y * w + x]
            if 2 <= x <= w - 3 and 2 <= y <= h - 3:
                for ky in range(y & 1, 5, 2):
                    Y = (y + 2 - ky) >> 1
                    if Y >= uh:
                        continue
                    for kx in range(x & 1, 5, 2):
                        X = (x + 2 - kx) >> 1
                        if X >= uw:
                            continue
                        row[Y * uw + X] += _binom5(ky) * _binom5(kx)
                continue
            for yc in _sources(y, h):
                yo = yc < 0 or yc >= h
                for ky in range(5):
                    vy = yc + 2 - ky
                    if vy & 1:
                        continue
                    Y = vy // 2
                    if Y < 0 or Y >= uh:
                        continue
                    for xc in _sources(x, w):
                        xo = xc < 0 or xc >= w
                        if xo and yo:
                            continue
                        for kx in range(5):
                            vx = xc + 2 - kx
                            if vx & 1:
                                continue
                            X = vx // 2
                            if X < 0 or X >= uw:
                                continue
                            row[Y * uw + X] += _binom5(ky) * _binom5(kx)
    return T


def _forward(oracle, w, h):
    """The forward decimation as a dense (uh*uw, h*w) matrix, one basis image at a time."""
    import ctypes

    uw, uh = (w + 1) // 2, (h + 1) // 2
    L = oracle.lib()
    D = np.zeros((uh * uw, h * w))
    img = np.zeros((h, w), np.float32)
    out = np.zeros((uh, uw), np.float32)
    for i in range(h * w):
        img.fill(0.0)
        img.flat[i] = 1.0
        L.or_gauss_downscale(img.ctypes.data_as(ctypes.c_void_p), w, h, out.ctypes.data_as(ctypes.c_void_p), uw, uh)
        D[:, i] = out.reshape(-1)
    return D, uw, uh


@pytest.mark.parametrize("w,h", [(15, 15), (16, 17), (17, 16), (20, 15), (31, 18), (18, 31), (24, 23)])
def test_transposed_decimation_is_the_exact_adjoint(oracle, w, h):
    D, uw, uh = _forward(oracle, w, h)
    T = _transposed(w, h, uw, uh)
    # the forward weights are products of k/16 factors: exact in FP32, so compare exactly
    np.testing.assert_array_equal(T, D.T)
    # and the rows that receive mirrored taps do receive them
    mirrored = [0, 1, h - 2, h - 1]
    assert all(np.count_nonzero(T.reshape(h, w, -1)[r]) > 0 for r in mirrored)


def _pixel_taps(x, y, w, h, uw, uh, has_grad):
    """adjoint_pixel's taps of an interior pixel in order: ('gx', row, col), ('gy', ...), ('up', ...)."""
    taps = []
    if has_grad:
        for j in range(7):
            xp = x - j + 3
            if 2 < xp < w - 3:
                taps.append(("gx", j, y, xp))
        for j in range(7):
            yp = y - j + 3
            if 2 < yp < h - 3:
                taps.append(("gy", j, yp, x))
    assert 2 <= x <= w - 3 and 2 <= y <= h - 3
    for ky in range(y & 1, 5, 2):
        Y = (y + 2 - ky) >> 1
        if Y >= uh:
            continue
        for kx in range(x & 1, 5, 2):
            X = (x + 2 - kx) >> 1
            if X >= uw:
                continue
            taps.append(("up", (ky, kx), Y, X))
    return taps


def _quad_taps(x, y, w, h, uw, uh, has_grad):
    """The kernel's four-pixel fast path (x a multiple of 4), restated: per pixel its taps in order,
    each read from the 16-byte loads the kernel makes; asserts that every load lies in its plane."""
    ub = (((x >> 1) - 1) & ~3) if (x >> 1) - 1 >= 0 else 0
    fast = x >= 8 and x + 10 <= w and 6 <= y and y + 7 <= h and ub + 8 <= uw and ((y + 2) >> 1) < uh
    if not fast:
        return None
    out = [[] for _ in range(4)]
    if has_grad:
        row = list(range(x - 4, x + 8))          # three 16-byte loads of the gradient row
        assert row[0] >= 0 and row[-1] < w
        for j in range(7):
            for i in range(4):
                out[i].append(("gx", j, y, row[i - j + 7]))
        for j in range(7):
            assert 0 <= y - j + 3 < h
            for i in range(4):
                out[i].append(("gy", j, y - j + 3, x + i))
    for ky in range(y & 1, 5, 2):
        Y = (y + 2 - ky) >> 1
        assert 0 <= Y < uh
        cols = list(range(ub, ub + 8))           # two 16-byte loads of the next level's row
        assert cols[0] >= 0 and cols[-1] < uw
        for i in range(4):
            for kx in range(i & 1, 5, 2):
                k = ((x + i + 2 - kx) >> 1) - ub
                assert 0 <= k < 8
                out[i].append(("up", (ky, kx), Y, cols[k]))
    return out


@pytest.mark.parametrize("w,h", [(15, 15), (40, 23), (80, 45), (129, 77), (160, 90), (320, 180), (1241, 376)])
def test_four_pixel_fast_path_matches_pixel_path(w, h):
    uw, uh = (w + 1) // 2, (h + 1) // 2
    taken = 0
    for has_grad in (True, False):
        for y in range(h):
            for x in range(0, w, 4):
                q = _quad_taps(x, y, w, h, uw, uh, has_grad)
                if q is None:
                    continue
                taken += 1
                for i in range(4):
                    assert q[i] == _pixel_taps(x + i, y, w, h, uw, uh, has_grad), (w, h, x + i, y)
    assert taken > 0 or w < 20 or h < 14
