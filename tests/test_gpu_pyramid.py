"""Pyramid + gradient kernels on the GPU: bit-identical to the oracle (and so to the reference)."""

import hashlib

import numpy as np
import pytest
import torch

from conftest import gpu_pyramid

pytestmark = pytest.mark.gpu


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("name", ["c1", "half", "odd", "tiny"])
def test_matches_reference_hashes(ctx, golden, name):
    inp, ref = golden
    for tag in ("prev", "next"):
        p = gpu_pyramid(ctx, inp[f"{name}/{tag}"])
        for l, (img, gx, gy) in enumerate(p.to_numpy()):
            assert _sha(img) == str(ref[f"{name}/{tag}/L{l}/img/sha"]), (tag, l, "img")
            assert _sha(gx) == str(ref[f"{name}/{tag}/L{l}/gx/sha"]), (tag, l, "gx")
            assert _sha(gy) == str(ref[f"{name}/{tag}/L{l}/gy/sha"]), (tag, l, "gy")


@pytest.mark.parametrize("shape", [(15, 15), (16, 17), (61, 97), (240, 376), (376, 1241), (480, 640), (33, 1000),
                                   (1000, 33), (720, 1280), (1200, 1920), (1920, 2560), (3000, 4000)])
def test_matches_oracle_random_sizes(ctx, oracle, shape):
    """Every level bit-identical to the oracle.  The sizes cover the deeper levels computed inside the
    levels 0-2 launch with no banded phase, one (1920x1200) and two (2560x1920), and a frame too
    large for that (4000x3000, generic stages)."""
    rng = np.random.default_rng(shape[0] * 7919 + shape[1])
    img = rng.integers(0, 256, shape, dtype=np.uint8)
    got = gpu_pyramid(ctx, img).to_numpy()
    want = oracle.pyramid(img)
    assert len(got) == len(want)
    for l, (g, w) in enumerate(zip(got, want)):
        for q in range(3):
            np.testing.assert_array_equal(g[q], w[q], err_msg=f"level {l} plane {q}")


def test_level_cap_and_f32_input(ctx, oracle):
    from cuvslam_b200.frontend import ImagePyramid

    rng = np.random.default_rng(3)
    img = rng.integers(0, 256, (300, 410), dtype=np.uint8)
    p = gpu_pyramid(ctx, img, max_levels=4)
    assert p.levels == 4
    for g, w in zip(p.to_numpy(), oracle.pyramid(img, max_levels=4)):
        np.testing.assert_array_equal(g[0], w[0])
    f = rng.random((300, 410), dtype=np.float32)
    q = ImagePyramid(410, 300)
    q.build_f32(ctx, torch.from_numpy(f).cuda())
    torch.cuda.synchronize()
    for g, w in zip(q.to_numpy(), oracle.pyramid_f32(f)):
        for k in range(3):
            np.testing.assert_array_equal(g[k], w[k])


def test_full_size_properties(ctx):
    """1920x1200 (7 levels): level l+1 of a constant image is constant except where corner taps are
    dropped, and gradients of a horizontal ramp are constant inside the 3-px border."""
    from cuvslam_b200.frontend import ImagePyramid

    w, h = 1920, 1200
    ramp = np.tile((np.arange(w) % 200).astype(np.uint8), (h, 1))
    p = ImagePyramid(w, h)
    p.build(ctx, torch.from_numpy(ramp).cuda())
    torch.cuda.synchronize()
    assert p.levels == 7
    gx = p.grad_x(0).cpu().numpy()
    inner = gx[3:-3, 10:190]
    assert np.abs(inner - inner[0, 0]).max() < 1e-4
    assert np.all(gx[:, :3] == 0) and np.all(gx[:, -3:] == 0)
    gy = p.grad_y(0).cpu().numpy()
    assert np.abs(gy).max() < 1e-4
