"""Pyramid + gradient kernels on the GPU: bit-identical to the oracle (and so to the reference)."""

import hashlib
import os
import sys

import numpy as np
import pytest
import torch

from conftest import ROOT, gpu_pyramid
from cuvslam_b200.frontend import ImagePyramid

sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))

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


def _rgb_variant(oracle, golden):
    from test_oracle_input import matching_rgb_variant

    path = os.path.join(ROOT, "tests", "golden", "input_reference.npz")
    if not os.path.exists(path):
        pytest.skip("input_reference.npz not generated")
    v = matching_rgb_variant(oracle, golden, np.load(path))
    assert v is not None, "no oracle variant reproduces the reference's RGB conversion"
    return v


@pytest.mark.parametrize("shape", [(17, 31), (40, 50), (61, 97), (162, 176), (163, 200), (480, 752), (1200, 1920)])
@pytest.mark.parametrize("mode", ["mono_box3", "rgb", "rgb_box3"])
def test_input_stage_matches_oracle(ctx, oracle, golden, shape, mode):
    """RGB8 input (gray conversion) and the box prefilter: every level bit-identical to the oracle.
    Mono frames of three or more levels take the prefilter inside the levels 0-2 kernel, smaller ones
    and every RGB frame the input kernel."""
    rgb, box = mode.startswith("rgb"), mode.endswith("box3")
    rng = np.random.default_rng(shape[0] * 31 + shape[1] + (7 if rgb else 0))
    img = rng.integers(0, 256, shape + ((3,) if rgb else ()), dtype=np.uint8)
    if rgb:
        oracle_img = oracle.rgb_to_gray(img, _rgb_variant(oracle, golden))
        base = oracle.box3(oracle_img) if box else oracle_img
    else:
        base = oracle.level0(img, box=True)
    want = oracle.pyramid_f32(base)
    h, w = shape
    p = ImagePyramid(w, h).build(ctx, torch.from_numpy(img).cuda(), blur_filter=box)
    torch.cuda.synchronize()
    got = p.to_numpy()
    assert len(got) == len(want)
    for l, (g, wv) in enumerate(zip(got, want)):
        for q in range(3):
            np.testing.assert_array_equal(g[q], wv[q], err_msg=f"level {l} plane {q}")


@pytest.mark.parametrize("name", ["c1", "odd", "tiny"])
@pytest.mark.parametrize("mode", ["mono_box3", "rgb", "rgb_box3"])
def test_input_stage_matches_reference_hashes(ctx, golden, name, mode):
    path = os.path.join(ROOT, "tests", "golden", "input_reference.npz")
    if not os.path.exists(path):
        pytest.skip("input_reference.npz not generated")
    from make_golden import INPUT_MODES, input_frame

    ref = np.load(path)
    inp, _ = golden
    rgb, box = INPUT_MODES[mode]
    img = input_frame(inp, name, rgb)
    h, w = img.shape[:2]
    p = ImagePyramid(w, h).build(ctx, torch.from_numpy(img).cuda(), blur_filter=bool(box))
    torch.cuda.synchronize()
    for l, (a, gx, gy) in enumerate(p.to_numpy()):
        assert _sha(a) == str(ref[f"{name}/{mode}/L{l}/img/sha"]), (l, "img")
        assert _sha(gx) == str(ref[f"{name}/{mode}/L{l}/gx/sha"]), (l, "gx")
        assert _sha(gy) == str(ref[f"{name}/{mode}/L{l}/gy/sha"]), (l, "gy")
