"""CPU checks of the input stage: the oracle's RGB -> gray conversion and box prefilter, followed by
its pyramid, against the reference's own kernels (tests/golden/input_reference.npz, made by
tests/golden/make_golden.py input-reference on a B200)."""

import hashlib
import os
import sys

import numpy as np
import pytest

from conftest import ROOT

sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))

GOLD = os.path.join(ROOT, "tests", "golden")


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.fixture(scope="module")
def input_ref():
    path = os.path.join(GOLD, "input_reference.npz")
    if not os.path.exists(path):
        pytest.skip("input_reference.npz not generated")
    return np.load(path)


def matching_rgb_variant(oracle, golden, input_ref):
    """The contraction of the reference's RGB expression: the oracle variant that reproduces the
    reference's level 0 of the 'odd' RGB frame bit for bit (None if none does)."""
    from make_golden import input_frame

    inp, _ = golden
    rgb = input_frame(inp, "odd", True)
    want = input_ref["odd/rgb/level0"]
    for v in range(5):
        if np.array_equal(oracle.rgb_to_gray(rgb, v), want):
            return v
    return None


def test_rgb_variant_is_pinned(oracle, golden, input_ref):
    assert matching_rgb_variant(oracle, golden, input_ref) == oracle.RGB_VARIANT


@pytest.mark.parametrize("name", ["c1", "odd", "tiny"])
@pytest.mark.parametrize("mode", ["mono_box3", "rgb", "rgb_box3"])
def test_input_stage_pyramid_matches_reference(oracle, golden, input_ref, name, mode):
    from make_golden import INPUT_MODES, input_frame

    inp, _ = golden
    rgb, box = INPUT_MODES[mode]
    pyr = oracle.pyramid_f32(oracle.level0(input_frame(inp, name, rgb), box=bool(box)))
    for l, (img, gx, gy) in enumerate(pyr):
        assert _sha(img) == str(input_ref[f"{name}/{mode}/L{l}/img/sha"]), (l, "img")
        assert _sha(gx) == str(input_ref[f"{name}/{mode}/L{l}/gx/sha"]), (l, "gx")
        assert _sha(gy) == str(input_ref[f"{name}/{mode}/L{l}/gy/sha"]), (l, "gy")


def test_box3_on_integers_is_the_integer_rule(oracle):
    """On integer input the prefilter is exact: interior = (sum of [1 2 1] x [1 2 1] weighted
    pixels) >> 4, border ring = input."""
    rng = np.random.default_rng(4)
    img = rng.integers(0, 256, (23, 31)).astype(np.float32)
    got = oracle.box3(img)
    k = np.array([1, 2, 1])
    want = img.copy()
    for y in range(1, 22):
        for x in range(1, 30):
            want[y, x] = int((np.outer(k, k) * img[y - 1:y + 2, x - 1:x + 2]).sum()) >> 4
    np.testing.assert_array_equal(got, want)
