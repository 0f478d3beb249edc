"""The CPU oracle against the reference's own kernels (outputs recorded on a B200 by
tests/golden/make_golden.py from oracle/_ref, i.e. cuVSLAM's cuda_kernels compiled unchanged)."""

import hashlib
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))

CASES = ["c1", "half", "odd", "tiny"]


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("name", CASES)
def test_pyramid_and_gradients_bit_exact(oracle, golden, name):
    inp, ref = golden
    for tag in ("prev", "next"):
        pyr = oracle.pyramid(inp[f"{name}/{tag}"])
        for l, (img, gx, gy) in enumerate(pyr):
            assert _sha(img) == str(ref[f"{name}/{tag}/L{l}/img/sha"]), (tag, l)
            assert _sha(gx) == str(ref[f"{name}/{tag}/L{l}/gx/sha"]), (tag, l)
            assert _sha(gy) == str(ref[f"{name}/{tag}/L{l}/gy/sha"]), (tag, l)
        assert f"{name}/{tag}/L{len(pyr)}/img/sha" not in ref  # same level count


def test_four_level_cap(oracle, golden):
    inp, ref = golden
    pyr = oracle.pyramid(inp["c1/prev"], max_levels=4)
    assert len(pyr) == 4
    for l, (img, _, _) in enumerate(pyr):
        assert _sha(img) == str(ref[f"c1/prev4/L{l}/img/sha"])


@pytest.mark.parametrize("name", CASES)
def test_selection_matches_reference(oracle, golden, name):
    """Oracle response (logf instead of the reference's __logf) + selection vs the reference's
    selected features: same count, same positions up to the refinement's division rounding."""
    inp, ref = golden
    pyr = oracle.pyramid(inp[f"{name}/prev"])
    resp = oracle.gftt(pyr[0][1], pyr[0][2])
    for tag, borders in (("sel0", (0, 0, 0, 0)), ("sel1", (3, 4, 5, 6))):
        alive = ref[f"{name}/sel1/alive"] if tag == "sel1" else None
        nd = 450 - (0 if alive is None else len(alive))
        s = oracle.select(resp, alive, nd, borders)
        rsel = ref[f"{name}/{tag}/sel"]
        assert len(s["sel"]) == len(rsel)
        if len(rsel):
            # identical set; order may differ only between exactly tied strengths
            d = np.abs(np.sort(s["sel"].view(np.complex64).ravel()) - np.sort(rsel.view(np.complex64).ravel()))
            assert d.max() < 1e-4
        np.testing.assert_allclose(s["bins"], ref[f"{name}/{tag}/bins"], rtol=2e-6, atol=1e-4)
        rkp = ref[f"{name}/{tag}/kp"]
        assert len(s["kp"]) == len(rkp)
        np.testing.assert_allclose(s["kp"][:, 2], rkp[:, 2], rtol=0, atol=1e-6)


@pytest.mark.parametrize("name", ["c1", "half", "odd"])
@pytest.mark.parametrize("run", ["lk_zero", "lk_pred", "lk_retrack", "lk_horiz", "lk_pred4"])
def test_lk_matches_reference(oracle, golden, name, run):
    """Oracle LK (texture-weight emulation) vs the reference kernel: identical track status and
    positions within 1e-3 px (texture hardware accumulates with its own rounding)."""
    inp, ref = golden
    src = {"lk_horiz": "lk_zero", "lk_pred4": "lk_pred"}.get(run, run)
    tin, tout = ref[f"{name}/{src}/in"], ref[f"{name}/{run}/out"]
    pp = oracle.pyramid(inp[f"{name}/prev"], max_levels=4 if run == "lk_pred4" else 10)
    cp = oracle.pyramid(inp[f"{name}/next"])
    o = oracle.lk(pp, cp, tin, horizontal=(run == "lk_horiz"))
    np.testing.assert_array_equal(o["track_status"], tout["track_status"])
    ok = o["track_status"] == 1
    d = np.linalg.norm(o["track"][ok] - tout["track"][ok], axis=1)
    assert d.max() < 1e-3
    np.testing.assert_array_equal(o["info"], tout["info"])


def test_lk_tracks_known_motion(oracle, golden):
    """Tracked positions follow the synthetic warp: median error against the analytic flow is small."""
    inp, ref = golden
    pp = oracle.pyramid(inp["c1/prev"])
    cp = oracle.pyramid(inp["c1/next"])
    o = oracle.lk(pp, cp, ref["c1/lk_pred/in"])
    ok = o["track_status"] == 1
    err = np.linalg.norm(o["track"][ok] - ref["c1/gt"][ok], axis=1)
    assert ok.mean() > 0.4
    assert np.median(err) < 0.3


def test_texture_weight_rule(oracle, golden):
    """Emulated cudaFilterModeLinear weights: exact on the sub-texel sweep, and within a few ulp of
    the hardware on random coordinates (the hardware's final accumulation rounds differently)."""
    from make_golden import tex_probe_inputs

    _, ref = golden
    img, step, sweep, xy = tex_probe_inputs()
    got = oracle.tex_sample(step, sweep)
    np.testing.assert_array_equal(got, ref["tex/sweep"])
    r = ref["tex/random"]
    got = oracle.tex_sample(img, xy)
    err = np.abs(got.astype(np.float64) - r) / np.maximum(np.abs(r).astype(np.float64), 1.0)
    assert err.max() < 2e-5
    assert np.mean(got == r) > 0.6


def test_bilinear_ramp_known_answer(oracle):
    """ImagePyramid.ComputePatchInterpolatesCorrectly (libs/sof/test/interpolation_test.cpp:24-72):
    on a vertical ramp, a quarter-pixel sample is exact in both sampling modes."""
    img = np.repeat(np.arange(64, dtype=np.float32)[:, None], 64, 1)
    for mode in (oracle.TEXTURE, oracle.EXACT):
        v = oracle.tex_sample(img, [(10.75, 10.75), (12.75, 20.75)], mode)
        np.testing.assert_array_equal(v, [10.25, 20.25])
        v = oracle.tex_sample(img.T.copy(), [(10.75, 10.75)], mode)
        np.testing.assert_array_equal(v, [10.25])


def test_lk_f64_close_to_fp32(oracle, golden):
    inp, ref = golden
    pp = oracle.pyramid(inp["half/prev"])
    cp = oracle.pyramid(inp["half/next"])
    t = ref["half/lk_pred/in"]
    a = oracle.lk(pp, cp, t, mode=oracle.EXACT)
    b = oracle.lk(pp, cp, t, f64=True)
    ok = (a["track_status"] == 1) & (b["track_status"] == 1)
    assert ok.sum() > 0.8 * min(a["track_status"].sum(), b["track_status"].sum())
    d = np.linalg.norm(a["track"][ok] - b["track"][ok], axis=1)
    assert np.median(d) < 1e-3
