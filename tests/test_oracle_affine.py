"""The affine-tracker oracle (oracle/st_oracle.c) on the CPU: its column-pivoting QR solve against
numpy, and its tracks and cache entries against the reference kernels' outputs in
tests/golden/st_reference.npz (the bar is stated in affine_cases.py)."""

import numpy as np
import pytest

from affine_cases import CASES, FAR_FRAC, frames, reference_agreement, runs, st_ref  # noqa: F401
from conftest import assert_tracks_equal


def _rel_residual(a, x, b):
    a64 = a.astype(np.float64)
    return np.linalg.norm(a64 @ x - b) / (np.linalg.norm(a64, 2) * np.linalg.norm(x) + np.linalg.norm(b))


@pytest.mark.parametrize("d", [2, 6])
def test_qr_solve_well_conditioned(oracle, d):
    """Symmetric positive definite systems (the normal equations' shape).  The reference's reflector
    takes v_q = c0 - sign(c0) |c| (st_tracker.cu:114-119), which cancels when a column is nearly
    aligned with its pivot axis, so the solve is backward stable only to ~1e-4 relative, not to
    float epsilon; the bound below is that, with margin."""
    rng = np.random.default_rng(d)
    worst = 0.0
    for _ in range(200):
        m = rng.normal(size=(d, d))
        a = (m @ m.T + d * np.eye(d)).astype(np.float32)
        b = rng.normal(size=d).astype(np.float32)
        ok, x = oracle.st_qr_solve(a, b)
        assert ok
        worst = max(worst, _rel_residual(a, x, b))
    assert worst <= 2e-3, worst


def test_qr_solve_rank_deficient(oracle):
    # a zero column and row: the rank rule drops the last pivots and the solve keeps the rest
    a = np.diag([2.0, 4.0, 0.0, 0.0, 5.0, 8.0]).astype(np.float32)
    b = np.array([2.0, 8.0, 0.0, 0.0, 15.0, 32.0], np.float32)
    ok, x = oracle.st_qr_solve(a, b)
    assert ok
    np.testing.assert_allclose(x, [1, 2, 0, 0, 3, 4], atol=1e-6)
    # all-zero 2x2 system (a flat patch): solvable only with a zero right side
    z = np.zeros((2, 2), np.float32)
    assert oracle.st_qr_solve(z, np.zeros(2, np.float32))[0]
    assert not oracle.st_qr_solve(z, np.array([1.0, 0.0], np.float32))[0]


def test_qr_solve_reference_structure(oracle):
    """A normal-equation matrix of the 6-parameter system built from random gradients (symmetric,
    positive semi-definite, entries spanning several magnitudes) is solved within the same bound."""
    rng = np.random.default_rng(3)
    ix, iy = np.meshgrid(np.arange(9) - 4.0, np.arange(9) - 4.0)
    ox, oy = ix.ravel(), iy.ravel()
    gx, gy = rng.normal(0, 20, 81), rng.normal(0, 20, 81)
    jac = np.stack([ox * gx, ox * gy, oy * gx, oy * gy, gx, gy], 1)
    a = (jac.T @ jac).astype(np.float32)
    b = rng.normal(0, 100, 6).astype(np.float32)
    ok, x = oracle.st_qr_solve(a, b)
    assert ok
    assert _rel_residual(a, x, b) <= 2e-3


def test_oracle_matches_reference(oracle, golden, st_ref):
    """The oracle with the texture-unit weights (one rounding per 4-tap sum) against the reference
    kernels' outputs: the bar of affine_cases.py, and the caches' level masks and patches."""
    if st_ref is None:
        pytest.skip("tests/golden/st_reference.npz not generated")
    results = []
    for name in CASES:
        prev, nxt = frames(golden, st_ref, name)
        pp, cp = oracle.pyramid(prev), oracle.pyramid(nxt)
        gt = st_ref[f"{name}/gt"]
        for tag, (t, ns, nf, cached) in runs(golden, name).items():
            assert_tracks_equal(t, st_ref[f"{name}/{tag}/in"])
            if cached:
                tc, cache = oracle.st_build_cache(pp, t, oracle.TEXTURE_WIDE)
                got = oracle.st_track_cached(cp, cache, tc, ns, nf, oracle.TEXTURE_WIDE)
                np.testing.assert_array_equal(tc["cache_index"], np.arange(len(t)))
                np.testing.assert_array_equal(cache["level_mask"], st_ref[f"{name}/{tag}/level_mask"])
                head = st_ref[f"{name}/{tag}/cache_head"]
                np.testing.assert_allclose(cache["patch"][:len(head)], head[:, :3240].copy().view(np.float32),
                                           atol=1e-3)
            else:
                got = oracle.st_track(pp, cp, t, ns, nf, oracle.TEXTURE_WIDE)
            results.append((f"{name}/{tag}", got, st_ref[f"{name}/{tag}/out"], gt))
    assert reference_agreement(results) <= FAR_FRAC


def test_oracle_disabled_and_outside(oracle):
    """search_radius < 0 and points outside level 0 are not tracked; fields other than the outputs
    stay as they were."""
    from cuvslam_b200.types import make_tracks

    rng = np.random.default_rng(4)
    img = rng.integers(0, 256, (64, 80), dtype=np.uint8)
    pp = oracle.pyramid(img)
    t = make_tracks(np.array([[40, 30], [-2, 10], [40, 30]], np.float32), None, 10.0, 0.8)
    t["search_radius_px"][2] = -1
    t["ncc"] = 7.0
    out = oracle.st_track(pp, pp, t, 0, 20)
    assert out["track_status"][1] == 0 and out["track_status"][2] == 0
    np.testing.assert_array_equal(out["ncc"][1:], [7.0, 7.0])
    np.testing.assert_array_equal(out["track"][1:], t["track"][1:])
    # identical frames: the track converges in place
    assert out["track_status"][0] == 1
    np.testing.assert_allclose(out["track"][0], t["track"][0], atol=1e-3)
