"""Affine (Shi-Tomasi) tracker on the GPU: bit-identical to the oracle's FP32 restatement (every
sampling mode, cached and uncached), and against the reference's st_track / st_build_cache +
st_track_with_cache kernels (tests/golden/st_reference.npz) within the stated tolerances."""

import numpy as np
import pytest
import torch

from conftest import assert_tracks_equal, gpu_pyramid
from cuvslam_b200 import _lib
from cuvslam_b200.frontend import (AFFINE_CACHE_BYTES, STFeatureTracker, STFeatureTrackerWithCache,
                                   tracks_from_device, tracks_to_device)
from cuvslam_b200.types import make_tracks

from affine_cases import CASES, frames as _frames, reference_agreement, runs as _runs, st_ref  # noqa: F401

pytestmark = pytest.mark.gpu


def _gpu(ctx, pp, cp, t, ns, nf, cached, sampling):
    d = tracks_to_device(t)
    if cached:
        tr = STFeatureTrackerWithCache(ctx, ns, nf, sampling)
        cache = tr.build_points_cache(pp, d)
        tr.track_points(cp, cache, d)
    else:
        cache = None
        STFeatureTracker(ctx, ns, nf, sampling).track_points(pp, cp, d)
    torch.cuda.synchronize()
    return tracks_from_device(d), cache


def _oracle(oracle, opp, ocp, t, ns, nf, cached, mode):
    if cached:
        tc, cache = oracle.st_build_cache(opp, t, mode)
        return oracle.st_track_cached(ocp, cache, tc, ns, nf, mode), cache
    return oracle.st_track(opp, ocp, t, ns, nf, mode), None


def _cache_records(cache, n):
    return cache[:n].cpu().numpy().reshape(-1).view(np.dtype([("patch", np.float32, (810,)),
                                                             ("patch_sums", np.float32, (10,)),
                                                             ("level_mask", np.uint32)]))


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("sampling", [_lib.FE_SAMPLE_TEXTURE, _lib.FE_SAMPLE_EXACT, _lib.FE_SAMPLE_TEXTURE_WIDE])
def test_matches_oracle(ctx, oracle, golden, st_ref, name, sampling):
    prev, nxt = _frames(golden, st_ref, name)
    pp, cp = gpu_pyramid(ctx, prev), gpu_pyramid(ctx, nxt)
    opp, ocp = oracle.pyramid(prev), oracle.pyramid(nxt)
    for tag, (t, ns, nf, cached) in _runs(golden, name).items():
        got, gcache = _gpu(ctx, pp, cp, t, ns, nf, cached, sampling)
        want, wcache = _oracle(oracle, opp, ocp, t, ns, nf, cached, sampling)
        assert_tracks_equal(got, want)
        if cached:
            g = _cache_records(gcache, len(t))
            np.testing.assert_array_equal(g["level_mask"], wcache["level_mask"])
            for i in range(len(t)):
                for lv in range(10):
                    if (wcache["level_mask"][i] >> lv) & 1:
                        np.testing.assert_array_equal(g["patch"][i, 81 * lv:81 * lv + 81],
                                                      wcache["patch"][i, 81 * lv:81 * lv + 81])
                        assert g["patch_sums"][i, lv].tobytes() == wcache["patch_sums"][i, lv].tobytes()


def test_matches_reference(ctx, golden, st_ref):
    if st_ref is None:
        pytest.skip("tests/golden/st_reference.npz not generated")
    results = []
    for name in CASES:
        prev, nxt = _frames(golden, st_ref, name)
        pp, cp = gpu_pyramid(ctx, prev), gpu_pyramid(ctx, nxt)
        gt = st_ref[f"{name}/gt"]
        for tag, (t, ns, nf, cached) in _runs(golden, name).items():
            assert_tracks_equal(t, st_ref[f"{name}/{tag}/in"])
            got, gcache = _gpu(ctx, pp, cp, t, ns, nf, cached, _lib.FE_SAMPLE_TEXTURE_WIDE)
            results.append((f"{name}/{tag}", got, st_ref[f"{name}/{tag}/out"], gt))
            if cached:
                g = _cache_records(gcache, len(t))
                m = st_ref[f"{name}/{tag}/level_mask"]
                np.testing.assert_array_equal(g["level_mask"], m)
                used = ((m[:, None] >> np.arange(10)[None, :]) & 1).astype(bool)
                np.testing.assert_allclose(g["patch_sums"][used], st_ref[f"{name}/{tag}/patch_sums"][used],
                                           rtol=1e-4, atol=1e-2)
                head = st_ref[f"{name}/{tag}/cache_head"]
                k = len(head)
                np.testing.assert_allclose(g["patch"][:k], head[:, :3240].copy().view(np.float32), atol=1e-3)
    reference_agreement(results)


def test_edge_cases(ctx, oracle):
    """Disabled tracks, points outside the image, patches over the border, flat patches (singular
    systems), an empty call, and cache indices outside the cache."""
    rng = np.random.default_rng(12)
    img = rng.integers(0, 256, (120, 160), dtype=np.uint8)
    img[40:80, 40:80] = 128
    nxt = np.roll(img, (1, 2), (0, 1))
    xy = np.array([[0, 0], [159.9, 119.9], [-1, 5], [60, 60], [4.5, 4.5], [80, 20], [150, 100], [160, 50],
                   [30, 100]], np.float32)
    t = make_tracks(xy, np.full_like(xy, 0.5), 160.0, 0.8)
    t["search_radius_px"][5] = -1.0
    t["initial_guess_map"][8] = (1.05, 0.02, -0.03, 0.97)
    pp, cp = gpu_pyramid(ctx, img), gpu_pyramid(ctx, nxt)
    opp, ocp = oracle.pyramid(img), oracle.pyramid(nxt)
    for cached in (0, 1):
        got, _ = _gpu(ctx, pp, cp, t, 0, 20, cached, _lib.FE_SAMPLE_TEXTURE)
        want, _ = _oracle(oracle, opp, ocp, t, 0, 20, cached, oracle.TEXTURE)
        assert_tracks_equal(got, want)
        assert got["track_status"][5] == 0 and got["track_status"][2] == 0
    tr = STFeatureTrackerWithCache(ctx)
    d = tracks_to_device(t)
    cache = tr.build_points_cache(pp, d)
    ht = tracks_from_device(d)
    ht["cache_index"][0] = -1
    ht["cache_index"][1] = len(t)  # beyond the cache
    ht["cache_index"][3] = -7
    d = tracks_to_device(ht)
    tr.track_points(cp, cache, d)
    out = tracks_from_device(d)
    assert out["track_status"][0] == 0 and out["track_status"][1] == 0 and out["track_status"][3] == 0
    # empty calls
    e = torch.zeros((0, 80), dtype=torch.uint8, device="cuda")
    assert STFeatureTracker(ctx).track_points(pp, cp, e)
    assert tr.build_points_cache(pp, e).shape[1] == AFFINE_CACHE_BYTES


def test_invalid_arguments(ctx):
    import ctypes

    img = np.zeros((64, 64), np.uint8)
    pp = gpu_pyramid(ctx, img)
    d = tracks_to_device(make_tracks(np.array([[10, 10]], np.float32)))
    lib = ctx.lib
    ptr = ctypes.c_void_p(d.data_ptr())
    assert lib.fe_track_affine(ctx.handle, ctypes.byref(pp.desc), ctypes.byref(pp.desc), ptr, 1, -1, 20, 0, None) \
        == _lib.FE_ERR_INVALID_ARGUMENT
    assert lib.fe_track_affine(ctx.handle, ctypes.byref(pp.desc), ctypes.byref(pp.desc), ptr, 1, 0, 20, 7, None) \
        == _lib.FE_ERR_INVALID_ARGUMENT
    small = gpu_pyramid(ctx, np.zeros((32, 32), np.uint8))
    assert lib.fe_track_affine(ctx.handle, ctypes.byref(small.desc), ctypes.byref(pp.desc), ptr, 1, 0, 20, 0, None) \
        == _lib.FE_ERR_INVALID_ARGUMENT
    assert lib.fe_affine_build_cache(ctx.handle, ctypes.byref(pp.desc), ptr, 1, None, 0, None) \
        == _lib.FE_ERR_INVALID_ARGUMENT
