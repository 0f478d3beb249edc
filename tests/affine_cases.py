"""Shared cases of the affine-tracker tests: the st_reference.npz runs and the agreement bar
against the reference kernels."""

import os
import sys

import numpy as np
import pytest

from conftest import ROOT

sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
import make_golden as MG  # noqa: E402

ST_REF = os.path.join(ROOT, "tests", "golden", "st_reference.npz")
CASES = MG.ST_CASES + ("rot",)


@pytest.fixture(scope="module")
def st_ref():
    return np.load(ST_REF) if os.path.exists(ST_REF) else None


def frames(golden, st_ref, name):
    """(prev, next) u8 frames of a case ("rot" from the fixture when present)."""
    inp, _ = golden
    if name == "rot" and st_ref is not None:
        return st_ref["rot/prev"], st_ref["rot/next"]
    prev, nxt, _ = MG.st_frames(name, inp)
    return prev, nxt


def runs(golden, name):
    """tag -> (records, n_shift, n_full, cached) of a case."""
    inp, ref = golden
    prev, _, warp = MG.st_frames(name, inp)
    r, _ = MG.st_runs(name, prev, warp, MG.st_points(name, ref, prev))
    return r


# Against the reference kernels (texture-unit sampling, FMA-contracted sequential sums): twenty
# affine Gauss-Newton steps amplify last-bit differences of the sampled values, so a marginal track
# can settle elsewhere or fall on the other side of the convergence or NCC gate.  The size of that
# effect is a property of the algorithm: the oracle run twice on these fixtures with sample values
# that differ only in their last bit (texture weights summed in FP32 vs rounded once) disagrees on
# up to 3% of statuses and moves 2.2% of the tracks both keep by more than 0.05 px.  Bar, per run:
# statuses agree on >= 95% of the tracks and the median offset of tracks both keep is <= 0.01 px
# (runs with >= 5 such tracks); over all runs: <= 4% of those tracks are more than 0.05 px apart,
# and their mean error against the true motion differs from the reference's by <= 0.01 px.
STATUS_AGREE = 0.95
FAR_PX, FAR_FRAC = 0.05, 0.04


def reference_agreement(results):
    """results: [(tag, got, want, gt)].  Asserts the bar above; returns the pooled far fraction."""
    common = far = 0
    err_got, err_want = [], []
    for tag, got, want, gt in results:
        agree = (got["track_status"] == want["track_status"]).mean()
        assert agree >= STATUS_AGREE, (tag, agree)
        ok = (got["track_status"] == 1) & (want["track_status"] == 1)
        d = np.linalg.norm(got["track"][ok] - want["track"][ok], axis=1)
        if ok.sum() >= 5:
            assert np.median(d) <= 0.01, (tag, np.median(d))
        common += int(ok.sum())
        far += int((d > FAR_PX).sum())
        err_got.append(np.linalg.norm(got["track"][ok] - gt[ok], axis=1))
        err_want.append(np.linalg.norm(want["track"][ok] - gt[ok], axis=1))
    assert common > 0 and far / common <= FAR_FRAC, (far, common)
    assert abs(np.concatenate(err_got).mean() - np.concatenate(err_want).mean()) <= 0.01
    return far / common
