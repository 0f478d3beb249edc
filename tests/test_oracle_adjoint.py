"""The FP64 adjoint of the differentiable LK tracker (oracle/lk_adjoint64.c) against central finite
differences of its own forward, in both modes: image pixels of both frames and track positions."""

import numpy as np
import pytest

from adjoint_cases import camera_case, mse_upstream, rel_err


@pytest.mark.parametrize("mode,iters", [(0, 400), (1, 10)])
def test_fp64_adjoint_matches_finite_differences(oracle, mode, iters):
    p8, c8, tracks, gt = camera_case(oracle, 3, 192, 144, 60)
    D = oracle.Diff64(p8.astype(np.float64), c8.astype(np.float64))
    pos, st = D.track(tracks, mode, iters)
    ok = st == 1
    if mode == oracle.IMPLICIT:
        # keep the tracks whose refinement has converged (the fixed point is what is differentiated)
        pos2, st2 = D.track(tracks, mode, iters // 2)
        ok &= (st2 == st) & (np.abs(pos2 - pos).max(1) < 1e-9)
    assert ok.sum() >= 20
    n = len(tracks)
    g = mse_upstream(pos, ok, gt, n)
    gp, gc, gtr, _ = D.backward(tracks, mode, iters, g)
    rng = np.random.default_rng(11)
    ip = rng.choice(np.flatnonzero(gp), 24, replace=False)
    ic = rng.choice(np.flatnonzero(gc), 24, replace=False)
    okt = np.flatnonzero(ok)[:12]
    fd_pix = D.fd(tracks, mode, iters, gt, ok, np.r_[np.zeros(24), np.ones(24)].astype(np.int32), np.r_[ip, ic],
                  h=1e-3)
    fd_pos = D.fd(tracks, mode, iters, gt, ok, np.r_[2 * np.ones(len(okt)), 3 * np.ones(len(okt))].astype(np.int32),
                  np.r_[okt, okt], h=1e-4)
    good = np.isfinite(fd_pix)
    assert good.sum() >= 40
    assert rel_err(np.r_[gp.ravel()[ip], gc.ravel()[ic]][good], fd_pix[good]) < 1e-5
    gpos = np.r_[gtr[okt, 0], gtr[okt, 1]]
    good = np.isfinite(fd_pos)
    assert rel_err(gpos[good], fd_pos[good]) < 1e-4
