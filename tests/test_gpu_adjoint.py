"""CUDA adjoint of the differentiable LK tracker: against the FP64 adjoint (oracle/lk_adjoint64.c),
against central finite differences (h = 1e-3) of the FP64 forward on 256 random pixels and on track
positions, deterministic, and through the torch.autograd.Function.  Tolerance: 1e-3 relative
(norm over the compared entries)."""

import numpy as np
import pytest
import torch

from adjoint_cases import camera_case, mse_upstream, rel_err
from cuvslam_b200.diff import DiffTracker

pytestmark = pytest.mark.gpu

ITERS = {"implicit": 20, "unrolled": 10}
ORACLE_ITERS = {"implicit": 40, "unrolled": 10}
TOL = 1e-3


def _setup(ctx, oracle, mode, w, h, nfeat, cam=3):
    p8, c8, tracks, gt = camera_case(oracle, cam, w, h, nfeat)
    n = len(tracks)
    t = DiffTracker(ctx, 1, h, w, n, mode=mode, iterations=ITERS[mode])
    prev = torch.from_numpy(p8.astype(np.float32) / 255.0).cuda()[None]
    cur = torch.from_numpy(c8.astype(np.float32) / 255.0).cuda()[None]
    xy = torch.from_numpy(np.ascontiguousarray(tracks["track"])).cuda()[None]
    t.set_inputs(prev, cur, xy)
    t.build_pyramids()
    t.forward_step()
    pos, st = t.outputs()
    torch.cuda.synchronize()
    pos = pos[0].double().cpu().numpy()
    st = st[0].cpu().numpy()
    # the pyramids hold 255 * frame (FP32 product), the oracle gets the same level-0 images
    s = np.float32(t.scale)
    D = oracle.Diff64((t.prev_img[0].cpu().numpy() * s).astype(np.float64),
                      (t.cur_img[0].cpu().numpy() * s).astype(np.float64))
    mo = oracle.IMPLICIT if mode == "implicit" else oracle.UNROLLED
    pos64, st64 = D.track(tracks, mo, ORACLE_ITERS[mode])
    # compared: tracks both trackers keep, at the same place (FP32 and FP64 decisions can differ
    # where a gate is met within rounding)
    ok = st & (st64 == 1) & (np.abs(pos - pos64).max(1) < 1e-3)
    if mode == "implicit":
        p2, s2 = D.track(tracks, mo, ORACLE_ITERS[mode] // 2)
        ok &= (s2 == st64) & (np.abs(p2 - pos64).max(1) < 1e-9)
    return t, D, mo, tracks, gt, pos, st, pos64, st64, ok


def _backward(t, g):
    t.grad_xy.copy_(torch.from_numpy(g.astype(np.float32)).cuda()[None])
    t.backward_step()
    torch.cuda.synchronize()
    return (t.grad_prev[0].double().cpu().numpy(), t.grad_cur[0].double().cpu().numpy(),
            t.grad_track[0].double().cpu().numpy(), t.grad_offset[0].double().cpu().numpy())


@pytest.mark.parametrize("mode", ["implicit", "unrolled"])
def test_forward_matches_fp64(ctx, oracle, mode):
    t, D, mo, tracks, gt, pos, st, pos64, st64, ok = _setup(ctx, oracle, mode, 320, 240, 200)
    both = (st == 1) & (st64 == 1)
    assert both.sum() >= 0.85 * max(st.sum(), st64.sum())
    d = np.linalg.norm(pos[both] - pos64[both], axis=1)
    assert np.median(d) < 1e-3 and np.percentile(d, 99) < 1e-2


@pytest.mark.parametrize("mode", ["implicit", "unrolled"])
@pytest.mark.parametrize("size", [(320, 240, 200), (1280, 720, 4096)])
def test_adjoint_matches_fp64(ctx, oracle, mode, size):
    w, h, nf = size
    t, D, mo, tracks, gt, pos, st, pos64, st64, ok = _setup(ctx, oracle, mode, w, h, nf)
    assert ok.sum() >= 0.2 * len(tracks)
    g = mse_upstream(pos64, ok, gt, len(tracks))
    gp, gc, gtr, gof = _backward(t, g)
    assert t.dropped() == 0
    rp, rc, rt, ro = D.backward(tracks, mo, ORACLE_ITERS[mode], g)
    assert rel_err(gp, rp) < TOL, "previous image"
    assert rel_err(gc, rc) < TOL, "current image"
    assert rel_err(gtr[ok], rt[ok]) < TOL, "track positions"
    if mode == "unrolled":
        assert rel_err(gof[ok], ro[ok]) < TOL, "offsets"
    else:
        assert not gof.any()
    # failed or excluded tracks contribute nothing
    assert not gtr[~ok].any()


@pytest.mark.parametrize("mode", ["implicit", "unrolled"])
def test_adjoint_matches_finite_differences(ctx, oracle, mode):
    t, D, mo, tracks, gt, pos, st, pos64, st64, ok = _setup(ctx, oracle, mode, 320, 240, 200)
    n = len(tracks)
    g = mse_upstream(pos64, ok, gt, n)
    gp, gc, gtr, _ = _backward(t, g)
    rng = np.random.default_rng(5)
    ip = rng.choice(np.flatnonzero(gp), 128, replace=False)
    ic = rng.choice(np.flatnonzero(gc), 128, replace=False)
    which = np.r_[np.zeros(128), np.ones(128)].astype(np.int32)
    fd = D.fd(tracks, mo, ORACLE_ITERS[mode], gt, ok, which, np.r_[ip, ic], h=1e-3)
    good = np.isfinite(fd)
    assert good.sum() >= 240
    assert rel_err(np.r_[gp.ravel()[ip], gc.ravel()[ic]][good], fd[good]) < TOL
    okt = np.flatnonzero(ok)[:32]
    fdp = D.fd(tracks, mo, ORACLE_ITERS[mode], gt, ok, np.r_[2 * np.ones(len(okt)), 3 * np.ones(len(okt))].astype(np.int32),
               np.r_[okt, okt], h=1e-4)
    good = np.isfinite(fdp)
    assert rel_err(np.r_[gtr[okt, 0], gtr[okt, 1]][good], fdp[good]) < TOL


@pytest.mark.parametrize("mode", ["implicit", "unrolled"])
def test_adjoint_is_deterministic(ctx, oracle, mode):
    t, D, mo, tracks, gt, pos, st, pos64, st64, ok = _setup(ctx, oracle, mode, 640, 480, 1500)
    g = mse_upstream(pos, st.astype(bool), gt, len(tracks))
    a = _backward(t, g)
    b = _backward(t, g)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x.view(np.uint64), y.view(np.uint64))


def test_autograd_function(ctx, oracle):
    p8, c8, tracks, gt = camera_case(oracle, 4, 320, 240, 150)
    n = len(tracks)
    t = DiffTracker(ctx, 2, 240, 320, n, mode="implicit")
    prev = torch.from_numpy(np.stack([p8, p8]).astype(np.float32) / 255.0).cuda().requires_grad_()
    cur = torch.from_numpy(np.stack([c8, c8]).astype(np.float32) / 255.0).cuda().requires_grad_()
    xy = torch.from_numpy(np.stack([tracks["track"]] * 2)).cuda().requires_grad_()
    pos, st = t(prev, cur, xy)
    gtt = torch.from_numpy(np.stack([gt, gt]).astype(np.float32)).cuda()
    loss = (((pos - gtt) ** 2).sum(-1) * st).sum() / (2 * n)
    loss.backward()
    assert prev.grad.shape == prev.shape and cur.grad.shape == cur.shape and xy.grad.shape == xy.shape
    # both cameras see the same frames: identical gradients
    torch.testing.assert_close(prev.grad[0], prev.grad[1], rtol=0, atol=0)
    torch.testing.assert_close(xy.grad[0], xy.grad[1], rtol=0, atol=0)
    # the function's image gradient is the plan's gradient times the intensity scale
    torch.testing.assert_close(prev.grad, t.grad_prev * 255.0, rtol=0, atol=0)
    assert torch.isfinite(prev.grad).all() and prev.grad.abs().sum() > 0


@pytest.mark.parametrize("mode", ["implicit", "unrolled"])
def test_adjoint_finite_differences_eight_cameras(ctx, oracle, mode):
    """At the LK adjoint configuration's size: 8 cameras of 1280x720, frames in [0, 1], 4096 tracks
    each, one plan over all cameras; the image gradients against central finite differences
    (h = 1e-3) of the FP64 forward on 256 random pixels (16 per camera and frame).  The loss counts
    64 random kept tracks per camera (the forward tracks all of them), so that few perturbations
    reach a track sitting on a decision threshold.  A pixel moves only its own camera's loss, so each
    probe re-runs one camera's FP64 forward; the probes run on a spawned process pool.  Tolerance
    1e-3 relative over the probes whose perturbation leaves every counted track's decisions (levels
    set up and accepted, steps per level, success) unchanged; at least 80% of the probes."""
    import multiprocessing as mp

    import adjoint_fd_pool

    cams, w, h = 8, 1280, 720
    cases = [camera_case(oracle, 40 + c, w, h, 4096) for c in range(cams)]
    n = min(len(c[2]) for c in cases)
    t = DiffTracker(ctx, cams, h, w, n, mode=mode, iterations=ITERS[mode])
    prev = torch.from_numpy(np.stack([c[0] for c in cases]).astype(np.float32) / 255.0).cuda()
    cur = torch.from_numpy(np.stack([c[1] for c in cases]).astype(np.float32) / 255.0).cuda()
    xy = torch.from_numpy(np.stack([np.ascontiguousarray(c[2]["track"][:n]) for c in cases])).cuda()
    t.set_inputs(prev, cur, xy)
    t.build_pyramids()
    t.forward_step()
    pos, st = t.outputs()
    torch.cuda.synchronize()
    pos, st = pos.double().cpu().numpy(), st.cpu().numpy()
    s = np.float32(t.scale)
    mo = oracle.IMPLICIT if mode == "implicit" else oracle.UNROLLED
    levels0 = [((t.prev_img[c].cpu().numpy() * s).astype(np.float64), (t.cur_img[c].cpu().numpy() * s).astype(np.float64))
               for c in range(cams)]
    # the workers rebuild these from the seeds: check that they get the same images
    again = adjoint_fd_pool.camera_inputs(40, w, h, 4096)
    assert np.array_equal(again[0], levels0[0][0]) and np.array_equal(again[1], levels0[0][1])
    g = np.zeros((cams, n, 2))
    oks = []
    rng = np.random.default_rng(11)
    for c in range(cams):
        D = oracle.Diff64(*levels0[c])
        pos64, st64 = D.track(cases[c][2][:n], mo, ORACLE_ITERS[mode])
        ok = st[c] & (st64 == 1) & (np.abs(pos[c] - pos64).max(1) < 1e-3)
        keep = np.zeros(n, bool)
        keep[rng.choice(np.flatnonzero(ok), min(64, int(ok.sum())), replace=False)] = True
        oks.append(keep)
        g[c] = mse_upstream(pos64, keep, cases[c][3][:n], n)
    t.grad_xy.copy_(torch.from_numpy(g.astype(np.float32)).cuda())
    t.backward_step()
    torch.cuda.synchronize()
    gp, gc = t.grad_prev.double().cpu().numpy(), t.grad_cur.double().cpu().numpy()
    tasks, want = [], []
    for c in range(cams):
        for which, grad in ((0, gp[c]), (1, gc[c])):
            for idx in rng.choice(np.flatnonzero(grad), 16, replace=False):
                tasks.append((40 + c, w, h, 4096, n, mo, ORACLE_ITERS[mode], oks[c].astype(np.uint8), which,
                              int(idx), 1e-3))
                want.append(grad.ravel()[idx])
    with mp.get_context("spawn").Pool(min(16, mp.cpu_count())) as pool:
        fd = np.array(pool.map(adjoint_fd_pool.probe, tasks, chunksize=1))
    good = np.isfinite(fd)
    assert good.sum() >= 0.8 * len(fd), good.sum()
    assert rel_err(np.array(want)[good], fd[good]) < TOL
