"""Central finite differences of the FP64 forward (oracle.Diff64.fd), one probe per task, for a
spawned process pool.  A worker rebuilds a camera from its seed (the same frames, features and
ground truth as the test's) and keeps its FP64 pyramids for later probes."""

import numpy as np

_CAMS = {}


def camera_inputs(cam, w, h, nfeat):
    """(level-0 images as the plan scales them: float32(u8) / 255 * 255 in FP32, then float64;
    tracks; ground truth) of camera `cam`."""
    from adjoint_cases import camera_case
    from oracle import oracle as O

    p8, c8, tracks, gt = camera_case(O, cam, w, h, nfeat)
    s = np.float32(255.0)
    lv = [((a.astype(np.float32) / s) * s).astype(np.float64) for a in (p8, c8)]
    return lv[0], lv[1], tracks, gt


def probe(args):
    """args: (camera, w, h, features, n, mode, iters, ok mask, which, index, h) -> derivative."""
    from oracle import oracle as O

    cam, w, h, nfeat, n, mode, iters, ok, which, index, step = args
    if cam not in _CAMS:
        prev, cur, tracks, gt = camera_inputs(cam, w, h, nfeat)
        _CAMS[cam] = (O.Diff64(prev, cur), tracks[:n], gt[:n])
    D, tracks, gt = _CAMS[cam]
    return float(D.fd(tracks, mode, iters, gt, ok, np.array([which], np.int32), np.array([index], np.int64), h=step,
                      strict=True)[0])
