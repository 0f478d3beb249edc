"""Shared inputs of the adjoint tests: a seeded camera (previous and warped current frame), Shi-Tomasi
features selected by the oracle on the previous frame, and the warp's ground truth."""

import numpy as np

from cuvslam_b200 import synthetic as S
from cuvslam_b200.types import make_tracks


def camera_case(oracle, cam, width, height, n_features):
    """(prev u8, cur u8, tracks (TRACK_DTYPE, zero offset), ground-truth positions (n, 2) float64)."""
    p8, c8, warp = S.frame_pair(cam, width, height)
    pyr = oracle.pyramid(p8)
    resp = oracle.gftt(pyr[0][1], pyr[0][2])
    xy = np.asarray(oracle.select(resp, None, n_features)["sel"], np.float32).reshape(-1, 2)
    gx, gy = warp.apply(xy[:, 0].astype(np.float64), xy[:, 1].astype(np.float64))
    return p8, c8, make_tracks(xy, np.zeros_like(xy)), np.stack([gx, gy], 1)


def mse_upstream(pos, ok, gt, n):
    """dL/dpos of L = sum_{ok} |pos - gt|^2 / n."""
    return np.where(ok[:, None], 2.0 * (pos - gt) / n, 0.0)


def rel_err(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
