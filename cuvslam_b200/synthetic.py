"""Seeded synthetic camera scenes for the tracking front-end workloads.

cuVSLAM's own tests read KITTI frames and git-lfs PNGs that are not available offline, so every
workload here is drawn from a seed instead.  A scene is a continuous intensity function

    f(p) = 128 + sum_k a_k exp(-|p - c_k|^2 / (2 s_k^2)) + value_noise(p)

with 400 Gaussian blobs (sigma U(2,20) px, amplitude U(-60,60)) and 4 octaves of lattice value noise.
A frame is f sampled through a similarity warp T (rotation, isotropic scale, translation), so the
ground-truth flow of every pixel is known analytically: pixel-centre coordinate p in the base
frame moves to T(p).  Frames other than the base get additive Gaussian noise (sigma 2) before
re-quantisation to uint8.

Coordinates: pixel (i, j) has its centre at (i, j).  cuVSLAM's LK works in texture coordinates
where pixel i spans [i, i+1) (lk_tracker.cu:150-160 samples at x - 0.5), so a track at texture
coordinate u sits at pixel-centre coordinate u - 0.5; `flow_texture` converts.
"""

from __future__ import annotations

import dataclasses
import math

import numpy as np

_MARGIN = 96.0  # scene content extends this far outside the frame so warps never see blank space


@dataclasses.dataclass(frozen=True)
class Similarity:
    """p' = s * R(theta) p + t, about the frame centre (cx, cy)."""

    theta: float = 0.0
    scale: float = 1.0
    tx: float = 0.0
    ty: float = 0.0
    cx: float = 0.0
    cy: float = 0.0

    def _mat(self):
        c, s = math.cos(self.theta), math.sin(self.theta)
        return np.array([[c, -s], [s, c]]) * self.scale

    def apply(self, x, y):
        m = self._mat()
        xc, yc = np.asarray(x, np.float64) - self.cx, np.asarray(y, np.float64) - self.cy
        return (m[0, 0] * xc + m[0, 1] * yc + self.cx + self.tx, m[1, 0] * xc + m[1, 1] * yc + self.cy + self.ty)

    def inverse_apply(self, x, y):
        m = np.linalg.inv(self._mat())
        xc = np.asarray(x, np.float64) - self.cx - self.tx
        yc = np.asarray(y, np.float64) - self.cy - self.ty
        return (m[0, 0] * xc + m[0, 1] * yc + self.cx, m[1, 0] * xc + m[1, 1] * yc + self.cy)


@dataclasses.dataclass
class Scene:
    width: int
    height: int
    blob_c: np.ndarray  # (n, 2)
    blob_sigma: np.ndarray  # (n,)
    blob_amp: np.ndarray  # (n,)
    noise_cells: list  # per octave: (cell_px, lattice values (ny, nx), amplitude)

    @staticmethod
    def draw(seed: int, width: int, height: int, n_blobs: int = 400) -> "Scene":
        rng = np.random.default_rng(seed)
        cx = rng.uniform(-_MARGIN, width + _MARGIN, n_blobs)
        cy = rng.uniform(-_MARGIN, height + _MARGIN, n_blobs)
        sigma = rng.uniform(2.0, 20.0, n_blobs)
        amp = rng.uniform(-60.0, 60.0, n_blobs)
        cells = []
        cell, a = 64.0, 16.0
        for _ in range(4):
            nx = int(math.ceil((width + 2 * _MARGIN) / cell)) + 2
            ny = int(math.ceil((height + 2 * _MARGIN) / cell)) + 2
            cells.append((cell, rng.uniform(-1.0, 1.0, (ny, nx)), a))
            cell, a = cell / 2.0, a / 2.0
        return Scene(width, height, np.stack([cx, cy], 1), sigma, amp, cells)

    def _value_noise(self, x, y):
        out = np.zeros_like(x)
        for cell, lat, a in self.noise_cells:
            u = (x + _MARGIN) / cell
            v = (y + _MARGIN) / cell
            i = np.clip(np.floor(u).astype(np.int64), 0, lat.shape[1] - 2)
            j = np.clip(np.floor(v).astype(np.int64), 0, lat.shape[0] - 2)
            fu = np.clip(u - i, 0.0, 1.0)
            fv = np.clip(v - j, 0.0, 1.0)
            fu = fu * fu * fu * (fu * (fu * 6 - 15) + 10)
            fv = fv * fv * fv * (fv * (fv * 6 - 15) + 10)
            top = lat[j, i] * (1 - fu) + lat[j, i + 1] * fu
            bot = lat[j + 1, i] * (1 - fu) + lat[j + 1, i + 1] * fu
            out += a * (top * (1 - fv) + bot * fv)
        return out

    def render(self, warp: Similarity | None = None, disparity: np.ndarray | None = None) -> np.ndarray:
        """Float64 intensity of the frame seen through `warp` (and an optional per-pixel
        horizontal disparity, for a rectified right camera)."""
        w, h = self.width, self.height
        ys, xs = np.mgrid[0:h, 0:w].astype(np.float64)
        if disparity is not None:
            xs = xs + disparity
        if warp is None:
            sx, sy, scale = xs, ys, 1.0
            centres, sig = self.blob_c, self.blob_sigma
        else:
            sx, sy = warp.inverse_apply(xs, ys)
            scale = warp.scale
            cxw, cyw = warp.apply(self.blob_c[:, 0], self.blob_c[:, 1])
            centres, sig = np.stack([cxw, cyw], 1), self.blob_sigma * scale
        img = 128.0 + self._value_noise(sx, sy)
        if disparity is not None:
            # Disparity shifts the sampling grid; render blobs through the same grid.
            for (bx, by), s, a in zip(self.blob_c, self.blob_sigma, self.blob_amp):
                r = 4.0 * s
                y0, y1 = max(int(by - r), 0), min(int(by + r) + 1, h)
                if y0 >= y1:
                    continue
                dx = xs[y0:y1] - bx
                dy = ys[y0:y1] - by
                img[y0:y1] += a * np.exp(-(dx * dx + dy * dy) / (2 * s * s))
            return img
        for (bx, by), s, a in zip(centres, sig, self.blob_amp):
            r = 4.0 * s
            x0, x1 = max(int(bx - r), 0), min(int(bx + r) + 1, w)
            y0, y1 = max(int(by - r), 0), min(int(by + r) + 1, h)
            if x0 >= x1 or y0 >= y1:
                continue
            dx = np.arange(x0, x1, dtype=np.float64) - bx
            dy = np.arange(y0, y1, dtype=np.float64) - by
            img[y0:y1, x0:x1] += a * np.exp(-(dy[:, None] ** 2 + dx[None, :] ** 2) / (2 * s * s))
        return img


def quantise(img: np.ndarray, rng: np.random.Generator | None = None, noise_sigma: float = 0.0) -> np.ndarray:
    if noise_sigma > 0.0:
        img = img + rng.normal(0.0, noise_sigma, img.shape)
    return np.clip(np.rint(img), 0, 255).astype(np.uint8)


def draw_similarity(seed: int, width: int, height: int, t_sigma: float = 2.0, rot_deg: float = 1.0,
                    scale_range: float = 0.01, t_uniform: float | None = None) -> Similarity:
    """Similarity warp about the frame centre: t ~ N(0, t_sigma) per axis (or U(-t_uniform, t_uniform)),
    theta ~ U(-rot_deg, rot_deg) degrees, s ~ U(1 - scale_range, 1 + scale_range)."""
    rng = np.random.default_rng(seed)
    if t_uniform is None:
        tx, ty = rng.normal(0.0, t_sigma, 2)
    else:
        tx, ty = rng.uniform(-t_uniform, t_uniform, 2)
    theta = math.radians(rng.uniform(-rot_deg, rot_deg))
    s = rng.uniform(1.0 - scale_range, 1.0 + scale_range)
    return Similarity(theta, s, float(tx), float(ty), (width - 1) / 2.0, (height - 1) / 2.0)


def frame_pair(camera_id: int, width: int, height: int, frame: int = 1):
    """Base frame and its warped successor for one camera (scene seed 1000 + camera id,
    warp seed 2000 + frame).  Returns (prev_u8, next_u8, warp)."""
    scene = Scene.draw(1000 + camera_id, width, height)
    prev = quantise(scene.render())
    warp = draw_similarity(2000 + frame + 7919 * camera_id, width, height)
    rng = np.random.default_rng(3000 + frame + 7919 * camera_id)
    nxt = quantise(scene.render(warp), rng, 2.0)
    return prev, nxt, warp


def stereo_right(camera_id: int, width: int, height: int) -> np.ndarray:
    """Rectified right image: the base frame resampled at x + d(x, y), d a smoothed U(5, 40) px field."""
    scene = Scene.draw(1000 + camera_id, width, height)
    rng = np.random.default_rng(4000 + camera_id)
    cell = 32.0
    lat = rng.uniform(5.0, 40.0, (int(height / cell) + 3, int(width / cell) + 3))
    ys, xs = np.mgrid[0:height, 0:width].astype(np.float64)
    u, v = xs / cell, ys / cell
    i, j = np.floor(u).astype(np.int64), np.floor(v).astype(np.int64)
    fu, fv = u - i, v - j
    fu = fu * fu * (3 - 2 * fu)
    fv = fv * fv * (3 - 2 * fv)
    d = (lat[j, i] * (1 - fu) + lat[j, i + 1] * fu) * (1 - fv) + (lat[j + 1, i] * (1 - fu) + lat[j + 1, i + 1] * fu) * fv
    rng2 = np.random.default_rng(5000 + camera_id)
    return quantise(scene.render(disparity=d), rng2, 2.0)


def sequence_frame(camera_id: int, width: int, height: int, frame: int):
    """Frame `frame` of a sequence: the base scene seen through its own similarity pose
    (t ~ U(-15, 15) px per axis, theta ~ U(-1.5, 1.5) deg), so consecutive frames differ by up to
    30 px and 3 deg.  Frame 0 is the unwarped base.  Returns (u8 image, pose)."""
    scene = Scene.draw(1000 + camera_id, width, height)
    if frame == 0:
        return quantise(scene.render()), Similarity(cx=(width - 1) / 2.0, cy=(height - 1) / 2.0)
    pose = draw_similarity(2000 + frame + 7919 * camera_id, width, height, rot_deg=1.5, t_uniform=15.0)
    rng = np.random.default_rng(3000 + frame + 7919 * camera_id)
    return quantise(scene.render(pose), rng, 2.0), pose


def flow_texture(warp: Similarity, u: np.ndarray) -> np.ndarray:
    """Ground-truth position, in the warped frame, of texture-coordinate points u (n, 2) of the base frame."""
    x, y = warp.apply(u[:, 0] - 0.5, u[:, 1] - 0.5)
    return np.stack([x + 0.5, y + 0.5], 1)


# Mixed-resolution 32-camera rig: 12 x 640x480, 12 x 1280x720, 8 x 1920x1200.
MULTICAM_SHAPES = [(640, 480)] * 12 + [(1280, 720)] * 12 + [(1920, 1200)] * 8


def multicam_feature_counts(seed: int = 77) -> list:
    rng = np.random.default_rng(seed)
    return [int(v) for v in rng.integers(300, 3001, len(MULTICAM_SHAPES))]
