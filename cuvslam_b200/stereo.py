"""Left-to-right (primary -> secondary camera) matching over the C ABI (fe_track_stereo).

Mirrors the reference's L2R step of MultiSOFGPU (libs/sof/sof_multicamera_gpu.cpp:69-190):
  EpipolarCurves                  the precomputed candidate table of one camera pair
                                  (libs/sof/epipolar_curves.h:26-64); `pinhole` builds it for two
                                  pinhole cameras as the EpipolarCurves constructor does
                                  (epipolar_curves.cpp:103-165)
  cross_cam_search_radius         MultiSOFBase::CrossCamSearchRadius (sof_multicamera_base.cpp:31-37)
  StereoMatcher.track_primary_to_secondary
                                  LaunchTrackingPrimaryToSecondary's candidate scan (lines 118-190),
                                  every camera pair of a rig in one launch and no host round trip
                                  per candidate
"""

import ctypes
from dataclasses import dataclass
from typing import Optional

import numpy as np
import torch

from . import _lib
from .frontend import ImagePyramid, _stream_handle

L2R_EARLY_EXIT_FRACTION = 0.8  # kL2REarlyExitFraction (libs/sof/internal/sof_multicamera_base.h:40)
L2R_NCC_THRESHOLD = 0.8        # ncc_threshold of every attempt (sof_multicamera_gpu.cpp:128)
NUM_DEPTH_SAMPLES = 50         # kNumDepthSamples (epipolar_curves.cpp:30)
MINIMUM_HITHER = 0.1           # FrustumProperties::MINIMUM_HITHER (libs/epipolar/near_plane.h:33)


def cross_cam_search_radius(top_level: int) -> float:
    """Search radius of the left-to-right attempts: 3 * 2^(top_level + 1) base-level pixels
    (CrossCamSearchRadius, sof_multicamera_base.cpp:31-37)."""
    return 3.0 * float(1 << (top_level + 1))


def auto_depth_range(baseline, min_depth=-1.0, max_depth=-1.0):
    """AutoDetectDepthRange (epipolar_curves.cpp:40-62): a finite negative bound is replaced by the
    value interpolated over the baseline between 7.5 cm (0.1 .. 20 m) and 0.5 m (7 .. 1000 m)."""
    t = min(max((baseline - 0.075) / (0.5 - 0.075), 0.0), 1.0)
    if np.isfinite(min_depth) and min_depth < 0:
        min_depth = 0.1 + t * (7.0 - 0.1)
    if np.isfinite(max_depth) and max_depth < 0:
        max_depth = 20.0 + t * (1000.0 - 20.0)
    if not (np.isfinite(min_depth) and np.isfinite(max_depth) and 0 < min_depth < max_depth):
        raise ValueError("EpipolarCurves: need finite 0 < min_depth < max_depth (negative = auto)")
    return float(min_depth), float(max_depth)


class EpipolarCurves:
    """Candidate table of one camera pair in device memory (fe_epipolar_curves; EpipolarCurves,
    epipolar_curves.h:26-64): for each corner (u, v) of the primary pyramid's top level,
    0 <= u <= top_width, 0 <= v <= top_height, a curve of secondary base-level positions, far to
    near."""

    def __init__(self, curves, top_level, device="cuda"):
        """curves[v][u]: sequence of (x, y) secondary base-level positions."""
        cw, ch, offsets, xy = curves_csr(curves)
        self.top_level = int(top_level)
        self.width, self.height = cw, ch
        self.inv_scale = 1.0 / float(1 << self.top_level)
        self.offsets_host = offsets
        self.xy_host = xy
        self.max_length = int(np.diff(offsets).max(initial=0))
        self.offsets = torch.from_numpy(offsets).to(device)
        self.xy = torch.from_numpy(xy if len(xy) else np.zeros((1, 2), np.float32)).to(device)
        self.desc = _lib.FeEpipolarCurves(cw, ch, self.inv_scale, self.offsets.data_ptr(), self.xy.data_ptr(),
                                          self.max_length)

    @classmethod
    def pinhole(cls, k_primary, k_secondary, secondary_from_primary, top_level, top_width, top_height,
                min_depth=-1.0, max_depth=-1.0, device="cuda"):
        """The table of two undistorted pinhole cameras (pinhole_curves) in device memory."""
        return cls(pinhole_curves(k_primary, k_secondary, secondary_from_primary, top_level, top_width, top_height,
                                  min_depth, max_depth), top_level, device)


def pinhole_curves(k_primary, k_secondary, secondary_from_primary, top_level, top_width, top_height,
                   min_depth=-1.0, max_depth=-1.0):
    """Corner curves (curves[v][u], lists of (x, y)) of two undistorted pinhole cameras, as the
    EpipolarCurves constructor builds them (epipolar_curves.cpp:103-165): k_* = (fx, fy, cx, cy);
    secondary_from_primary = (R 3x3, t 3), the rigid transform from primary to secondary camera
    coordinates.  Depths are sampled log-uniformly from max_depth down to min_depth along each
    corner's primary ray; a sample is kept when it lies in front of the secondary camera, inside its
    top level, and at least one top-level pixel from the last kept sample."""
    R = np.asarray(secondary_from_primary[0], np.float32).reshape(3, 3)
    t = np.asarray(secondary_from_primary[1], np.float32).reshape(3)
    min_depth, max_depth = auto_depth_range(float(np.linalg.norm(t)), min_depth, max_depth)
    scale = np.float32(1 << int(top_level))
    inv_scale = np.float32(1.0) / scale
    log_min, log_max = np.float32(np.log(min_depth)), np.float32(np.log(max_depth))
    log_step = (log_max - log_min) / np.float32(NUM_DEPTH_SAMPLES - 1)
    depths = np.exp(log_max - log_step * np.arange(NUM_DEPTH_SAMPLES, dtype=np.float32)).astype(np.float32)
    fx, fy, cx, cy = (np.float32(v) for v in k_primary)
    gx, gy, gcx, gcy = (np.float32(v) for v in k_secondary)
    curves = []
    for v in range(top_height + 1):
        row = []
        for u in range(top_width + 1):
            ray = np.array([(np.float32(u) * scale - cx) / fx, (np.float32(v) * scale - cy) / fy, 1.0], np.float32)
            p = (depths[:, None] * ray[None, :]) @ R.T + t[None, :]
            curve = []
            last_u, last_v = np.float32(-1e9), np.float32(-1e9)
            for s in range(NUM_DEPTH_SAMPLES):
                z = p[s, 2]
                if not z > MINIMUM_HITHER:
                    continue
                ur = (gx * (p[s, 0] / z) + gcx) * inv_scale
                vr = (gy * (p[s, 1] / z) + gcy) * inv_scale
                if ur < 0 or vr < 0 or ur >= top_width or vr >= top_height:
                    continue
                du, dv = ur - last_u, vr - last_v
                if du * du + dv * dv < 1.0:
                    continue
                last_u, last_v = ur, vr
                curve.append((float(ur * scale), float(vr * scale)))
            row.append(curve)
        curves.append(row)
    return curves


def curves_csr(curves):
    """(width, height, offsets (width*height + 1,) int32, xy (m, 2) float32) of curves[v][u]."""
    ch = len(curves)
    cw = len(curves[0]) if ch else 0
    lens = np.array([len(curves[v][u]) for v in range(ch) for u in range(cw)], np.int64)
    offsets = np.zeros(cw * ch + 1, np.int64)
    np.cumsum(lens, out=offsets[1:])
    if offsets[-1] >= 2**31:
        raise ValueError("epipolar table too large")
    xy = np.zeros((int(offsets[-1]), 2), np.float32)
    for v in range(ch):
        for u in range(cw):
            c = curves[v][u]
            if len(c):
                j = v * cw + u
                xy[offsets[j]:offsets[j + 1]] = np.asarray(c, np.float32).reshape(-1, 2)
    return cw, ch, offsets.astype(np.int32), xy


@dataclass
class StereoPair:
    """One primary -> secondary pair of a left-to-right match.  uv: (n, 2) float32 CUDA tensor of
    primary base-level positions; candidates either `curves` or explicit (cand_offsets (n + 1,)
    int32, cand_xy (m, 2) float32, max_candidates)."""
    primary: ImagePyramid
    secondary: ImagePyramid
    uv: torch.Tensor
    curves: Optional[EpipolarCurves] = None
    cand_offsets: Optional[torch.Tensor] = None
    cand_xy: Optional[torch.Tensor] = None
    max_candidates: int = 0
    valid: Optional[torch.Tensor] = None
    search_radius: Optional[float] = None
    ncc_threshold: float = L2R_NCC_THRESHOLD


class StereoMatcher:
    """fe_track_stereo over a fixed set of camera pairs; owns the output buffers.  Replaces
    MultiSOFGPU::LaunchTrackingPrimaryToSecondary (sof_multicamera_gpu.cpp:69-190)."""

    def __init__(self, ctx, sampling=_lib.FE_SAMPLE_TEXTURE, early_exit_fraction=L2R_EARLY_EXIT_FRACTION,
                 horizontal=True):
        """horizontal: the 1-D tracker of rectified pairs (lr_tracker = LKHorizontal), else 2-D LK
        (lr_tracker = LK, the reference's default)."""
        self.ctx = ctx
        self.sampling = int(sampling)
        self.frac = float(early_exit_fraction)
        self.horizontal = bool(horizontal)

    def track_primary_to_secondary(self, pairs, outputs=None, stream=None):
        """Matches every pair in one launch.  Returns [(tracks (n, 80) uint8 TrackData records,
        winner (n,) int32, stats (4,) int32)] per pair; `outputs` (the same list from an earlier
        call) is reused when given."""
        dev = self.ctx.device
        descs = (_lib.FeStereoPair * len(pairs))()
        keep = []
        if outputs is None:
            outputs = [(torch.empty((p.uv.shape[0], 80), dtype=torch.uint8, device=dev),
                        torch.empty(p.uv.shape[0], dtype=torch.int32, device=dev),
                        torch.empty(4, dtype=torch.int32, device=dev)) for p in pairs]
        for d, p, (out, win, st) in zip(descs, pairs, outputs):
            uv = p.uv.contiguous()
            if uv.dtype != torch.float32 or uv.dim() != 2 or uv.shape[1] != 2 or not uv.is_cuda:
                raise ValueError("uv must be an (n, 2) float32 CUDA tensor")
            keep.append(uv)
            d.primary = ctypes.pointer(p.primary.desc)
            d.secondary = ctypes.pointer(p.secondary.desc)
            d.uv = uv.data_ptr()
            d.n = uv.shape[0]
            if p.valid is not None:
                v = p.valid.to(torch.uint8).contiguous()
                keep.append(v)
                d.valid = v.data_ptr()
            if p.cand_offsets is not None:
                off = p.cand_offsets.to(torch.int32).contiguous()
                cxy = p.cand_xy.to(torch.float32).contiguous()
                keep += [off, cxy]
                d.cand_offsets = off.data_ptr()
                d.cand_xy = cxy.data_ptr()
                d.max_candidates = int(p.max_candidates)
            elif p.curves is not None:
                d.curves = ctypes.pointer(p.curves.desc)
            else:
                raise ValueError("a pair needs curves or explicit candidates")
            radius = p.search_radius if p.search_radius is not None else cross_cam_search_radius(p.primary.levels - 1)
            d.search_radius = float(radius)
            d.ncc_threshold = float(p.ncc_threshold)
            d.out = out.data_ptr()
            d.winner = win.data_ptr()
            d.stats = st.data_ptr()
        _lib.check(self.ctx.lib.fe_track_stereo(self.ctx.handle, descs, len(pairs), ctypes.c_float(self.frac),
                                                int(self.horizontal), self.sampling, _stream_handle(stream)),
                   "fe_track_stereo")
        self._keep = keep  # inputs stay alive until the next call (the launch is asynchronous)
        return outputs
