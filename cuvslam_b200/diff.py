"""Differentiable LK tracking: the fe_adjoint_* plan of the C ABI and a torch.autograd.Function.

The forward is the reference tracker with exact bilinear sampling and one of two iteration rules
(include/cuvslam_fe.h, "Differentiable LK"); the backward is the hand-written adjoint kernel
(implicit-function theorem at the converged level-0 displacement, or unrolled iterations with
patches re-sampled from the pyramids).  The reference tracker works at uint8 intensity scale (its
Hessian carries +1 on the diagonal), so images given in [0, 1] are scaled by `intensity_scale`
(255) into the pyramids; gradients are returned with respect to the images as given.
"""

import ctypes

import numpy as np
import torch

from . import _lib
from .frontend import ImagePyramid, _ptr, _stream_handle
from .types import make_tracks

IMPLICIT = _lib.FE_ADJOINT_IMPLICIT
UNROLLED = _lib.FE_ADJOINT_UNROLLED
_MODES = {"implicit": IMPLICIT, "unrolled": UNROLLED, IMPLICIT: IMPLICIT, UNROLLED: UNROLLED}


class DiffTracker:
    """Differentiable LK over `batch` cameras of one size with `n_tracks` tracks each (no counterpart
    in the reference, which has no backward).

    Owns the frames (`prev_img`, `cur_img`, as given: the intensity scale is applied inside the
    pyramid build), the pyramids, the track records and the gradient buffers, and one fe_adjoint
    plan over them (so forward and backward allocate nothing and can be captured in a CUDA graph).  One
    forward may be outstanding per tracker: a second forward overwrites the saved state.
    recompute_pyramids: the backward rebuilds the pyramids from the saved images instead of
    relying on the forward's (pyramids are then free to be reused between the two)."""

    def __init__(self, ctx, batch, height, width, n_tracks, mode="implicit", iterations=None, tolerance=1e-4,
                 intensity_scale=255.0, recompute_pyramids=False, search_radius=2048.0, ncc_threshold=0.8):
        self.ctx = ctx
        self.lib = ctx.lib
        self.mode = _MODES[mode]
        self.iterations = int(iterations if iterations is not None else (20 if self.mode == IMPLICIT else 10))
        self.tolerance = float(tolerance)
        self.scale = float(intensity_scale)
        self.recompute = bool(recompute_pyramids)
        self.B, self.H, self.W, self.N = int(batch), int(height), int(width), int(n_tracks)
        dev = ctx.device
        self.prev_pyr = [ImagePyramid(width, height, device=dev) for _ in range(self.B)]
        self.cur_pyr = [ImagePyramid(width, height, device=dev) for _ in range(self.B)]
        self.prev_img = torch.zeros((self.B, self.H, self.W), dtype=torch.float32, device=dev)
        self.cur_img = torch.zeros_like(self.prev_img)
        recs = make_tracks(np.zeros((self.B * self.N, 2), np.float32), None, search_radius, ncc_threshold)
        self.tracks_in = torch.from_numpy(recs.view(np.uint8).reshape(-1, 80).copy()).to(dev)
        self.tracks_out = self.tracks_in.clone()
        self.grad_xy = torch.zeros((self.B, self.N, 2), dtype=torch.float32, device=dev)
        self.grad_prev = torch.zeros((self.B, self.H, self.W), dtype=torch.float32, device=dev)
        self.grad_cur = torch.zeros_like(self.grad_prev)
        self.grad_track = torch.zeros((self.B, self.N, 2), dtype=torch.float32, device=dev)
        self.grad_offset = torch.zeros_like(self.grad_track)
        jobs = (_lib.FeAdjointJob * self.B)()
        for b in range(self.B):
            j = jobs[b]
            j.prev = ctypes.pointer(self.prev_pyr[b].desc)
            j.cur = ctypes.pointer(self.cur_pyr[b].desc)
            j.tracks_in = self.tracks_in.data_ptr() + b * self.N * 80
            j.tracks_out = self.tracks_out.data_ptr() + b * self.N * 80
            j.n_tracks = self.N
            j.grad_xy = self.grad_xy[b].data_ptr()
            j.grad_prev = self.grad_prev[b].data_ptr()
            j.grad_prev_pitch_bytes = self.W * 4
            j.grad_cur = self.grad_cur[b].data_ptr()
            j.grad_cur_pitch_bytes = self.W * 4
            j.grad_track = self.grad_track[b].data_ptr()
            j.grad_offset = self.grad_offset[b].data_ptr()
            j.prev_image = self.prev_img[b].data_ptr()
            j.cur_image = self.cur_img[b].data_ptr()
            j.image_pitch_bytes = self.W * 4
            j.image_scale = self.scale
        h = ctypes.c_void_p()
        _lib.check(self.lib.fe_adjoint_create(ctx.handle, jobs, self.B, self.mode, self.iterations,
                                              ctypes.c_float(self.tolerance), ctypes.byref(h)), "fe_adjoint_create")
        self.handle = h
        self._jobs = jobs
        self._fields_in = self.tracks_in.view(torch.float32).view(self.B, self.N, 20)
        self._fields_out = self.tracks_out.view(torch.float32).view(self.B, self.N, 20)

    # ---------------------------------------------------------------- steps
    def build_pyramids(self, stream=None):
        """Both pyramids of every camera from intensity_scale * the frames, in one batched build."""
        _lib.check(self.lib.fe_adjoint_build_pyramids(self.handle, _stream_handle(stream)), "fe_adjoint_build_pyramids")

    def set_inputs(self, prev, cur, xy, offset=None):
        """prev, cur: (B, H, W) float32 frames (used in place when they are the tracker's own
        `prev_img` / `cur_img` buffers, else copied there); xy, offset: (B, N, 2) track positions
        and initial displacement guesses."""
        if prev.data_ptr() != self.prev_img.data_ptr():
            self.prev_img.copy_(prev.detach())
        if cur.data_ptr() != self.cur_img.data_ptr():
            self.cur_img.copy_(cur.detach())
        self._fields_in[:, :, 0:2] = xy.detach()
        self._fields_in[:, :, 2:4] = 0.0 if offset is None else offset.detach()

    def forward_step(self, stream=None):
        _lib.check(self.lib.fe_adjoint_forward(self.handle, _stream_handle(stream)), "fe_adjoint_forward")

    def backward_step(self, stream=None):
        _lib.check(self.lib.fe_adjoint_backward(self.handle, _stream_handle(stream)), "fe_adjoint_backward")

    def outputs(self):
        """(positions (B, N, 2), status (B, N) bool) of the last forward."""
        st = self.tracks_out.view(self.B, self.N, 80)[:, :, 32] != 0
        return self._fields_out[:, :, 0:2], st

    def dropped(self):
        """Tracks of the last backward that got no gradient (unrolled iterates spread too far)."""
        out = torch.zeros(1, dtype=torch.int32, device=self.ctx.device)
        _lib.check(self.lib.fe_adjoint_dropped(self.handle, _ptr(out), _stream_handle()), "fe_adjoint_dropped")
        return int(out.item())

    def kernel_count(self, backward):
        return self.lib.fe_adjoint_kernel_count(self.handle, int(bool(backward)))

    def __call__(self, prev, cur, xy, offset=None):
        """Differentiable tracking: returns (positions (B, N, 2), status (B, N)); gradients flow to
        prev, cur, xy and offset."""
        if offset is None:
            offset = torch.zeros_like(xy)
        return _TrackFn.apply(self, prev, cur, xy, offset)

    def close(self):
        if getattr(self, "handle", None):
            self.lib.fe_adjoint_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class _TrackFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, tracker, prev, cur, xy, offset):
        tracker.set_inputs(prev, cur, xy, offset)
        tracker.build_pyramids()
        tracker.forward_step()
        pos, status = tracker.outputs()
        ctx.tracker = tracker
        ctx.mark_non_differentiable(status)
        return pos.clone(), status.clone()

    @staticmethod
    def backward(ctx, g_pos, g_status):
        t = ctx.tracker
        t.grad_xy.copy_(g_pos if g_pos is not None else torch.zeros_like(t.grad_xy))
        if t.recompute:
            t.build_pyramids()
        t.backward_step()
        s = t.scale
        return None, t.grad_prev * s, t.grad_cur * s, t.grad_track.clone(), t.grad_offset.clone()
