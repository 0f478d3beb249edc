"""Host-side mirror of the cuVSLAM GPU front-end interface over the C ABI.

The classes keep the method names, argument meaning and error behaviour of the reference host
wrappers that MonoSOFGPU calls (libs/cuda_modules):
  ImagePyramid.build                         GaussianGPUImagePyramid::build (image_pyramid.h:81-98)
                                             + GPUGradientPyramid::set (gradient_pyramid.cpp:83-118)
  Selection.compute_gftt_and_select_features GPUSelection::computeGFTTAndSelectFeatures
                                             (selection_v2.cpp:27-184)
  LKFeatureTracker.track_points              GPULKFeatureTracker::track_points (lk_tracker.cpp:24-73)
Device memory comes from PyTorch (plumbing only); every computation runs in libcuvslam_fe.so.
"""

import ctypes

import numpy as np
import torch

from . import _lib
from .types import TRACK_DTYPE


# LK's default sampling: the texture unit's own linear filtering, as the reference samples its
# pyramid planes (lk_tracker.cu's tex2D reads).  FE_SAMPLE_TEXTURE restates that filtering in FP32
# and equals the oracle bit for bit; FE_SAMPLE_HARDWARE is the faster kernel.
DEFAULT_LK_SAMPLING = _lib.FE_SAMPLE_HARDWARE


def _stream_handle(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


class Context:
    """Owns the library's per-device scratch (fe_create / fe_destroy): the per-wrapper state of
    GPUSelection and GPULKFeatureTracker (selection_v2.h:28-58, lk_tracker.h:27-37)."""

    def __init__(self, device=0):
        self.lib = _lib.load()
        self.device = torch.device("cuda", device) if isinstance(device, int) else torch.device(device)
        torch.cuda.set_device(self.device)
        h = ctypes.c_void_p()
        _lib.check(self.lib.fe_create(self.device.index or 0, ctypes.byref(h)), "fe_create")
        self.handle = h

    def device_status(self, stream=None):
        """Synchronises `stream`, then reads and clears the device flags of this context's kernels
        (fe_device_status): 0 when no bounded wait ran out.  Raises FeError on a device fault."""
        flags = ctypes.c_int32(0)
        st = None if stream is None else ctypes.c_void_p(stream.cuda_stream)
        rc = self.lib.fe_device_status(self.handle, st, ctypes.byref(flags))
        if rc == _lib.FE_ERR_DEVICE_FAULT:
            raise _lib.FeError(f"device fault: flags {flags.value:#x} (a bounded wait ran out)")
        _lib.check(rc, "fe_device_status")
        return flags.value

    def set_wait_limit(self, iterations):
        """Iteration limit of the pyramid's bounded waits for launches planned from now on."""
        _lib.check(self.lib.fe_set_wait_limit(self.handle, int(iterations)), "fe_set_wait_limit")

    def close(self):
        if getattr(self, "handle", None):
            self.lib.fe_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ImagePyramid:
    """Image pyramid + gradient pyramid in one device buffer (fe_pyramid): GaussianGPUImagePyramid +
    GPUGradientPyramid (image_pyramid.h:56-162, gradient_pyramid.h:30-59)."""

    def __init__(self, width, height, max_levels=10, device="cuda"):
        lib = _lib.load()
        self.width, self.height = int(width), int(height)
        nbytes = lib.fe_pyramid_bytes(self.width, self.height, max_levels)
        if nbytes <= 0:
            raise ValueError(f"bad pyramid size {width}x{height}")
        self.storage = torch.empty(nbytes, dtype=torch.uint8, device=device)
        self.desc = _lib.FePyramid()
        _lib.check(lib.fe_pyramid_init(_ptr(self.storage), nbytes, self.width, self.height, max_levels,
                                       ctypes.byref(self.desc)), "fe_pyramid_init")
        self._f32 = self.storage.view(torch.float32)

    @property
    def levels(self):
        return self.desc.levels

    def level_size(self, l):
        return self.desc.width[l], self.desc.height[l]

    def _plane(self, ptr, l):
        off = (ptr - self.storage.data_ptr()) // 4
        w, h = self.desc.width[l], self.desc.height[l]
        return self._f32.as_strided((h, w), (self.desc.pitch_bytes[l] // 4, 1), off)

    def image(self, l):
        return self._plane(self.desc.image[l], l)

    def grad_x(self, l):
        return self._plane(self.desc.grad_x[l], l)

    def grad_y(self, l):
        return self._plane(self.desc.grad_y[l], l)

    def build(self, ctx, image_u8, blur_filter=False, stream=None):
        """Builds all levels and gradients from a (height, width) uint8 mono or (height, width, 3)
        uint8 RGB CUDA tensor; blur_filter applies the box prefilter first (the reference's
        GaussianGPUImagePyramid::build(image, blur_filter))."""
        img = image_u8
        if img.dtype != torch.uint8 or img.dim() not in (2, 3) or not img.is_cuda or \
                (img.dim() == 3 and img.shape[2] != 3):
            raise ValueError("image must be a (h, w) or (h, w, 3) uint8 CUDA tensor")
        if img.dim() == 3:
            if img.stride(2) != 1 or img.stride(1) != 3:
                img = img.contiguous()
            h, w, _ = img.shape
            _lib.check(ctx.lib.fe_build_pyramid_rgb(ctx.handle, _ptr(img), img.stride(0), w, h, int(bool(blur_filter)),
                                                    ctypes.byref(self.desc), _stream_handle(stream)),
                       "fe_build_pyramid_rgb")
            return self
        if img.stride(1) != 1:
            img = img.contiguous()
        h, w = img.shape
        _lib.check(ctx.lib.fe_build_pyramid(ctx.handle, _ptr(img), img.stride(0), w, h, int(bool(blur_filter)),
                                            ctypes.byref(self.desc), _stream_handle(stream)), "fe_build_pyramid")
        return self

    def build_f32(self, ctx, image_f32, stream=None):
        img = image_f32
        if img.dtype != torch.float32 or img.dim() != 2 or not img.is_cuda:
            raise ValueError("image must be a 2-D float32 CUDA tensor")
        if img.stride(1) != 1:
            img = img.contiguous()
        h, w = img.shape
        _lib.check(ctx.lib.fe_build_pyramid_f32(ctx.handle, _ptr(img), img.stride(0) * 4, w, h,
                                                ctypes.byref(self.desc), _stream_handle(stream)),
                   "fe_build_pyramid_f32")
        return self

    def to_numpy(self):
        """[(image, grad_x, grad_y)] per level as host arrays."""
        return [(self.image(l).cpu().numpy(), self.grad_x(l).cpu().numpy(), self.grad_y(l).cpu().numpy())
                for l in range(self.levels)]


def track_mono(ctx, prev, cur, tracks, retrack_ncc=0.85, sampling=DEFAULT_LK_SAMPLING, stream=None):
    """MonoSOFGPU::launch's track + retrack passes as collect merges them (fe_track_mono;
    sof_mono_gpu.cpp:34-104)."""
    _lib.check(ctx.lib.fe_track_mono(ctx.handle, ctypes.byref(prev.desc), ctypes.byref(cur.desc), _ptr(tracks),
                                     tracks.shape[0], ctypes.c_float(retrack_ncc), int(sampling),
                                     _stream_handle(stream)), "fe_track_mono")


def tracks_to_device(tracks, device="cuda"):
    """TRACK_DTYPE records -> (n, 80) uint8 CUDA tensor (the TrackData array the kernels update,
    cuda_kernels.h:76-87)."""
    arr = np.ascontiguousarray(tracks, dtype=TRACK_DTYPE)
    return torch.from_numpy(arr.view(np.uint8).reshape(len(arr), 80).copy()).to(device)


def tracks_from_device(t):
    return t.cpu().numpy().reshape(-1).view(TRACK_DTYPE).copy()


class LKFeatureTracker:
    """GPULKFeatureTracker (horizontal=False) / GPULKTrackerHorizontal (horizontal=True):
    track_points of cuda_modules/lk_tracker.cpp:24-73 (kernels lk_tracker.cu:69-379, 381-665)."""

    def __init__(self, ctx, horizontal=False, sampling=DEFAULT_LK_SAMPLING):
        self.ctx = ctx
        self.horizontal = bool(horizontal)
        self.sampling = sampling

    def track_points(self, previous_image_pyramid, current_image_pyramid, track_data, num_tracks=None,
                     stream=None):
        """Advances `track_data` ((n, 80) uint8 CUDA tensor of TrackData) in place; asynchronous."""
        n = track_data.shape[0] if num_tracks is None else int(num_tracks)
        if n == 0:
            return True
        if track_data.dtype != torch.uint8 or track_data.dim() != 2 or track_data.shape[1] != 80:
            raise ValueError("track_data must be an (n, 80) uint8 tensor of TrackData records")
        _lib.check(self.ctx.lib.fe_track(self.ctx.handle, ctypes.byref(previous_image_pyramid.desc),
                                         ctypes.byref(current_image_pyramid.desc), _ptr(track_data), n,
                                         int(self.horizontal), int(self.sampling), _stream_handle(stream)),
                   "fe_track")
        return True


AFFINE_CACHE_BYTES = 81 * 10 * 4 + 10 * 4 + 4  # fe_affine_cache (PointCacheData<float, 9>)


def _check_tracks(track_data):
    if track_data.dtype != torch.uint8 or track_data.dim() != 2 or track_data.shape[1] != 80:
        raise ValueError("track_data must be an (n, 80) uint8 tensor of TrackData records")


class STFeatureTracker:
    """GPUSTFeatureTracker (cuda_modules/st_tracker.cpp:22-78): affine tracking, previous patches
    sampled from the previous pyramid.  The reference tracker is built with (0, 20)."""

    def __init__(self, ctx, n_shift_only_iterations=0, n_full_mapping_iterations=20,
                 sampling=_lib.FE_SAMPLE_TEXTURE):
        self.ctx = ctx
        self.n_shift = int(n_shift_only_iterations)
        self.n_full = int(n_full_mapping_iterations)
        self.sampling = sampling

    def track_points(self, previous_image_pyramid, current_image_pyramid, track_data, num_tracks=None,
                     stream=None):
        """Advances `track_data` ((n, 80) uint8 CUDA tensor) in place; asynchronous.  The current
        pyramid supplies the image and both gradients."""
        n = track_data.shape[0] if num_tracks is None else int(num_tracks)
        if n == 0:
            return True
        _check_tracks(track_data)
        _lib.check(self.ctx.lib.fe_track_affine(self.ctx.handle, ctypes.byref(previous_image_pyramid.desc),
                                                ctypes.byref(current_image_pyramid.desc), _ptr(track_data), n,
                                                self.n_shift, self.n_full, int(self.sampling),
                                                _stream_handle(stream)), "fe_track_affine")
        return True


class STFeatureTrackerWithCache(STFeatureTracker):
    """GPUSTFeatureTrackerWithCache (cuda_modules/st_tracker.cpp:80-160): previous patches built
    once into a cache ((n, AFFINE_CACHE_BYTES) uint8 tensor), then tracked against it."""

    def build_points_cache(self, previous_image_pyramid, track_data, cache_data=None, num_tracks=None, stream=None):
        """Fills cache_data[i] from track i and sets its cache_index = i; returns the cache."""
        n = track_data.shape[0] if num_tracks is None else int(num_tracks)
        if cache_data is None:
            cache_data = torch.zeros((max(n, 1), AFFINE_CACHE_BYTES), dtype=torch.uint8, device=track_data.device)
        if n == 0:
            return cache_data
        _check_tracks(track_data)
        if cache_data.dtype != torch.uint8 or cache_data.dim() != 2 or cache_data.shape[1] != AFFINE_CACHE_BYTES \
                or cache_data.shape[0] < n:
            raise ValueError(f"cache_data must be an (>= n, {AFFINE_CACHE_BYTES}) uint8 tensor")
        _lib.check(self.ctx.lib.fe_affine_build_cache(self.ctx.handle, ctypes.byref(previous_image_pyramid.desc),
                                                      _ptr(track_data), n, _ptr(cache_data), int(self.sampling),
                                                      _stream_handle(stream)), "fe_affine_build_cache")
        return cache_data

    def track_points(self, current_image_pyramid, cache_data, track_data, num_tracks=None, stream=None):
        n = track_data.shape[0] if num_tracks is None else int(num_tracks)
        if n == 0:
            return True
        _check_tracks(track_data)
        if cache_data.dtype != torch.uint8 or cache_data.dim() != 2 or cache_data.shape[1] != AFFINE_CACHE_BYTES:
            raise ValueError(f"cache_data must be an (m, {AFFINE_CACHE_BYTES}) uint8 tensor")
        _lib.check(self.ctx.lib.fe_track_affine_cached(self.ctx.handle, ctypes.byref(current_image_pyramid.desc),
                                                       _ptr(cache_data), cache_data.shape[0], _ptr(track_data), n,
                                                       self.n_shift, self.n_full, int(self.sampling),
                                                       _stream_handle(stream)), "fe_track_affine_cached")
        return True


class Selection:
    """GPUSelection: Shi-Tomasi response + deterministic feature selection on pyramid level 0
    (computeGFTTAndSelectFeatures, selection_v2.cpp:27-184)."""

    def __init__(self, ctx):
        self.ctx = ctx
        self._count = torch.zeros(1, dtype=torch.int32, device=ctx.device)

    def select_async(self, pyramid, border_top, border_bottom, border_left, border_right, mask, alive_features,
                     num_desired, stream=None):
        """Enqueues selection; returns (xy (num_desired, 2) tensor, count (1,) int32 tensor)."""
        out = torch.empty((max(int(num_desired), 1), 2), dtype=torch.float32, device=self.ctx.device)
        count = torch.zeros(1, dtype=torch.int32, device=self.ctx.device)
        alive = None
        n_alive = 0
        if alive_features is not None and len(alive_features) > 0:
            alive = torch.as_tensor(alive_features, dtype=torch.float32).reshape(-1, 2).to(self.ctx.device).contiguous()
            n_alive = alive.shape[0]
        m = None
        if mask is not None:
            m = torch.as_tensor(mask, dtype=torch.uint8).to(self.ctx.device).contiguous()
        _lib.check(self.ctx.lib.fe_select(self.ctx.handle, ctypes.byref(pyramid.desc), int(border_top),
                                          int(border_bottom), int(border_left), int(border_right),
                                          None if m is None else _ptr(m), 0 if m is None else m.stride(0),
                                          None if alive is None else _ptr(alive), n_alive, int(num_desired),
                                          _ptr(out), _ptr(count), _stream_handle(stream)), "fe_select")
        self._keep = (alive, m)
        return out, count

    def compute_gftt_and_select_features(self, pyramid, border_top, border_bottom, border_left, border_right,
                                         input_mask, alive_features, num_desired_new_features, stream=None):
        """Blocking form with the reference's signature: returns the new features as an (k, 2) tensor."""
        out, count = self.select_async(pyramid, border_top, border_bottom, border_left, border_right, input_mask,
                                       alive_features, num_desired_new_features, stream)
        (stream or torch.cuda.current_stream()).synchronize()
        return out[: int(count.item())]

    def debug_maps(self, width, height):
        """(response, nms) maps of the last selection as (height, width) float32 CUDA tensors; the
        context must have been created with CUVSLAM_FE_DEBUG_MAPS set in the environment."""
        r, n = ctypes.c_void_p(), ctypes.c_void_p()
        _lib.check(self.ctx.lib.fe_select_debug(self.ctx.handle, ctypes.byref(r), ctypes.byref(n)), "fe_select_debug")
        return (torch.as_tensor(_DeviceArray(r.value, (height, width)), device=self.ctx.device),
                torch.as_tensor(_DeviceArray(n.value, (height, width)), device=self.ctx.device))


class _DeviceArray:
    """A float32 device buffer owned by the library, exposed through __cuda_array_interface__."""

    def __init__(self, ptr, shape):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": "<f4", "data": (int(ptr), False),
                                         "version": 2, "strides": None}


class TrackFinish:
    """MonoSOFGPU's retrack pass and finish filters for one camera (fe_track_finish;
    sof_mono_gpu.cpp:80-104,144-208, sof_mono_base.cpp:40-125).  age: (n,)
    int32/uint32 CUDA tensor of track ages (0 = dead), updated in place; predicted: optional (n, 2)
    float32 CUDA tensor (NaN = no prediction); mask: optional (h, w) uint8 CUDA tensor."""

    def __init__(self, age, retrack_ncc=0.85, predicted=None, mask=None, collapse=True):
        self.age = age
        self.retrack_ncc = float(retrack_ncc)
        self.predicted = predicted.contiguous() if predicted is not None else None
        self.mask = mask.contiguous() if mask is not None else None
        self.collapse = bool(collapse)
        self.alive_count = torch.zeros(1, dtype=torch.int32, device=age.device)

    def desc(self):
        d = _lib.FeTrackFinish()
        d.retrack_ncc = self.retrack_ncc
        d.age = self.age.data_ptr()
        d.predicted = self.predicted.data_ptr() if self.predicted is not None else None
        d.mask = self.mask.data_ptr() if self.mask is not None else None
        d.mask_pitch_bytes = self.mask.stride(0) if self.mask is not None else 0
        d.collapse = int(self.collapse)
        d.alive_count = self.alive_count.data_ptr()
        return d


def finish_tracks(ctx, tracks, finish, width, height, border=(0, 0, 0, 0), stream=None):
    """fe_finish_tracks for one camera: tracks is the (n, 80) uint8 TrackData tensor after LK."""
    c = (_lib.FeFinishCamera * 1)()
    c[0].tracks = tracks.data_ptr()
    c[0].n = tracks.shape[0]
    c[0].width, c[0].height = int(width), int(height)
    for k in range(4):
        c[0].border[k] = int(border[k])
    c[0].opts = finish.desc()
    _lib.check(ctx.lib.fe_finish_tracks(ctx.handle, c, 1, _stream_handle(stream)), "fe_finish_tracks")


class CameraFrame:
    """One camera of a batched frame step (fe_camera_frame); finish: optional TrackFinish.  No
    counterpart in the reference, which runs cameras one after another
    (MultiSOFBase::trackNextFrame, sof_multicamera_base.cpp:62-116)."""

    def __init__(self, image_u8, cur, prev=None, tracks=None, num_desired=0, border=(0, 0, 0, 0), finish=None):
        self.image = image_u8.contiguous()
        self.cur = cur
        self.prev = prev
        self.tracks = tracks
        self.num_desired = int(num_desired)
        self.border = tuple(int(b) for b in border)
        self.finish = finish
        dev = image_u8.device
        self.new_xy = torch.zeros((max(self.num_desired, 1), 2), dtype=torch.float32, device=dev)
        self.new_count = torch.zeros(1, dtype=torch.int32, device=dev)


class Batch:
    """Batched multi-camera frame step captured in a CUDA graph (fe_batch_*); no counterpart in the
    reference (sof_multicamera_base.cpp:62-116 loops over the cameras)."""

    def __init__(self, ctx, frames, sampling=DEFAULT_LK_SAMPLING):
        self.ctx = ctx
        self.frames = list(frames)
        arr = (_lib.FeCameraFrame * len(self.frames))()
        self._finish_descs = []
        for i, f in enumerate(self.frames):
            a = arr[i]
            a.image = f.image.data_ptr()
            a.image_pitch_bytes = f.image.stride(0)
            a.height, a.width = f.image.shape
            a.prev = ctypes.pointer(f.prev.desc) if f.prev is not None else None
            a.cur = ctypes.pointer(f.cur.desc)
            a.tracks = f.tracks.data_ptr() if f.tracks is not None else None
            a.n_tracks = f.tracks.shape[0] if f.tracks is not None else 0
            a.num_desired = f.num_desired
            a.new_xy = f.new_xy.data_ptr()
            a.new_count = f.new_count.data_ptr()
            for k in range(4):
                a.border[k] = f.border[k]
            if f.finish is not None:
                d = f.finish.desc()
                self._finish_descs.append(d)
                a.finish = ctypes.pointer(d)
        h = ctypes.c_void_p()
        _lib.check(ctx.lib.fe_batch_create(ctx.handle, arr, len(self.frames), int(sampling), ctypes.byref(h)),
                   "fe_batch_create")
        self.handle = h

    def run(self, stream=None):
        _lib.check(self.ctx.lib.fe_batch_run(self.handle, _stream_handle(stream)), "fe_batch_run")

    def run_part(self, part, stream=None):
        """part: 0 pyramids, 1 LK, 2 selection (enqueued directly, no graph)."""
        _lib.check(self.ctx.lib.fe_batch_run_part(self.handle, int(part), _stream_handle(stream)), "fe_batch_run_part")

    def kernel_count(self):
        return self.ctx.lib.fe_batch_kernel_count(self.handle)

    def lk_work(self, stream=None):
        """Runs the batch's LK part once with the kernel's work counters on (fe_batch_lk_work) and
        returns (levels set up, Gauss-Newton steps, NCC evaluations) summed over all tracks."""
        c = torch.zeros(3, dtype=torch.int64, device=self.ctx.device)
        _lib.check(self.ctx.lib.fe_batch_lk_work(self.handle, _ptr(c), _stream_handle(stream)), "fe_batch_lk_work")
        (stream or torch.cuda.current_stream()).synchronize()
        return tuple(int(v) for v in c.cpu())

    def autotune(self, reps=10, stream=None):
        """Chooses the LK block shape, the response-tile overlap and the pyramid stage tile by
        timing the step (fe_batch_autotune); returns the chosen shapes."""
        _lib.check(self.ctx.lib.fe_batch_autotune(self.handle, int(reps), _stream_handle(stream)), "fe_batch_autotune")
        return self.tuning()

    OVERLAP = ["after LK", "beside LK", "beside deep pyramid stages and LK", "before LK", "after LK and the burn"]

    def set_tuning(self, lk_block="8x4", response_overlap="beside LK", stage_tile=8, l012_ctas_per_sm=2):
        shape = ["8x4", "8x3", "4x8", "12x2"].index(lk_block)
        tile = int(stage_tile) | (64 if int(l012_ctas_per_sm) == 3 else 0)
        _lib.check(self.ctx.lib.fe_batch_set_tuning(self.handle, shape, self.OVERLAP.index(response_overlap), tile),
                   "fe_batch_set_tuning")

    def tuning(self):
        v = [ctypes.c_int32() for _ in range(3)]
        _lib.check(self.ctx.lib.fe_batch_tuning(self.handle, *[ctypes.byref(x) for x in v]), "fe_batch_tuning")
        shapes = ["8x4", "8x3", "4x8", "12x2"]
        return {"lk_block": shapes[v[0].value], "response_overlap": self.OVERLAP[v[1].value],
                "stage_tile": v[2].value & 31, "l012_ctas_per_sm": 3 if v[2].value & 64 else 2}

    def run_plain(self, stream=None):
        _lib.check(self.ctx.lib.fe_batch_run_plain(self.handle, _stream_handle(stream)), "fe_batch_run_plain")

    def close(self):
        if getattr(self, "handle", None):
            self.ctx.lib.fe_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
