"""ctypes binding of libcuvslam_fe.so (the C ABI declared in include/cuvslam_fe.h).

The shared library is built in-tree by cuvslam_b200/csrc/Makefile (see cuvslam_b200.build).
There is no fallback: if the library is missing or fails to load, importing the front-end raises.
"""

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcuvslam_fe.so")
MAX_LEVELS = 10

FE_OK = 0
FE_ERR_INVALID_ARGUMENT = 1
FE_ERR_CUDA = 2
FE_ERR_OUT_OF_MEMORY = 3
FE_ERR_CAPACITY = 4
FE_ERR_DEVICE_FAULT = 5
FE_DEFAULT_WAIT_LIMIT = 1 << 22
FE_SAMPLE_TEXTURE = 0
FE_SAMPLE_EXACT = 1
FE_SAMPLE_TEXTURE_WIDE = 2
FE_SAMPLE_HARDWARE = 3


class FePyramid(ctypes.Structure):
    _fields_ = [
        ("levels", ctypes.c_int32),
        ("width", ctypes.c_int32 * MAX_LEVELS),
        ("height", ctypes.c_int32 * MAX_LEVELS),
        ("pitch_bytes", ctypes.c_int64 * MAX_LEVELS),
        ("image", ctypes.c_void_p * MAX_LEVELS),
        ("grad_x", ctypes.c_void_p * MAX_LEVELS),
        ("grad_y", ctypes.c_void_p * MAX_LEVELS),
    ]


class FeTrackFinish(ctypes.Structure):
    _fields_ = [
        ("retrack_ncc", ctypes.c_float),
        ("age", ctypes.c_void_p),
        ("predicted", ctypes.c_void_p),
        ("mask", ctypes.c_void_p),
        ("mask_pitch_bytes", ctypes.c_int64),
        ("collapse", ctypes.c_int32),
        ("alive_count", ctypes.c_void_p),
    ]


class FeFinishCamera(ctypes.Structure):
    _fields_ = [
        ("tracks", ctypes.c_void_p),
        ("n", ctypes.c_int32),
        ("width", ctypes.c_int32),
        ("height", ctypes.c_int32),
        ("border", ctypes.c_int32 * 4),
        ("opts", FeTrackFinish),
    ]


class FeCameraFrame(ctypes.Structure):
    _fields_ = [
        ("image", ctypes.c_void_p),
        ("image_pitch_bytes", ctypes.c_int64),
        ("width", ctypes.c_int32),
        ("height", ctypes.c_int32),
        ("prev", ctypes.POINTER(FePyramid)),
        ("cur", ctypes.POINTER(FePyramid)),
        ("tracks", ctypes.c_void_p),
        ("n_tracks", ctypes.c_int32),
        ("num_desired", ctypes.c_int32),
        ("new_xy", ctypes.c_void_p),
        ("new_count", ctypes.c_void_p),
        ("border", ctypes.c_int32 * 4),
        ("finish", ctypes.POINTER(FeTrackFinish)),
    ]


class FeAdjointJob(ctypes.Structure):
    _fields_ = [
        ("prev", ctypes.POINTER(FePyramid)),
        ("cur", ctypes.POINTER(FePyramid)),
        ("tracks_in", ctypes.c_void_p),
        ("tracks_out", ctypes.c_void_p),
        ("n_tracks", ctypes.c_int32),
        ("grad_xy", ctypes.c_void_p),
        ("grad_prev", ctypes.c_void_p),
        ("grad_prev_pitch_bytes", ctypes.c_int64),
        ("grad_cur", ctypes.c_void_p),
        ("grad_cur_pitch_bytes", ctypes.c_int64),
        ("grad_track", ctypes.c_void_p),
        ("grad_offset", ctypes.c_void_p),
        ("prev_image", ctypes.c_void_p),
        ("cur_image", ctypes.c_void_p),
        ("image_pitch_bytes", ctypes.c_int64),
        ("image_scale", ctypes.c_float),
    ]


FE_ADJOINT_IMPLICIT = 0
FE_ADJOINT_UNROLLED = 1


class FeEpipolarCurves(ctypes.Structure):
    _fields_ = [
        ("width", ctypes.c_int32),
        ("height", ctypes.c_int32),
        ("inv_scale", ctypes.c_float),
        ("offsets", ctypes.c_void_p),
        ("xy", ctypes.c_void_p),
        ("max_length", ctypes.c_int32),
    ]


class FeStereoPair(ctypes.Structure):
    _fields_ = [
        ("primary", ctypes.POINTER(FePyramid)),
        ("secondary", ctypes.POINTER(FePyramid)),
        ("uv", ctypes.c_void_p),
        ("valid", ctypes.c_void_p),
        ("n", ctypes.c_int32),
        ("cand_offsets", ctypes.c_void_p),
        ("cand_xy", ctypes.c_void_p),
        ("max_candidates", ctypes.c_int32),
        ("curves", ctypes.POINTER(FeEpipolarCurves)),
        ("search_radius", ctypes.c_float),
        ("ncc_threshold", ctypes.c_float),
        ("out", ctypes.c_void_p),
        ("winner", ctypes.c_void_p),
        ("stats", ctypes.c_void_p),
    ]


class FeError(RuntimeError):
    pass


_lib = None

# name -> (restype, argtypes)
_P = ctypes.c_void_p
_I = ctypes.c_int
_I64 = ctypes.c_int64
_SIGS = {
    "fe_abi_version": (_I, []),
    "fe_status_string": (ctypes.c_char_p, [_I]),
    "fe_last_cuda_error": (_I, []),
    "fe_create": (_I, [_I, ctypes.POINTER(_P)]),
    "fe_destroy": (_I, [_P]),
    "fe_device_status": (_I, [_P, _P, ctypes.POINTER(ctypes.c_int32)]),
    "fe_set_wait_limit": (_I, [_P, _I]),
    "fe_pyramid_levels": (_I, [_I, _I, _I]),
    "fe_pyramid_bytes": (_I64, [_I, _I, _I]),
    "fe_pyramid_init": (_I, [_P, _I64, _I, _I, _I, ctypes.POINTER(FePyramid)]),
    "fe_build_pyramid": (_I, [_P, _P, _I64, _I, _I, _I, ctypes.POINTER(FePyramid), _P]),
    "fe_build_pyramid_f32": (_I, [_P, _P, _I64, _I, _I, ctypes.POINTER(FePyramid), _P]),
    "fe_build_pyramid_rgb": (_I, [_P, _P, _I64, _I, _I, _I, ctypes.POINTER(FePyramid), _P]),
    "fe_select": (_I, [_P, ctypes.POINTER(FePyramid), _I, _I, _I, _I, _P, _I64, _P, _I, _I, _P, _P, _P]),
    "fe_select_noalloc": (_I, [ctypes.POINTER(FePyramid), _I, _I, _I, _I, _P, _I64, _P, _I, _I, _P, _P, _P]),
    "fe_select_debug": (_I, [_P, ctypes.POINTER(_P), ctypes.POINTER(_P)]),
    "fe_track": (_I, [_P, ctypes.POINTER(FePyramid), ctypes.POINTER(FePyramid), _P, _I, _I, _I, _P]),
    "fe_track_stereo": (_I, [_P, ctypes.POINTER(FeStereoPair), _I, ctypes.c_float, _I, _I, _P]),
    "fe_track_mono": (_I, [_P, ctypes.POINTER(FePyramid), ctypes.POINTER(FePyramid), _P, _I, ctypes.c_float, _I, _P]),
    "fe_finish_tracks": (_I, [_P, ctypes.POINTER(FeFinishCamera), _I, _P]),
    "fe_track_affine": (_I, [_P, ctypes.POINTER(FePyramid), ctypes.POINTER(FePyramid), _P, _I, _I, _I, _I, _P]),
    "fe_affine_build_cache": (_I, [_P, ctypes.POINTER(FePyramid), _P, _I, _P, _I, _P]),
    "fe_track_affine_cached": (_I, [_P, ctypes.POINTER(FePyramid), _P, _I, _P, _I, _I, _I, _I, _P]),
    "fe_batch_create": (_I, [_P, ctypes.POINTER(FeCameraFrame), _I, _I, ctypes.POINTER(_P)]),
    "fe_batch_run": (_I, [_P, _P]),
    "fe_batch_run_plain": (_I, [_P, _P]),
    "fe_batch_run_part": (_I, [_P, _I, _P]),
    "fe_batch_kernel_count": (_I, [_P]),
    "fe_batch_lk_work": (_I, [_P, _P, _P]),
    "fe_batch_autotune": (_I, [_P, _I, _P]),
    "fe_batch_tuning": (_I, [_P, _P, _P, _P]),
    "fe_batch_set_tuning": (_I, [_P, _I, _I, _I]),
    "fe_batch_destroy": (_I, [_P]),
    "fe_adjoint_create": (_I, [_P, ctypes.POINTER(FeAdjointJob), _I, _I, _I, ctypes.c_float, ctypes.POINTER(_P)]),
    "fe_adjoint_build_pyramids": (_I, [_P, _P]),
    "fe_adjoint_forward": (_I, [_P, _P]),
    "fe_adjoint_backward": (_I, [_P, _P]),
    "fe_adjoint_kernel_count": (_I, [_P, _I]),
    "fe_adjoint_dropped": (_I, [_P, _P, _P]),
    "fe_adjoint_destroy": (_I, [_P]),
    "fe_track_diff": (_I, [_P, ctypes.POINTER(FePyramid), ctypes.POINTER(FePyramid), _P, _P, _I, _I, _I,
                           ctypes.c_float, _P]),
    "fe_track_backward": (_I, [_P, ctypes.POINTER(FePyramid), ctypes.POINTER(FePyramid), _P, _P, _I, _I, _I,
                               ctypes.c_float, _P, _P, _I64, _P, _I64, _P, _P, _P]),
}

EXPORTED = tuple(_SIGS)


def load():
    """Loads libcuvslam_fe.so; raises if it is absent (no fallback path exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is not built; run `python -c 'import cuvslam_b200.build as b; b.build()'`")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def check(rc, what=""):
    if rc != FE_OK:
        lib = load()
        msg = lib.fe_status_string(rc).decode()
        raise FeError(f"{what}: {msg} (status {rc}, cuda error {lib.fe_last_cuda_error()})")
