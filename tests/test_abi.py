"""The C ABI library: loads, exports every entry point include/cuvslam_fe.h declares, and its
host-only logic (level rule, layout, argument checking) behaves; no GPU compute is issued."""

import ctypes
import os
import re

import numpy as np
import pytest

from cuvslam_b200 import _lib
from cuvslam_b200.types import TRACK_DTYPE, level_sizes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "cuvslam_fe.h")).read()
    return sorted(set(re.findall(r"FE_API\s+[\w\s\*]+?\b(fe_\w+)\s*\(", src)))


def test_exports_every_declared_symbol():
    lib = _lib.load()
    names = _declared()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n
    assert sorted(_lib.EXPORTED) == names


def test_abi_version_and_status_strings():
    lib = _lib.load()
    assert lib.fe_abi_version() == 1
    assert lib.fe_status_string(0) == b"ok"
    assert lib.fe_status_string(4) == b"size limit exceeded"


@pytest.mark.parametrize("wh", [(752, 480), (1241, 376), (1280, 720), (1920, 1200), (640, 480), (31, 17), (15, 15),
                                (29, 29), (30, 30)])
def test_level_rule(wh, oracle):
    lib = _lib.load()
    w, h = wh
    for cap in (10, 4, 1):
        n = lib.fe_pyramid_levels(w, h, cap)
        assert n == len(level_sizes(w, h, cap)) == len(oracle.level_sizes(w, h, cap))
    assert lib.fe_pyramid_levels(752, 480, 10) == 6
    assert lib.fe_pyramid_levels(1920, 1200, 10) == 7
    assert lib.fe_pyramid_levels(1241, 376, 10) == 5


def test_pyramid_layout_host_only():
    lib = _lib.load()
    w, h = 752, 480
    nbytes = lib.fe_pyramid_bytes(w, h, 10)
    base = 1 << 20  # a fake 256-byte aligned device address: fe_pyramid_init never dereferences it
    d = _lib.FePyramid()
    assert lib.fe_pyramid_init(ctypes.c_void_p(base), nbytes, w, h, 10, ctypes.byref(d)) == 0
    assert d.levels == 6
    end = base
    for l, (lw, lh) in enumerate(level_sizes(w, h)):
        assert (d.width[l], d.height[l]) == (lw, lh)
        assert d.pitch_bytes[l] % 256 == 0 and d.pitch_bytes[l] >= lw * 4
        for p in (d.image[l], d.grad_x[l], d.grad_y[l]):
            assert p % 256 == 0 and p >= end
            end = p + d.pitch_bytes[l] * lh
    assert end <= base + nbytes
    # too small / misaligned
    assert lib.fe_pyramid_init(ctypes.c_void_p(base), nbytes - 1, w, h, 10, ctypes.byref(d)) == 1
    assert lib.fe_pyramid_init(ctypes.c_void_p(base + 16), nbytes, w, h, 10, ctypes.byref(d)) == 1


def test_argument_checks_need_no_device():
    lib = _lib.load()
    d = _lib.FePyramid()
    assert lib.fe_build_pyramid(None, None, 0, 10, 10, 0, ctypes.byref(d), None) == 1
    assert lib.fe_track(None, None, None, None, 0, 0, 0, None) == 1
    assert lib.fe_select(None, None, 0, 0, 0, 0, None, 0, None, 0, 0, None, None, None) == 1
    assert lib.fe_create(0, None) == 1
    assert lib.fe_destroy(None) == 1
    assert lib.fe_batch_run(None, None) == 1


def test_track_record_layout():
    assert TRACK_DTYPE.itemsize == 80
    assert TRACK_DTYPE.fields["track_status"][1] == 32
    assert TRACK_DTYPE.fields["initial_guess_map"][1] == 48
    assert TRACK_DTYPE.fields["ncc"][1] == 72
    t = np.zeros(1, TRACK_DTYPE)
    assert t.view(np.uint8).size == 80
