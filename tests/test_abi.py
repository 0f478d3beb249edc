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


def _c_layout(structs, fields, constants):
    """sizeof and offsetof of the header's structs, and the values of its constants, as a C
    compiler lays them out (gcc on the header)."""
    import shutil
    import subprocess
    import tempfile

    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("gcc not available")
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "cuvslam_fe.h"', "int main(void) {"]
    for s in structs:
        lines.append(f'  printf("sizeof {s} %zu\\n", sizeof({s}));')
        for f in fields[s]:
            lines.append(f'  printf("offset {s}.{f} %zu\\n", offsetof({s}, {f}));')
    for c in constants:
        lines.append(f'  printf("const {c} %d\\n", (int)({c}));')
    lines.append("  return 0;\n}")
    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "layout.c"), os.path.join(d, "layout")
        open(src, "w").write("\n".join(lines))
        subprocess.run([gcc, "-std=c99", "-I", os.path.join(ROOT, "include"), src, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout
    got = {}
    for line in out.splitlines():
        kind, name, value = line.split()
        got[(kind, name)] = int(value)
    return got


def test_ctypes_structs_match_the_header():
    """Every ctypes restatement in _lib.py has the header's size, field names and offsets, and the
    Python constants equal the header's."""
    import ctypes

    from cuvslam_b200 import frontend

    pairs = {"fe_pyramid": _lib.FePyramid, "fe_track_finish": _lib.FeTrackFinish,
             "fe_finish_camera": _lib.FeFinishCamera, "fe_camera_frame": _lib.FeCameraFrame,
             "fe_adjoint_job": _lib.FeAdjointJob, "fe_epipolar_curves": _lib.FeEpipolarCurves,
             "fe_stereo_pair": _lib.FeStereoPair}
    fields = {c: [f[0] for f in py._fields_] for c, py in pairs.items()}
    fields["fe_track_data"] = ["track", "offset", "info", "track_status", "cache_index", "initial_guess_map",
                               "search_radius_px", "ncc_threshold", "ncc"]
    fields["fe_affine_cache"] = ["patch", "patch_sums", "level_mask"]
    constants = ["FE_MAX_LEVELS", "FE_ABI_VERSION", "FE_OK", "FE_ERR_INVALID_ARGUMENT", "FE_SAMPLE_TEXTURE",
                 "FE_SAMPLE_EXACT", "FE_SAMPLE_TEXTURE_WIDE", "FE_SAMPLE_HARDWARE", "FE_ADJOINT_IMPLICIT",
                 "FE_ADJOINT_UNROLLED"]
    c = _c_layout(list(fields), fields, constants)
    for name, py in pairs.items():
        assert c[("sizeof", name)] == ctypes.sizeof(py), name
        for f in fields[name]:
            assert c[("offset", f"{name}.{f}")] == getattr(py, f).offset, (name, f)
    assert c[("sizeof", "fe_track_data")] == TRACK_DTYPE.itemsize
    for f in fields["fe_track_data"]:
        assert c[("offset", f"fe_track_data.{f}")] == TRACK_DTYPE.fields[f][1], f
    assert c[("sizeof", "fe_affine_cache")] == frontend.AFFINE_CACHE_BYTES
    assert c[("const", "FE_MAX_LEVELS")] == _lib.MAX_LEVELS
    for k in constants[2:]:
        assert c[("const", k)] == getattr(_lib, k), k


@pytest.mark.parametrize("lang,std", [("c", "c99"), ("c++", "c++11")])
def test_header_is_plain_c_and_cxx(lang, std):
    """The header compiles alone, warning-free and pedantic, for C consumers (ctypes, cgo, JNI stubs)
    and for C++."""
    import shutil
    import subprocess

    cc = shutil.which("gcc" if lang == "c" else "g++")
    if cc is None:
        pytest.skip("compiler not available")
    r = subprocess.run([cc, f"-std={std}", "-Wall", "-Wextra", "-pedantic", "-Werror", "-fsyntax-only", "-I",
                        os.path.join(ROOT, "include"), "-x", lang, "-"], input='#include "cuvslam_fe.h"\n',
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def _prototypes():
    """name -> (return type, [parameter types]) of every FE_API declaration, comments removed."""
    src = open(os.path.join(ROOT, "include", "cuvslam_fe.h")).read()
    src = re.sub(r"/\*.*?\*/", " ", src, flags=re.S)
    out = {}
    for ret, name, params in re.findall(r"FE_API\s+([\w\s\*]+?)\b(fe_\w+)\s*\(([^)]*)\)\s*;", src):
        types = []
        for p in [p.strip() for p in params.split(",") if p.strip() and p.strip() != "void"]:
            types.append(re.sub(r"\s*\b\w+$", "", p) if re.search(r"[\w\*]\s+\**\w+$", p) else p)
        out[name] = (" ".join(ret.split()), [" ".join(t.replace("*", " * ").split()) for t in types])
    return out


def _c_kind(t):
    if "*" in t or t in ("fe_stream",):
        return "ptr"
    return {"int": "i32", "int32_t": "i32", "int64_t": "i64", "float": "f32", "size_t": "i64"}[t]


def _py_kind(t):
    if t in (ctypes.c_void_p, ctypes.c_char_p) or (isinstance(t, type) and issubclass(t, ctypes._Pointer)):
        return "ptr"
    return {ctypes.c_int: "i32", ctypes.c_int32: "i32", ctypes.c_int64: "i64", ctypes.c_float: "f32"}[t]


def test_ctypes_signatures_match_the_prototypes():
    """Each _lib.py signature has the header prototype's arity, and every argument and return value
    the same kind (pointer, 32-bit or 64-bit integer, float)."""
    protos = _prototypes()
    assert sorted(protos) == sorted(_lib._SIGS)
    for name, (res, args) in _lib._SIGS.items():
        cret, cargs = protos[name]
        assert len(args) == len(cargs), (name, len(args), len(cargs))
        assert _py_kind(res) == _c_kind(cret), (name, cret)
        for i, (a, ca) in enumerate(zip(args, cargs)):
            assert _py_kind(a) == _c_kind(ca), (name, i, ca)


def test_every_entry_rejects_null_handles():
    """Every entry point called with NULL pointers and zero sizes returns FE_ERR_INVALID_ARGUMENT
    (the two launch-count queries: -1) without touching a device, each in a child process so that
    a crash would show as a failure rather than end the test run."""
    import subprocess
    import sys

    host_only = {"fe_abi_version", "fe_status_string", "fe_last_cuda_error", "fe_pyramid_levels", "fe_pyramid_bytes"}
    names = [n for n in _lib._SIGS if n not in host_only]
    code = """
import ctypes, json, sys
from cuvslam_b200 import _lib
lib = _lib.load()
out = {}
for name in sys.argv[1:]:
    res, args = _lib._SIGS[name]
    vals = [0.0 if a is ctypes.c_float else (0 if a in (ctypes.c_int, ctypes.c_int64) else None) for a in args]
    out[name] = getattr(lib, name)(*vals)
print(json.dumps(out))
"""
    r = subprocess.run([sys.executable, "-c", code] + names, capture_output=True, text=True, timeout=120,
                       cwd=ROOT, env={**os.environ, "PYTHONPATH": ROOT})
    assert r.returncode == 0, r.stderr
    import json

    got = json.loads(r.stdout.strip().splitlines()[-1])
    for name in names:
        want = -1 if name.endswith("kernel_count") else _lib.FE_ERR_INVALID_ARGUMENT
        assert got[name] == want, (name, got[name])


_CITE = re.compile(r"\b[\w/]+\.(?:cpp|cu|cuh|h):\d+|counterpart")
# entries that replace a reference interface: each cites it in its own comment
_DROP_IN = ["fe_create", "fe_build_pyramid", "fe_build_pyramid_rgb", "fe_build_pyramid_f32", "fe_select", "fe_track",
            "fe_track_mono", "fe_track_stereo", "fe_finish_tracks", "fe_track_affine", "fe_affine_build_cache",
            "fe_track_affine_cached", "fe_pyramid_levels"]


def test_header_cites_the_reference_it_replaces():
    """Each declaration's section of the header, from its banner down to the declaration, cites a
    reference file:line or says the entry has no counterpart; the drop-in entries cite it in the
    comment right above them."""
    src = open(os.path.join(ROOT, "include", "cuvslam_fe.h")).read()
    banners = [m.start() for m in re.finditer(r"/\* -{20,} \*/\n/\*", src)]
    decls = list(re.finditer(r"FE_API\s+[\w\s\*]+?\b(fe_\w+)\s*\(", src))
    for m in decls:
        start = max([b for b in banners if b < m.start()], default=0)
        assert _CITE.search(src[start:m.start()]), m.group(1)
    for m in decls:
        if m.group(1) not in _DROP_IN:
            continue
        before = src[:m.start()]
        comment = before[before.rfind("/*"):before.rfind("*/")]
        assert _CITE.search(comment) and "counterpart" not in comment, m.group(1)
