"""The product path stays apart from the checker: the package never imports the oracle, the native
library links neither the oracle nor the reference harness, bench.py imports the oracle only in
its CPU-baseline and reference legs and its parity checker (run after the timed regions), and
without the native library the package fails loudly (there is no CPU fallback)."""

import ast
import glob
import os
import shutil
import subprocess

import pytest

from conftest import ROOT


def _imports(tree):
    for node in ast.walk(tree):
        if isinstance(node, ast.Import):
            yield from (a.name for a in node.names)
        elif isinstance(node, ast.ImportFrom) and node.module:
            yield node.module


def test_package_never_imports_the_oracle():
    for path in glob.glob(os.path.join(ROOT, "cuvslam_b200", "*.py")):
        mods = list(_imports(ast.parse(open(path).read())))
        assert not [m for m in mods if m.split(".")[0] == "oracle"], path


def test_library_links_no_checker():
    lib = os.path.join(ROOT, "cuvslam_b200", "libcuvslam_fe.so")
    if not os.path.exists(lib) or shutil.which("readelf") is None:
        pytest.skip("library or readelf not available")
    out = subprocess.run(["readelf", "-d", lib], capture_output=True, text=True, check=True).stdout
    needed = [l for l in out.splitlines() if "NEEDED" in l]
    assert needed and not [l for l in needed if "oracle" in l or "cuvslam_ref" in l], needed


def test_bench_uses_the_oracle_only_in_cpu_legs():
    tree = ast.parse(open(os.path.join(ROOT, "bench.py")).read())
    top = [m for node in tree.body if isinstance(node, (ast.Import, ast.ImportFrom)) for m in _imports(node)]
    assert "oracle" not in [m.split(".")[0] for m in top]
    users = set()
    for node in ast.walk(tree):
        if isinstance(node, ast.FunctionDef) and any(m.split(".")[0] == "oracle" for m in _imports(node)):
            users.add(node.name)
    # the reference arm / CPU baseline of the headline, the CPU legs of the other workloads, and the
    # checkers against the reference's own kernels (the headline's parity, the stream's deviation)
    assert users <= {"cpu_reference_step_fn", "config_sequence", "config_stereo_plain", "config_l2r",
                     "config_affine", "reference_parity", "stream_reference_deviation"}, users
    assert "main" not in users


def test_missing_library_fails_loudly(monkeypatch):
    from cuvslam_b200 import _lib

    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setattr(_lib, "LIB_PATH", os.path.join(ROOT, "cuvslam_b200", "no_such_library.so"))
    with pytest.raises(ImportError):
        _lib.load()
