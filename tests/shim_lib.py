"""Builds tests/shim_frame.cpp (the test driver of include/cuvslam_fe_shim.hpp) into a shared library
linked against cuvslam_b200/libcuvslam_fe.so and the CUDA runtime."""

import os
import shutil
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def compile_args(out=None):
    gxx = shutil.which("g++")
    if gxx is None:
        return None
    lib_dir = os.path.join(ROOT, "cuvslam_b200")
    args = [gxx, "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"), "-I",
            os.path.join(CUDA, "include"), os.path.join(ROOT, "tests", "shim_frame.cpp")]
    if out is None:
        return args + ["-fsyntax-only"]
    return args + ["-shared", "-fPIC", "-Wl,--no-undefined", "-o", out, "-L", lib_dir, "-lcuvslam_fe",
                   f"-Wl,-rpath,{lib_dir}", "-L", os.path.join(CUDA, "lib64"), "-lcudart"]


def build(out_dir):
    """Compiles and links the driver into out_dir; returns the library's path."""
    out = os.path.join(out_dir, "libshim_frame.so")
    r = subprocess.run(compile_args(out), capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(r.stderr)
    return out
