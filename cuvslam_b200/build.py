"""In-tree build of the native library (nvcc, sm_100a) and, for tests, the CPU oracle."""

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def build_library(extra_flags=""):
    """Compiles cuvslam_b200/libcuvslam_fe.so from cuvslam_b200/csrc (make; nvcc -gencode sm_100a)."""
    cmd = ["make", "-s", "-C", os.path.join(HERE, "csrc")]
    if extra_flags:
        cmd.append(f"EXTRA={extra_flags}")
    subprocess.check_call(cmd)
    return os.path.join(HERE, "libcuvslam_fe.so")


def build_checkers(reference=None):
    """Test infrastructure: the CPU oracle and, given a cuVSLAM checkout (`reference`, else the
    CUVSLAM_REFERENCE environment variable), the harness around the reference's own kernels
    (oracle/_ref)."""
    subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle")])
    # builds oracle/_ref when a checkout with the kernels is given, and does nothing otherwise
    ref = reference or os.environ.get("CUVSLAM_REFERENCE", "")
    subprocess.check_call(["bash", os.path.join(ROOT, "oracle", "build_ref.sh")] + ([ref] if ref else []))


def build():
    build_library()
