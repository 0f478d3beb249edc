"""The C++ binding sketches of INTEGRATION.md compile against include/cuvslam_fe.h (g++ -fsyntax-only).

cuVSLAM's own types that the sketches use (TrackData, GPUArrayPinned, the selection settings,
CUDA_CHECK, ...) are declared here as stand-ins with the reference's shapes; the library's
declarations come from the real header, so a call whose arguments no longer fit an entry point
fails to compile.  The Python example's names are checked against the package's exports."""

import os
import re
import shutil
import subprocess

import pytest

from conftest import ROOT

PRELUDE = r"""
#include <cstddef>
#include <cstdint>
#include "cuvslam_fe.h"
typedef struct CUstream_st* cudaStream_t;  // as in cuda_runtime_api.h
int cudaMalloc(void** p, size_t bytes);
#define CUDA_CHECK(x) (void)(x)
#define FE_CHECK(x) (void)(x)
struct alignas(16) TrackData { unsigned char bytes[80]; };  // cuda_kernels.h:76-87
template <class T> struct GPUArrayPinned { T* ptr(); const T* ptr() const; size_t size() const; };
struct Settings { int border_top, border_bottom, border_left, border_right; };
struct PointCacheDataT { unsigned char bytes[sizeof(fe_affine_cache)]; };  // PointCacheData<float, 9>
enum class TrackerType { LK, LKHorizontal };
float CrossCamSearchRadius(int top_level);
"""


def _blocks():
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    return re.findall(r"```cpp\n(.*?)```", text, re.S)


def _compile(src):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    r = subprocess.run([gxx, "-std=c++17", "-fsyntax-only", "-Wall", "-I", os.path.join(ROOT, "include"), "-x", "c++",
                        "-"], input=src, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_four_sketches_present():
    assert len(_blocks()) == 4


def test_wrapper_classes_compile():
    _compile(PRELUDE + _blocks()[0])


def test_stereo_sketch_compiles():
    body = _blocks()[1]
    _compile(PRELUDE + """
void stereo_sketch(fe_context* ctx, fe_stereo_pair* pairs, int npairs, int top_w, int top_h, int top_level,
                   const int32_t* d_offsets, const float* d_xy, int32_t max_len, const fe_pyramid& primary_pyr_desc,
                   const fe_pyramid& secondary_pyr_desc, const float* d_uvL, const uint8_t* d_valid, int n,
                   GPUArrayPinned<TrackData>& tracks_data, int32_t* d_winner, int32_t* d_stats,
                   float kL2REarlyExitFraction, TrackerType lr_tracker, cudaStream_t stream) {
""" + body + """
  pairs[0] = pair;
}
""")


def test_affine_sketch_compiles():
    body = _blocks()[2]
    _compile(PRELUDE + _blocks()[0] + """
void affine_sketch(fe_context* ctx, const GaussianGPUImagePyramidB200& prev, const GaussianGPUImagePyramidB200& cur,
                   GPUArrayPinned<TrackData>& td, GPUArrayPinned<PointCacheDataT>& cache_data, size_t n,
                   int n_shift_only_iterations_, int n_full_mapping_iterations_, cudaStream_t s) {
""" + body + """
}
""")


def test_adjoint_sketch_compiles():
    body = _blocks()[3].replace("/* ... loss, dL/dpos into d_dLdpos ... */", "")
    _compile(PRELUDE + """
void adjoint_sketch(fe_context* ctx, const fe_pyramid& prev_desc, const fe_pyramid& cur_desc, const float* d_prev_f32,
                    const float* d_cur_f32, int w, const fe_track_data* d_tracks, fe_track_data* d_tracks_out, int n,
                    const float* d_dLdpos, float* d_gprev, float* d_gcur, float* d_gtrack, float* d_goffset,
                    cudaStream_t s) {
""" + body + """
}
""")


def test_python_example_names_exist():
    """The Python example's imports and calls name what the package exports."""
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    block = re.findall(r"```python\n(.*?)```", text, re.S)[0]
    imports = [l for l in block.splitlines() if l.startswith("from ")]
    ns = {}
    for line in imports:
        exec(line, ns)
    for name in re.findall(r"\b([A-Z][A-Za-z]+|tracks_to_device|make_tracks)\(", block):
        assert name in ns, name
