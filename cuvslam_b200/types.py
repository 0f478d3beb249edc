"""Record layouts shared with cuVSLAM's kernel layer.

`TRACK_DTYPE` is the 80-byte `cuvslam::cuda::TrackData` record (cuda_kernels.h:76-87 in
libs/cuda_modules/cuda_kernels) that `GPULKFeatureTracker::track_points` reads and writes; offsets
were taken from the reference's struct (float2 track @0, float2 offset @8, float info[4] @16,
bool track_status @32, int cache_index @36, float4 initial_guess_map @48 (16-byte aligned),
float search_radius_px @64, float ncc_threshold @68, float ncc @72, size 80 with 16-byte alignment).
`KEYPOINT_DTYPE` is `cuvslam::cuda::Keypoint` (x, y, strength).
"""

import numpy as np

TRACK_DTYPE = np.dtype(
    {
        "names": ["track", "offset", "info", "track_status", "cache_index", "initial_guess_map",
                  "search_radius_px", "ncc_threshold", "ncc"],
        "formats": [("<f4", 2), ("<f4", 2), ("<f4", 4), "u1", "<i4", ("<f4", 4), "<f4", "<f4", "<f4"],
        "offsets": [0, 8, 16, 32, 36, 48, 64, 68, 72],
        "itemsize": 80,
    }
)

KEYPOINT_DTYPE = np.dtype([("x", "<f4"), ("y", "<f4"), ("strength", "<f4")])

MAX_LEVELS = 10
MIN_LEVEL_DIM = 15


def make_tracks(xy, offset=None, search_radius=2048.0, ncc_threshold=0.8) -> np.ndarray:
    """TrackData records as MonoSOFGPU::launch fills them (sof_mono_gpu.cpp:45-63)."""
    xy = np.asarray(xy, np.float32).reshape(-1, 2)
    t = np.zeros(len(xy), TRACK_DTYPE)
    t["track"] = xy
    if offset is not None:
        t["offset"] = np.asarray(offset, np.float32).reshape(-1, 2)
    t["cache_index"] = -1
    t["initial_guess_map"] = (1.0, 0.0, 0.0, 1.0)
    t["search_radius_px"] = search_radius
    t["ncc_threshold"] = ncc_threshold
    return t


def level_sizes(width: int, height: int, max_levels: int = MAX_LEVELS):
    """Pyramid level sizes by the reference rule: halve with (d+1)/2 while both sides stay >= 15,
    at most `max_levels` levels (GPUImagePyramid::prepare_levels, image_pyramid.h:136-151;
    ScaleDownDim, cuda_modules/image_pyramid.cpp:24)."""
    sizes = []
    w, h = width, height
    while len(sizes) < max_levels:
        sizes.append((w, h))
        w, h = (w + 1) // 2, (h + 1) // 2
        if w < MIN_LEVEL_DIM or h < MIN_LEVEL_DIM:
            break
    return sizes
