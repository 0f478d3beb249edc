"""B200-native visual-tracking front-end (cuVSLAM's pyramid + Shi-Tomasi + pyramidal LK hot path).

Compute runs in libcuvslam_fe.so (hand-written sm_100a CUDA behind a C ABI, include/cuvslam_fe.h);
`cuvslam_b200.frontend` mirrors the reference's host-wrapper interface on top of it.
"""

__version__ = "0.1.0"
