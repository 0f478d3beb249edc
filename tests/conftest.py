import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O

    O.lib()
    return O


@pytest.fixture(scope="session")
def golden():
    import numpy as np

    inp = np.load(os.path.join(ROOT, "tests", "golden", "inputs.npz"))
    ref = np.load(os.path.join(ROOT, "tests", "golden", "reference.npz"))
    return inp, ref


@pytest.fixture(scope="session")
def ctx():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from cuvslam_b200.frontend import Context

    c = Context(0)
    yield c
    c.close()


def gpu_pyramid(ctx, img_u8, max_levels=10):
    import torch

    from cuvslam_b200.frontend import ImagePyramid

    h, w = img_u8.shape
    p = ImagePyramid(w, h, max_levels)
    p.build(ctx, torch.from_numpy(img_u8).cuda())
    torch.cuda.synchronize()
    return p


def assert_tracks_equal(a, b):
    """Field-by-field bit equality of TrackData records (padding bytes are not data)."""
    import numpy as np

    assert a.shape == b.shape
    for name in a.dtype.names:
        x, y = np.ascontiguousarray(a[name]), np.ascontiguousarray(b[name])
        if x.dtype.kind == "f":
            x, y = x.view(np.uint32), y.view(np.uint32)
        np.testing.assert_array_equal(x, y, err_msg=name)
