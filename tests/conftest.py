import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the sm_100a kernels")


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


HAS_GPU = _has_gpu()


def pytest_collection_modifyitems(config, items):
    if HAS_GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle
    oracle.orc().orc_set_threads(min(16, os.cpu_count() or 1))
    return oracle


@pytest.fixture(scope="session")
def atl():
    """The library with argument errors returned instead of exiting."""
    import atlas_b200
    atlas_b200.lib()
    atlas_b200.atlb_set_error_mode(1)
    return atlas_b200


@pytest.fixture(scope="session")
def gpu(atl):
    """The library on a GPU (device 0), sharing one stream with torch: the
    tensors a test creates are ordered before the library's kernels that read
    them (the library's own stream would not wait for torch's)."""
    import torch
    assert atl.atlb_init(0) == 0
    s = torch.cuda.Stream(device=0)
    torch.cuda.set_stream(s)
    atl.atlb_set_stream(s.cuda_stream)
    return atl
