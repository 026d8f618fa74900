"""Shared fixtures.  Tests marked `gpu` need a CUDA device (sm_100a); the rest
run on CPU only."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for sub in ("crystal-opt_b200", "oracle"):
    p = os.path.join(ROOT, sub)
    if p not in sys.path:
        sys.path.insert(0, p)


if "CRYSTAL_OPT_REF" not in os.environ:  # the reference tree the build recipe uses, when present
    sys.path.insert(0, ROOT)
    from __graft_entry__ import REFERENCE_TREE  # noqa: E402

    if os.path.isdir(REFERENCE_TREE):
        os.environ["CRYSTAL_OPT_REF"] = REFERENCE_TREE


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def _has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


HAS_GPU = _has_gpu()


@pytest.fixture(scope="session")
def sj():
    import starjoin
    starjoin.load()
    return starjoin


@pytest.fixture(scope="session")
def oracle():
    import oracle as o
    o.load()
    return o


@pytest.fixture(scope="session")
def engine(sj):
    if not HAS_GPU:
        pytest.skip("no CUDA device")
    eng = sj.Engine(0)
    yield eng
    eng.close()


@pytest.fixture(scope="session")
def torch_cuda():
    if not HAS_GPU:
        pytest.skip("no CUDA device")
    import torch
    return torch
