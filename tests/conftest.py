import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "gpu-pathed_b200"), os.path.join(ROOT, "oracle"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs through the C ABI")
    # build what is missing (the GPU box receives prebuilt libraries with the snapshot)
    lib = os.path.join(ROOT, "gpu-pathed_b200", "libpathed.so")
    olib = os.path.join(ROOT, "oracle", "liboracle.so")
    if not (os.path.exists(lib) and os.path.exists(olib)):
        import __graft_entry__

        __graft_entry__.build()


def _has_gpu():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle

    return oracle.Oracle()


@pytest.fixture(scope="session")
def ref_lib():
    import oracle

    if not os.path.exists(oracle.REF_LIB):
        pytest.skip("reference CPU build not available")
    return oracle.RefCPU()
