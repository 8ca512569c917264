import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "ifos3d-dev_b200")
ORACLE = os.path.join(ROOT, "oracle")
for p in (PKG, ORACLE, ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


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
def oracle():
    from pyoracle import Oracle
    return Oracle("oracle")


@pytest.fixture(scope="session")
def ref_oracle():
    from pyoracle import Oracle, have_ref, REFERENCE_SRC
    if not have_ref() and not os.path.isdir(os.path.join(REFERENCE_SRC, "src")):
        pytest.skip("reference build not available")
    return Oracle("ref")


@pytest.fixture(scope="session")
def ifosb_mod():
    import ifosb
    ifosb.build_library()
    return ifosb
