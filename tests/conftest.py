import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "gdlog-multinode_b200")
# Root of the reference project's sources, where tests that read its data
# files or drivers find them (GDLOG_REFERENCE overrides); tests that need it
# skip when it is absent.
REF_ROOT = os.environ.get("GDLOG_REFERENCE", "/root/reference")
# What `make -C oracle dropin` built from it: the reference's drivers linked
# against the drop-in headers, and the data files they run on.
DROPIN = os.path.join(REPO, "oracle", "_ref", "dropin")
for p in (PKG, os.path.join(REPO, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle_lib():
    from gdlog_b200 import ORACLE_LIB
    if not os.path.exists(ORACLE_LIB):
        pytest.fail(f"oracle not built: {ORACLE_LIB} (run __graft_entry__.build())")
    return ORACLE_LIB
