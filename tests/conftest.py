import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)

from oracle.build_ref import REF_SRC as REFERENCE_DIR  # noqa: E402  (the reference tree the recipe reads)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libcgli_fu_flow.so")


def have_reference() -> bool:
    return os.path.isdir(REFERENCE_DIR)


@pytest.fixture(scope="session")
def cuda_lib():
    from cgli_fu_flow_b200 import build, solver
    build.build()
    return solver.load_library()
