import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "oracle"), os.path.join(ROOT, "gvdb-voxels_b200"), ROOT, os.path.dirname(__file__),
          os.path.join(os.path.dirname(__file__), "golden")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA path through the C-ABI")


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def gvdb2_mod():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test collected without a CUDA device")
    sys.path.insert(0, os.path.join(ROOT, "gvdb-voxels_b200"))
    import build as gbuild
    gbuild.build()
    import gvdb2
    return gvdb2
