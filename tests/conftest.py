import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")
# The reference checkout (CPU pins only; absent on GPU machines, where those tests skip).
REFERENCE = os.environ.get("FGSS_REFERENCE", "/root/reference")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs the CUDA library)")


@pytest.fixture(scope="session")
def ctx():
    import new_fgssjoin_b200 as F
    c = F.Context(device=0)
    yield c
    c.close()
