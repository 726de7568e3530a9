import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 (B200) GPU")


@pytest.fixture(scope="session")
def orc():
    """The oracle (CPU restatement of the reference), built on first use."""
    from oracle import oracle as O
    O.lib()
    return O


@pytest.fixture(scope="session")
def mqw():
    """The product's Python binding; builds the native library if needed."""
    import multistageqw_b200 as M
    if not os.path.exists(M.LIB_PATH):
        from multistageqw_b200 import build
        build.build()
    M.lib()
    return M


@pytest.fixture(scope="session")
def ctx(mqw):
    c = mqw.Context(0)
    yield c
    c.close()


def load_golden(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)
