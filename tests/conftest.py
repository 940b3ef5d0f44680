import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (run with -m gpu)")


@pytest.fixture(scope="session")
def ctx():
    import magik_b200 as M
    c = M.Context(0)
    yield c
    c.close()


def small_scene(**kw):
    """Kerr a = 0.9 render scene shrunk to a size the oracle traces in seconds."""
    import magik_b200 as M
    base = dict(width=48, height=27, spp=2)
    base.update(kw)
    return M.scene_defaults(**base)
