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


def room_scene(**kw):
    """The reference's box-and-light scene (walls at x, z = +-40 M, floor and
    ceiling at y = -+20 M, light 40 x 2 x 40 M straddling the ceiling) around
    the Kerr a = 0.9 hole, camera 18 M out and 10 degrees above the equator,
    disk off, shrunk like small_scene."""
    import math
    base = dict(room_on=1, cam_r=18.0, cam_incl_rad=math.radians(80.0), disk_r_out=0.0)
    base.update(kw)
    return small_scene(**base)
