"""The metric plugin contract on the GPU: the test-only plugin
(tests/plugin/metric_schwarzschild_user.cuh, Schwarzschild restated under
the user tag 16 against magik_b200/src/renderer/relativity/metric.cuh),
compiled into a variant of the library, gives records bit-identical to the
built-in metric<MGK_METRIC_SCHWARZSCHILD> through every kernel of the path
(k_generate, k_integrate, k_refine, k_tail; the room's reflections; the
shaded film), in all three precisions.

The variant library runs in a child process (MGK_LIB), so that this process
keeps the default build loaded."""
import json
import os
import subprocess
import sys

import pytest

from magik_b200 import build as B

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import json, sys
import numpy as np
import torch
sys.path.insert(0, ROOT)
import magik_b200 as M
from magik_b200 import abi
from tests.conftest import small_scene, room_scene

out = {}
with M.Context(0) as ctx:
    for prec in (abi.PRECISION_REF32, abi.PRECISION_MIXED, abi.PRECISION_F64):
        for room in (False, True):
            make = room_scene if room else small_scene
            kw = dict(metric=abi.METRIC_SCHWARZSCHILD, spin=0.0, precision=prec, width=40, height=24, spp=2)
            if not room:
                kw.update(cam_r=30.0, disk_r_in=6.0)
            a_s = make(**kw)
            b_s = make(**kw)
            b_s.metric = 16
            n = a_s.width * a_s.height * a_s.spp
            a = ctx.trace_rays(a_s, 0, n)
            b = ctx.trace_rays(b_s, 0, n)
            key = f"{prec}/{int(room)}"
            out[key] = {"same": bool(np.array_equal(a.view(np.uint8), b.view(np.uint8))),
                        "classes": np.bincount(a["cls"], minlength=abi.RAY_CLASSES).tolist(),
                        "bounces": int(a["bounces"].sum())}
            fa = torch.empty(a_s.width * a_s.height * 3, dtype=torch.float32, device="cuda")
            fb = torch.empty_like(fa)
            stars = torch.from_numpy(M.star_catalog(7, 3000).view(np.uint8)).cuda()
            ctx.render(a_s, stars, fa)
            ctx.render(b_s, stars, fb)
            out[key]["film_same"] = bool(torch.equal(fa, fb)) and bool(torch.isfinite(fa).all())
print(json.dumps(out))
"""


def test_user_metric_equals_builtin_schwarzschild_on_the_gpu():
    lib = B.user_metric_build()
    env = dict(os.environ, MGK_LIB=lib)
    r = subprocess.run([sys.executable, "-c", CHILD.replace("ROOT", repr(ROOT))], env=env, cwd=ROOT,
                       capture_output=True, text=True, timeout=1200)
    assert r.returncode == 0, r.stderr[-3000:]
    res = json.loads(r.stdout.strip().splitlines()[-1])
    assert len(res) == 6
    for key, v in res.items():
        assert v["same"], (key, v)
        assert v["film_same"], (key, v)
    # the frames exercise the disk, escapes, the horizon and (in the room) reflections
    plain = res["1/0"]["classes"]
    assert plain[1] > 0 and plain[2] > 0 and plain[3] > 0
    assert res["1/1"]["bounces"] > 0
