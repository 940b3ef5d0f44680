"""The metric plugin contract (magik_b200/src/renderer/relativity/metric.cuh),
checked on the CPU with a test-only plugin: Schwarzschild restated under the
user tag 16 (tests/plugin/metric_schwarzschild_user.cuh), compiled into a
variant of the library the way a reference-side metric<T> specialisation is
dropped into a build.

* The metric members that run on the host (compute_g, compute_inv_g,
  reference_observer, make_params) of every supported metric give
  g g^-1 = 1 and g(u, u) = -1, and the plugin's equal the built-in
  Schwarzschild's bit for bit (tests/plugin/check_metrics_host.cu, built
  with nvcc and run here).
* The variant library accepts tag 16 and derives the same scene constants
  for it as for the built-in Schwarzschild; the default library refuses it.
The GPU side (records and films bit-identical) is tests/test_gpu_plugin.py.
"""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

import magik_b200 as M
from magik_b200 import abi
from magik_b200 import build as B

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PLUGIN = os.path.join(ROOT, "tests", "plugin")
USER_TAG = 16


def _nvcc():
    try:
        return B.nvcc()
    except RuntimeError:
        return None


@pytest.mark.skipif(_nvcc() is None, reason="nvcc not found")
def test_metric_members_on_the_host(tmp_path):
    exe = str(tmp_path / "check_metrics")
    header = os.path.join(PLUGIN, "metric_schwarzschild_user.cuh")
    cmd = [_nvcc(), "-std=c++17", "-O1", "-gencode", "arch=compute_100a,code=sm_100a",
           "-Xcompiler", "-ffp-contract=off", "-x", "cu", f'-DMGK_USER_METRIC_HEADER="{header}"',
           os.path.join(PLUGIN, "check_metrics_host.cu"), "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout


def _variant():
    lib = B.user_metric_build()
    L = C.CDLL(lib)
    L.mgk_scene_constants.argtypes = [C.POINTER(abi.Scene), C.POINTER(C.c_double)]
    L.mgk_scene_constants.restype = C.c_int32
    return L


def test_variant_library_accepts_the_user_metric():
    L = _variant()
    out1, out16 = (C.c_double * 32)(), (C.c_double * 32)()
    s = M.scene_defaults(metric=abi.METRIC_SCHWARZSCHILD, spin=0.0)
    assert L.mgk_scene_constants(C.byref(s), out1) == abi.SUCCESS
    s.metric = USER_TAG
    assert L.mgk_scene_constants(C.byref(s), out16) == abi.SUCCESS
    assert np.array_equal(np.frombuffer(out1, np.uint64), np.frombuffer(out16, np.uint64))
    # validation takes the plugin's horizon: an explicit camera inside it is
    # refused with MGK_ERROR_INVALID_ARGUMENT (not MGK_ERROR_UNKNOWN_METRIC),
    # before any device call
    L.mgk_trace_rays_static.argtypes = [C.POINTER(abi.Scene), C.c_uint64, C.c_uint32, C.c_void_p, C.c_void_p]
    L.mgk_trace_rays_static.restype = C.c_int32
    for metric in (abi.METRIC_SCHWARZSCHILD, USER_TAG):
        s = M.scene_defaults(metric=metric, spin=0.0, width=8, height=8, spp=1, cam_explicit=1)
        s.cam_pos[0], s.cam_pos[1], s.cam_pos[2] = 0.0, 0.0, 1.5
        for i in range(9):
            s.cam_axes[i] = 1.0 if i in (0, 4, 8) else 0.0
        assert L.mgk_trace_rays_static(C.byref(s), 0, 64, None, None) == abi.ERROR_INVALID_POINTER
        assert L.mgk_trace_rays_static(C.byref(s), 0, 64, C.c_void_p(16), None) == abi.ERROR_INVALID_ARGUMENT


def test_default_library_refuses_an_unlisted_metric():
    """Validation takes the supported_metrics list: tag 16 is not in the
    default build (the check runs before any device call)."""
    import torch
    s = M.scene_defaults(metric=USER_TAG, width=8, height=8, spp=1)
    out = torch.empty(64 * 128, dtype=torch.uint8)
    rc = M.lib().mgk_trace_rays_static(C.byref(s), 0, 64, out.data_ptr(), None)
    assert rc == abi.ERROR_UNKNOWN_METRIC
