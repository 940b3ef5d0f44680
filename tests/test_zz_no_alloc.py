"""The allocation-free trace entry point, mgk_trace_rays_static.

It serves callers that may not allocate device memory once they run: a host
application that gives the renderer a fixed share of the GPU and forbids
later cudaMalloc calls, or an interactive loop that cannot take the
device-wide synchronisation an allocation may cause.  Its scratch is a static
array inside the library, so it must give the same records as mgk_trace_rays
(which uses the context's cudaMalloc'd arena).  Two calls in a row check that
the state one call leaves in the shared array does not leak into the next.

This file sorts last so that a run stopping at the first failure has already
run every other test.
"""
import ctypes as C

import numpy as np
import pytest

import magik_b200 as M
from magik_b200 import abi
from tests.conftest import room_scene, small_scene

pytestmark = pytest.mark.gpu


def _static(scene, first, n):
    import torch
    out = torch.empty(n * 128, dtype=torch.uint8, device="cuda")
    M.trace_rays_static(scene, first, n, out)
    torch.cuda.synchronize()
    return out.cpu().numpy().view(M.RESULT_DTYPE)


@pytest.mark.parametrize("precision", [abi.PRECISION_MIXED, abi.PRECISION_F64])
def test_static_entry_matches_context_entry_on_two_calls(ctx, precision):
    s = small_scene(width=64, height=32, spp=2, precision=precision)
    n = s.width * s.height * s.spp  # 4096 rays
    ref = ctx.trace_rays(s, 0, n)
    for _ in range(2):
        got = _static(s, 0, n)
        assert np.array_equal(got.view(np.uint8), ref.view(np.uint8))
    # a different range right after: counters left by the previous call are cleared
    ref2 = ctx.trace_rays(s, 1000, 3000)
    assert np.array_equal(_static(s, 1000, 3000).view(np.uint8), ref2.view(np.uint8))


@pytest.mark.parametrize("precision", [abi.PRECISION_MIXED, abi.PRECISION_F64])
def test_static_entry_matches_context_entry_in_the_room(ctx, precision):
    """Room scenes: mgk_trace_rays continues reflected rays in further
    integrator passes, the static entry point in the tail kernel; the records
    must still be the same bytes, on two calls in a row."""
    s = room_scene(width=48, height=27, spp=2, precision=precision)
    n = s.width * s.height * s.spp
    ref = ctx.trace_rays(s, 0, n)
    assert (ref["bounces"] > 0).mean() > 0.5  # most rays reflect at least once
    for _ in range(2):
        assert np.array_equal(_static(s, 0, n).view(np.uint8), ref.view(np.uint8))


def test_static_entry_at_its_maximum_in_f64(ctx):
    """The largest call (MGK_STATIC_MAX_RAYS rays) in the widest layout (F64,
    ~7 MiB of the 8 MiB array) gives the context entry point's records."""
    s = small_scene(width=128, height=64, spp=2, precision=abi.PRECISION_F64)
    n = M.STATIC_MAX_RAYS
    assert n == s.width * s.height * s.spp
    ref = ctx.trace_rays(s, 0, n)
    assert np.array_equal(_static(s, 0, n).view(np.uint8), ref.view(np.uint8))


def test_static_entry_rejects_more_than_its_maximum():
    import torch
    s = small_scene(width=256, height=128, spp=1)
    out = torch.empty((M.STATIC_MAX_RAYS + 1) * 128, dtype=torch.uint8, device="cuda")
    rc = M.lib().mgk_trace_rays_static(C.byref(s), 0, M.STATIC_MAX_RAYS + 1, out.data_ptr(), None)
    assert rc == abi.ERROR_INVALID_ARGUMENT
    rc = M.lib().mgk_trace_rays_static(C.byref(s), 0, M.STATIC_MAX_RAYS, out.data_ptr(), None)
    assert rc == abi.SUCCESS
