"""The render manager on the GPU: commands through the command queue system,
progressive sampling on the worker thread, frames fetched through a host
framebuffer collection, statistics; and the explicit camera the commands
drive, against the oracle."""
import math
import time

import numpy as np
import pytest

import magik_b200 as M
from magik_b200 import abi
from magik_b200 import manager as MG
from oracle import oracle_py as O
from tests.conftest import room_scene

pytestmark = pytest.mark.gpu

SEED = 0x5EED  # the manager's base seed: sample k renders with SEED + k


def _setup_commands(w=64, h=36):
    return [MG.command("SET_CAMERA_RESOLUTION", w, h), MG.command("SET_KERR_DIMENSIONLESS_SPIN_PARAMETER", 0.9),
            MG.command("SET_ABSOLUTE_ERROR_TOLERANCE", 1e-7), MG.command("SET_RELATIVE_ERROR_TOLERANCE", 1e-7),
            MG.command("SET_N_GEODESIC_STEP_LIMIT", 4000), MG.add_aov("beauty", 4), MG.add_aov("rgb", 3)]


def _dispatch(m, timeout=10.0):
    t = time.time()
    while True:
        rc, ok = m.dispatch()
        assert rc == 0
        if ok:
            return
        assert time.time() - t < timeout, "worker never released the command buffer"
        time.sleep(0.005)


def _wait_samples(m, n, timeout=60.0):
    t = time.time()
    while True:
        st = m.statistics()
        if st["x_sample"] >= n:
            return st
        assert m.error() == 0, m.error()
        assert time.time() - t < timeout, f"only {st['x_sample']} samples"
        time.sleep(0.01)


def test_manager_renders_the_accumulated_mean(ctx):
    """After the worker paused, the fetched AOV equals the display colour of
    the mean of samples 0..N-1 rendered one by one through mgk_render (the
    same seeds), bit for bit."""
    import torch
    m = MG.RenderManager(0)
    assert m.rc == 0
    try:
        cmds = _setup_commands()
        for c in cmds:
            assert m.push(c) == 0
        _dispatch(m)
        _wait_samples(m, 3)
        assert m.push(MG.command("SET_STATE_PAUSE")) == 0
        _dispatch(m)
        # the worker finishes its iteration and idles; the sample count settles
        n0 = -1
        for _ in range(200):
            st = m.statistics()
            if st["x_sample"] == n0:
                break
            n0 = st["x_sample"]
            time.sleep(0.05)
        time.sleep(0.1)
        rc, new = m.fetch()
        assert rc == 0 and new
        n = m.statistics()["x_sample"]
        beauty, rgb = m.aov("beauty"), m.aov("rgb")
        assert beauty.shape == (36, 64, 4) and rgb.shape == (36, 64, 3)
        assert (beauty[..., 3] == 1.0).all() and np.array_equal(beauty[..., :3], rgb)
        assert m.aov("missing") is None
        # the same samples through the library directly
        stage = MG.stage_defaults()
        assert MG.stage_apply(stage, MG.chunks(*cmds)) == 0
        acc = None
        for k in range(n):
            rc, sc, ds = MG.stage_scene(stage, SEED + k)
            assert rc == 0
            film = torch.empty(sc.width * sc.height * 3, dtype=torch.float32, device="cuda")
            ctx.render(sc, None, film)
            f = film.cpu().numpy()
            acc = f.copy() if acc is None else (acc + f).astype(np.float32)
        mean = (acc / np.float32(n)).astype(np.float32)
        out = torch.empty(len(mean), dtype=torch.float32, device="cuda")
        ctx.display(M.display_prepare(ds), torch.from_numpy(mean).cuda(), out)
        want = out.cpu().numpy().reshape(36, 64, 3)
        assert np.isfinite(want).all() and (want > 0).mean() > 0.3
        assert np.array_equal(rgb, want)
        # statistics of the latest sample: one integrator pass per reflection
        st = m.statistics()
        L = st["latest_wavefront_history_length"]
        A, B = st["h_latest_advance_A_queue_count_history"], st["h_latest_advance_B_queue_count_history"]
        # pass 0 and room_reflection_limit + 1 continuation passes
        assert L == 12 and A[0] == 64 * 36 and all(A[p + 1] == B[p] for p in range(L - 1))
        assert sum(st["h_latest_redistribute_queue_count_history"]) > 0
        assert st["total_wavefront_sample_time_seconds"] > 0 and st["total_wavefront_buffer_size"] > 0
        assert st["total_framebuffer_swapchain_size"] == 2 * 64 * 36 * 7 * 4
        # nothing new until the next sample
        assert m.fetch() == (0, False)
        assert m.error() == 0
    finally:
        m.close()


def test_manager_settings_clear_the_accumulation(ctx):
    m = MG.RenderManager(0)
    try:
        for c in _setup_commands(32, 18):
            m.push(c)
        _dispatch(m)
        _wait_samples(m, 4)
        m.push(MG.command("SET_CAMERA_POSITION", 0, 1.0, 1.0, 8.0))
        m.push(MG.command("SET_STATE_PAUSE"))
        _dispatch(m)
        t = time.time()
        while m.statistics()["x_sample"] != 0:  # the accumulation restarted
            assert time.time() - t < 30
            time.sleep(0.005)
        time.sleep(0.05)
        assert m.statistics()["x_sample"] == 0  # paused
        m.push(MG.command("SET_STATE_RENDER"))
        _dispatch(m)
        _wait_samples(m, 2)
        assert m.error() == 0
    finally:
        m.close()


def test_manager_command_queue_errors_and_modes(ctx):
    m = MG.RenderManager(0, n_chunks=4)
    try:
        assert m.push(MG.command("SET_MAX_SUBSTEPS", 3)) == 0
        assert m.push(MG.command("SET_CAMERA_POSITION", 0, 1.0, 1.0, 1.0)) == MG.ERROR_COMMAND_BUFFER_OVERFLOW
        import ctypes as C
        buf = (C.c_uint32 * 4)(9999, 0, 0, 0)
        assert MG._lib().magik_cqs_push_command(m.h, C.addressof(buf)) == MG.ERROR_INVALID_COMMAND
        raw = (C.c_uint8 * 16)()
        assert MG._lib().magik_cqs_push_command(m.h, C.addressof(raw) + 1) == MG.ERROR_PACKED_COMMAND_NOT_ALLIGNED
        cfg = MG.HostConfig()
        fb = C.c_void_p()
        assert MG._lib().magik_configure_framebuffer_collection(C.byref(fb), MG.CONFIG_OPENGL_INTEROP) == 0
        assert MG._lib().magik_extract_config_host(m.h, C.byref(cfg), fb, b"x") == MG.ERROR_AOV_INCORRECT_EXTRACT_CALL
        MG._lib().magik_destroy_framebuffer_collection(fb)
        assert MG._lib().magik_configure_framebuffer_collection(C.byref(fb), 7) == MG.UNKNOWN_ENUM_TYPE
    finally:
        m.close()
    m = MG.RenderManager(0, n_chunks=4, drop_overflow=True)
    try:
        assert m.push(MG.command("SET_CAMERA_POSITION", 0, 1.0, 1.0, 1.0)) == 0  # dropped
    finally:
        m.close()
    m = MG.RenderManager(0, headless=True)
    try:
        assert m.fetch()[0] == MG.ERROR_AOV_SWAPCHAIN_NOT_INITALIZED
    finally:
        m.close()
    assert MG.RenderManager(64).rc == MG.INVALID_CUDA_DEVICE


def test_manager_reports_an_invalid_stage(ctx):
    """A camera outside the room: the worker records the scene's error and renders nothing."""
    m = MG.RenderManager(0)
    try:
        for c in _setup_commands(16, 16) + [MG.command("SET_CAMERA_POSITION", 0, 0.0, 0.0, 50.0)]:
            m.push(c)
        _dispatch(m)
        t = time.time()
        while m.error() == 0:
            assert time.time() - t < 10
            time.sleep(0.005)
        assert m.error() == abi.ERROR_INVALID_ARGUMENT
        assert m.statistics()["x_sample"] == 0
    finally:
        m.close()


@pytest.mark.parametrize("precision", [abi.PRECISION_MIXED, abi.PRECISION_F64])
def test_explicit_moving_camera_bit_exact(ctx, precision):
    """An explicit camera (position, rotated axes) whose observer moves: every
    record equal to the oracle's."""
    s = room_scene(precision=precision, cam_explicit=1)
    a = 0.4
    s.cam_pos[:] = (6.0, -3.0, 17.0)
    s.cam_axes[:] = (math.cos(a), 0.0, -math.sin(a), 0.0, 1.0, 0.0, math.sin(a), 0.0, math.cos(a))
    s.cam_velocity[:] = (0.2, 0.0, -0.3)
    n = s.width * s.height * s.spp
    gpu = ctx.trace_rays(s, 0, n)
    orc = O.trace_rays(s, 0, n)
    from tests.test_gpu_parity import compare_records
    compare_records(gpu, orc)
    assert (gpu["cls"] == abi.RAY_LIGHT).any()
