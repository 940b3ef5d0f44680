"""The render-manager API on the CPU: the command queue system's command
layouts and parsing, every command's effect on the stage (the reference's
command.cpp semantics, range checks included), and the stage -> scene
conversion.  The manager itself needs a GPU (tests/test_gpu_manager.py)."""
import math
import struct

import numpy as np
import pytest

import magik_b200 as M
from magik_b200 import abi
from magik_b200 import manager as MG


def test_command_sizes_match_the_reference_structs():
    # magik.h:942-1212: 4-byte type plus the fields
    expect = {"SET_STATE_RENDER": 4, "ADD_AOV": 524, "REMOVE_AOV": 520, "PRINTF": 520, "SET_METRIC_KERR": 4,
              "SET_ABSOLUTE_ERROR_TOLERANCE": 8, "SET_MAX_SUBSTEPS": 8, "SET_OBSERVER_LOCAL_PROPER_VELOCITY": 16,
              "SET_CAMERA_POSITION": 20, "SET_CAMERA_ORIENTATION": 20, "SET_CAMERA_RESOLUTION": 12,
              "SET_VIEW_TRANSFORM": 8, "SET_N_REFLECTED_LIMIT": 8}
    for name, (tid, fmt) in MG.COMMANDS.items():
        size = MG.command_size(tid)
        assert size == 4 + struct.calcsize("<" + fmt), name
        if name in expect:
            assert size == expect[name], name
    assert MG.command_size(1234) == 0 and MG.command_size(6303) == 0


def test_stage_defaults_are_the_references():
    s = MG.stage_defaults()
    assert s.metric_type == abi.METRIC_KERR
    assert s.abs_tol == pytest.approx(1e-3) and s.rel_tol == pytest.approx(1e-10) and s.n_max_substep == 56
    assert s.celestial_sphere_radius == 1000.0 and s.kerr_spin == pytest.approx(0.999)
    assert s.kerr_mass == pytest.approx(6.7329546075e26, rel=1e-7)
    assert (s.x_resolution, s.y_resolution) == (2195, 1860) and list(s.position) == [2.0, 0.0, 9.0]
    assert list(s.orientation) == [1, 0, 0, 0, 1, 0, 0, 0, 1]
    assert (s.n_isi_bin, s.isi_min_nm, s.isi_max_nm) == (24, 360.0, 830.0)
    assert s.view_transform == abi.VIEW_TRANSFORM["GRAN_TURISMO_7"] and s.white_point == 5600.0
    assert (s.n_geodesic_step_limit, s.n_reflected_limit) == (512, 10)
    assert list(s.box_max) == [20, 10, 20] and list(s.light_min) == [-10, 9.5, -10]
    assert s.rendering == 1 and s.n_aov == 0 and s.clear_requested == 0


@pytest.mark.parametrize("name,args,field,value", [
    ("SET_METRIC_SCHWARZSCHILD", (), "metric_type", abi.METRIC_SCHWARZSCHILD),
    ("SET_ABSOLUTE_ERROR_TOLERANCE", (1e-6,), "abs_tol", np.float32(1e-6)),
    ("SET_RELATIVE_ERROR_TOLERANCE", (1e-7,), "rel_tol", np.float32(1e-7)),
    ("SET_MAX_SUBSTEPS", (12,), "n_max_substep", 12),
    ("SET_CELESTIAL_SPHERE_RADIUS", (500.0,), "celestial_sphere_radius", 500.0),
    ("SET_SCHWARZSCHILD_EVENT_HORIZON_SCALAR", (1.5,), "schwarzschild_horizon_scalar", 1.5),
    ("SET_SCHWARZSCHILD_MASS_PARAMETER", (2e27,), "schwarzschild_mass", np.float32(2e27)),
    ("SET_KERR_EVENT_HORIZON_SCALAR", (1.25,), "kerr_horizon_scalar", 1.25),
    ("SET_KERR_MASS_PARAMETER", (1e27,), "kerr_mass", np.float32(1e27)),
    ("SET_KERR_DIMENSIONLESS_SPIN_PARAMETER", (0.5,), "kerr_spin", 0.5),
    ("SET_N_INTRINSIC_SPECTRAL_IRRADIANCE_BIN", (32,), "n_isi_bin", 32),
    ("SET_SAMPLE_DOMAIN_MAXIMUM_WAVELENGTH_NM", (780.0,), "isi_max_nm", 780.0),
    ("SET_SAMPLE_DOMAIN_MINIMUM_WAVELENGTH_NM", (380.0,), "isi_min_nm", 380.0),
    ("SET_REDISTRIBUTION_STANDARD_DEVIATION_NM", (5.0,), "redistribution_sigma_nm", 5.0),
    ("SET_SCENE_COLORSPACE", (3,), "scene_colorspace", 3),
    ("SET_VIEW_TRANSFORM", (4,), "view_transform", 4),
    ("SET_DISPLAY_COLORSPACE", (0,), "display_colorspace", 0),
    ("SET_OUTPUT_FORMAT", (0,), "output_format", 0),
    ("SET_WHITE_BALANCE_WHITE_POINT", (6500.0,), "white_point", 6500.0),
    ("SET_WHITE_BALANCE_TINT", (0.25,), "tint", 0.25),
    ("SET_VIEW_TRANSFORM_REINHARD_EXTENDED_WHITE_LUMINANCE", (2.0,), "reinhard_white_luminance", 2.0),
    ("SET_VIEW_TRANSFORM_KHRONOS_PBR_NEUTRAL_START_COMPRESSION", (0.5,), "khronos_start_compression", 0.5),
    ("SET_VIEW_TRANSFORM_KHRONOS_PBR_NEUTRAL_DESATURATION", (0.25,), "khronos_desaturation", 0.25),
    ("SET_VIEW_TRANSFORM_GT7_MODE", (0,), "gt7_mode", 0),
    ("SET_VIEW_TRANSFORM_GT7_SDR_PAPER_WHITE_BALANCE", (200.0,), "gt7_sdr_paper_white", 200.0),
    ("SET_VIEW_TRANSFORM_GT7_REFERENCE_LUMINANCE", (80.0,), "gt7_reference_luminance", 80.0),
    ("SET_VIEW_TRANSFORM_GT7_JZAZBZ_EXPONENT_SCALE_FACTOR", (1.5,), "gt7_jzazbz_exponent_scale", 1.5),
    ("SET_VIEW_TRANSFORM_AGX_LOOK", (2,), "agx_look", 2),
    ("SET_N_GEODESIC_STEP_LIMIT", (2000,), "n_geodesic_step_limit", 2000),
    ("SET_N_REFLECTED_LIMIT", (3,), "n_reflected_limit", 3),
])
def test_each_setting_command(name, args, field, value):
    s = MG.stage_defaults()
    assert MG.stage_apply(s, MG.chunks(MG.command(name, *args))) == 0
    assert getattr(s, field) == value
    assert s.clear_requested == 1


@pytest.mark.parametrize("name,args,field", [
    # range checks of command.cpp: values outside are ignored
    ("SET_ABSOLUTE_ERROR_TOLERANCE", (0.0,), "abs_tol"), ("SET_RELATIVE_ERROR_TOLERANCE", (-1.0,), "rel_tol"),
    ("SET_MAX_SUBSTEPS", (0,), "n_max_substep"), ("SET_CELESTIAL_SPHERE_RADIUS", (0.0,), "celestial_sphere_radius"),
    ("SET_KERR_EVENT_HORIZON_SCALAR", (1.0,), "kerr_horizon_scalar"),
    ("SET_SCHWARZSCHILD_EVENT_HORIZON_SCALAR", (0.5,), "schwarzschild_horizon_scalar"),
    ("SET_N_INTRINSIC_SPECTRAL_IRRADIANCE_BIN", (65,), "n_isi_bin"),
    ("SET_N_INTRINSIC_SPECTRAL_IRRADIANCE_BIN", (0,), "n_isi_bin"),
    ("SET_VIEW_TRANSFORM_GT7_JZAZBZ_EXPONENT_SCALE_FACTOR", (1.0,), "gt7_jzazbz_exponent_scale"),
    ("SET_N_GEODESIC_STEP_LIMIT", (0,), "n_geodesic_step_limit"), ("SET_N_REFLECTED_LIMIT", (0,), "n_reflected_limit"),
])
def test_out_of_range_settings_are_ignored(name, args, field):
    s = MG.stage_defaults()
    before = getattr(s, field)
    assert MG.stage_apply(s, MG.chunks(MG.command(name, *args))) == 0
    assert getattr(s, field) == before and s.clear_requested == 0


def test_camera_commands():
    s = MG.stage_defaults()
    buf = MG.chunks(MG.command("SET_CAMERA_POSITION", 0, 1.0, -2.0, 3.5),
                    MG.command("SET_CAMERA_ORIENTATION", 0, 0.3, -0.7, 1.1),
                    MG.command("SET_CAMERA_RESOLUTION", 0, 5),
                    MG.command("SET_OBSERVER_LOCAL_PROPER_VELOCITY", 1e7, 0.0, -2e7),
                    MG.command("SET_ACTIVE_CAMERA", 3))
    assert MG.stage_apply(s, buf) == 0
    assert list(s.position) == [1.0, -2.0, 3.5]
    assert (s.x_resolution, s.y_resolution) == (2, 5)  # 0 -> 2 (command.cpp:398-399)
    assert list(s.observer_velocity) == [1e7, 0.0, -2e7]

    def R(ax, t):
        c, n = math.cos(t), math.sin(t)
        return {"x": np.array([[1, 0, 0], [0, c, -n], [0, n, c]]), "y": np.array([[c, 0, n], [0, 1, 0], [-n, 0, c]]),
                "z": np.array([[c, -n, 0], [n, c, 0], [0, 0, 1]])}[ax]
    want = R("x", np.float32(0.3)) @ R("y", np.float32(-0.7)) @ R("z", np.float32(1.1))
    assert np.allclose(np.array(s.orientation).reshape(3, 3), want, atol=1e-6)


def test_state_aov_and_printf_commands(capfd):
    s = MG.stage_defaults()
    buf = MG.chunks(MG.command("SET_STATE_PAUSE"), MG.add_aov("beauty", 4), MG.add_aov("depth", 1),
                    MG.add_aov("beauty", 3), MG.printf("hello from the queue"))
    assert MG.stage_apply(s, buf) == 0
    assert s.rendering == 0 and s.aovs() == {"beauty": 4, "depth": 1}  # an existing name is kept
    assert "hello from the queue" in capfd.readouterr().out
    assert s.clear_requested == 0
    assert MG.stage_apply(s, MG.chunks(MG.remove_aov("beauty"), MG.command("SET_STATE_RENDER"),
                                       MG.command("CLEAR_RENDER_BUFFER"))) == 0
    assert s.aovs() == {"depth": 1} and s.rendering == 1 and s.clear_requested == 1


def test_invalid_and_truncated_buffers():
    s = MG.stage_defaults()
    good = MG.command("SET_MAX_SUBSTEPS", 9)
    bad = np.concatenate([MG.chunks(good), np.array([9999], np.uint32)])
    assert MG.stage_apply(s, bad) == MG.ERROR_INVALID_COMMAND and s.n_max_substep == 9
    s = MG.stage_defaults()
    trunc = MG.chunks(good, MG.command("SET_CAMERA_POSITION", 0, 1.0, 2.0, 3.0))[:-1]
    assert MG.stage_apply(s, trunc) == MG.ERROR_OUT_OF_BOUNDS_COMMAND_BUFFER_READ
    assert s.n_max_substep == 9 and list(s.position) == [2.0, 0.0, 9.0]
    assert MG.stage_apply(s, np.zeros(0, np.uint32)) == 0


def test_stage_scene_units_and_room():
    s = MG.stage_defaults()
    rc, sc, ds = MG.stage_scene(s, seed=7)
    assert rc == 0
    L = 6.67430e-11 * float(np.float32(6.7329546075e26)) / 299792458.0 ** 2  # 0.5 m
    assert L == pytest.approx(0.5, rel=1e-6)
    assert sc.metric == abi.METRIC_KERR and sc.spin == pytest.approx(0.999) and sc.cam_explicit == 1
    assert list(sc.cam_pos) == pytest.approx([2 / L, 0.0, 9 / L])
    assert list(sc.cam_axes) == [1, 0, 0, 0, 1, 0, 0, 0, 1]
    assert list(sc.room_max) == pytest.approx([20 / L, 10 / L, 20 / L]) and sc.room_on == 1
    assert list(sc.light_min) == pytest.approx([-10 / L, 9.5 / L, -10 / L])
    assert sc.escape_radius == pytest.approx(1000 / L) and sc.room_reflection_limit == 10
    assert sc.spectral_mode == abi.SPECTRAL_SAMPLED and sc.n_bins == 24
    assert (sc.lambda_min_nm, sc.lambda_max_nm) == (360.0, 830.0) and sc.spp == 1 and sc.seed == 7
    assert (sc.width, sc.height) == (2195, 1860) and sc.max_steps == 512 and sc.disk_r_out == 0.0
    assert sc.precision == abi.PRECISION_MIXED
    assert ds.view_transform == abi.VIEW_TRANSFORM["GRAN_TURISMO_7"] and ds.white_point_K == 5600.0
    # a larger celestial sphere than MIXED's float range allows runs in F64
    MG.stage_apply(s, MG.chunks(MG.command("SET_CELESTIAL_SPHERE_RADIUS", 8000.0)))
    rc, sc, _ = MG.stage_scene(s)
    assert rc == 0 and sc.precision == abi.PRECISION_F64
    # a camera outside the room is refused
    MG.stage_apply(s, MG.chunks(MG.command("SET_CAMERA_POSITION", 0, 0.0, 0.0, 30.0)))
    rc, _, _ = MG.stage_scene(s)
    assert rc == abi.ERROR_INVALID_ARGUMENT
    # observer velocity in units of c; orientation columns become the camera axes
    s = MG.stage_defaults()
    MG.stage_apply(s, MG.chunks(MG.command("SET_OBSERVER_LOCAL_PROPER_VELOCITY", 0.0, 0.0, -299792458.0 * 0.5),
                                MG.command("SET_CAMERA_ORIENTATION", 0, 0.0, 0.5, 0.0)))
    rc, sc, _ = MG.stage_scene(s)
    assert rc == 0 and list(sc.cam_velocity) == pytest.approx([0, 0, -0.5])
    O = np.array(s.orientation, dtype=np.float64).reshape(3, 3)
    assert np.allclose(np.array(sc.cam_axes).reshape(3, 3), O.T)


def test_manager_without_gpu_and_graphics_entry_points():
    import torch
    L = MG._lib()
    assert L.magik_gl_init(None) == MG.ERROR_GL_LOADER_FAILED
    import ctypes as C
    a, b, c = C.c_uint32(), C.c_uint32(), C.c_uint32()
    txt = C.c_char_p()
    assert L.magik_get_version(C.byref(a), C.byref(b), C.byref(c), C.byref(txt)) == 0
    assert (a.value, b.value, c.value) == (0, 7, 0) and b"Magik" in txt.value
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    m = MG.RenderManager(0)
    assert m.rc == MG.INVALID_CUDA_DEVICE and m.h is None
