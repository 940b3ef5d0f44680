"""ctypes mirror of include/mgk_manager.h: the reference's render-manager API
(magik_render_manager_*, the command queue system, framebuffer collections,
renderer statistics) and the library's stage helpers.

Commands are built as the reference's command structs, byte for byte
(`command(...)` and the named builders below), and pushed as 4-byte aligned
buffers, as a C host would push `&cmd`."""
import ctypes as C
import struct

import numpy as np

from . import abi

# e_magik_result_types used by the manager (magik.h:38-110)
SUCCESS = 0
ERROR_INVALID_POINTER = 2
UNKNOWN_ENUM_TYPE = 3
INVALID_CUDA_DEVICE = 4
ERROR_COMMAND_BUFFER_OVERFLOW = 402
ERROR_INVALID_COMMAND = 403
ERROR_PACKED_COMMAND_NOT_ALLIGNED = 404
ERROR_OUT_OF_BOUNDS_COMMAND_BUFFER_READ = 408
ERROR_AOV_INCORRECT_EXTRACT_CALL = 900
ERROR_AOV_SWAPCHAIN_NOT_INITALIZED = 902
ERROR_GL_LOADER_FAILED = 1000
ERROR_GL_FUNCTIONS_NOT_LOADED = 1001

DISPLAY_SWAPCHAIN, DISPLAY_HEADLESS = 0, 1
CONFIG_HOST, CONFIG_CUDA, CONFIG_OPENGL_INTEROP, CONFIG_VULKAN_INTEROP = 0, 1, 2, 3
MAX_AOV = 16
AOV_NAME_BYTES = 512

# command type -> (id, struct format after the type field)
COMMANDS = {
    "SET_STATE_RENDER": (1000, ""), "SET_STATE_PAUSE": (1001, ""), "CLEAR_RENDER_BUFFER": (1002, ""),
    "ADD_AOV": (1003, "I512sI"), "REMOVE_AOV": (1004, "I512s"), "PRINTF": (2000, "I512s"),
    "SET_METRIC_MINKOWSKI": (4000, ""), "SET_METRIC_SCHWARZSCHILD": (4001, ""), "SET_METRIC_KERR": (4002, ""),
    "SET_ABSOLUTE_ERROR_TOLERANCE": (4100, "f"), "SET_RELATIVE_ERROR_TOLERANCE": (4101, "f"),
    "SET_MAX_SUBSTEPS": (4102, "I"), "SET_OBSERVER_LOCAL_PROPER_VELOCITY": (4200, "fff"),
    "SET_CELESTIAL_SPHERE_RADIUS": (4300, "f"), "SET_SCHWARZSCHILD_EVENT_HORIZON_SCALAR": (4400, "f"),
    "SET_SCHWARZSCHILD_MASS_PARAMETER": (4401, "f"), "SET_KERR_EVENT_HORIZON_SCALAR": (4402, "f"),
    "SET_KERR_MASS_PARAMETER": (4403, "f"), "SET_KERR_DIMENSIONLESS_SPIN_PARAMETER": (4404, "f"),
    "SET_ACTIVE_CAMERA": (5000, "I"), "SET_CAMERA_POSITION": (5001, "Ifff"), "SET_CAMERA_ORIENTATION": (5002, "Ifff"),
    "SET_CAMERA_RESOLUTION": (5003, "II"), "SET_N_INTRINSIC_SPECTRAL_IRRADIANCE_BIN": (6000, "I"),
    "SET_SAMPLE_DOMAIN_MAXIMUM_WAVELENGTH_NM": (6001, "f"), "SET_SAMPLE_DOMAIN_MINIMUM_WAVELENGTH_NM": (6002, "f"),
    "SET_REDISTRIBUTION_STANDARD_DEVIATION_NM": (6003, "f"), "SET_COLOR_MATCHING_FUNCTION": (6100, "i"),
    "SET_SCENE_COLORSPACE": (6101, "i"), "SET_VIEW_TRANSFORM": (6102, "i"), "SET_DISPLAY_COLORSPACE": (6103, "i"),
    "SET_OUTPUT_FORMAT": (6104, "i"), "SET_WHITE_BALANCE_WHITE_POINT": (6200, "f"),
    "SET_WHITE_BALANCE_TINT": (6201, "f"), "SET_VIEW_TRANSFORM_REINHARD_EXTENDED_WHITE_LUMINANCE": (6300, "f"),
    "SET_VIEW_TRANSFORM_KHRONOS_PBR_NEUTRAL_START_COMPRESSION": (6301, "f"),
    "SET_VIEW_TRANSFORM_KHRONOS_PBR_NEUTRAL_DESATURATION": (6302, "f"), "SET_VIEW_TRANSFORM_GT7_MODE": (6304, "i"),
    "SET_VIEW_TRANSFORM_GT7_SDR_PAPER_WHITE_BALANCE": (6305, "f"),
    "SET_VIEW_TRANSFORM_GT7_REFERENCE_LUMINANCE": (6306, "f"),
    "SET_VIEW_TRANSFORM_GT7_JZAZBZ_EXPONENT_SCALE_FACTOR": (6407, "f"), "SET_VIEW_TRANSFORM_AGX_LOOK": (6308, "i"),
    "SET_N_GEODESIC_STEP_LIMIT": (7000, "I"), "SET_N_REFLECTED_LIMIT": (7001, "I"),
}

MANAGER_EXPORTS = [
    "magik_render_manager_create", "magik_render_manager_destroy", "magik_render_manager_fetch_error",
    "magik_fetch_renderer_statistics", "magik_destroy_renderer_statistics", "magik_configure_framebuffer_collection",
    "magik_framebuffer_collection_fetch", "magik_extract_config_host", "magik_extract_config_cuda",
    "magik_extract_config_opengl_interop", "magik_extract_vulkan_interop", "magik_destroy_framebuffer_collection",
    "magik_cqs_push_command", "magik_cqs_dispatch_command_buffer", "magik_gl_init", "magik_get_version",
    "mgk_stage_defaults", "mgk_stage_apply", "mgk_command_size", "mgk_stage_scene",
]


def command(name, *args):
    """The bytes of one command struct (little-endian, 4-byte fields)."""
    tid, fmt = COMMANDS[name]
    return struct.pack("<i" + fmt, tid, *args)


def add_aov(name, channels):
    b = name.encode()
    return command("ADD_AOV", len(b), b, channels)


def remove_aov(name):
    b = name.encode()
    return command("REMOVE_AOV", len(b), b)


def printf(text):
    b = text.encode()
    return command("PRINTF", len(b), b)


def chunks(*cmds):
    """Concatenated commands as a uint32 array (a command buffer)."""
    data = b"".join(cmds)
    assert len(data) % 4 == 0
    return np.frombuffer(data, dtype=np.uint32).copy()


class Aov(C.Structure):
    _fields_ = [("channels", C.c_uint32), ("name_length", C.c_uint32), ("name", C.c_char * AOV_NAME_BYTES)]


class Stage(C.Structure):
    _fields_ = [
        ("metric_type", C.c_int32), ("abs_tol", C.c_float), ("rel_tol", C.c_float), ("n_max_substep", C.c_uint32),
        ("observer_velocity", C.c_float * 3), ("celestial_sphere_radius", C.c_float),
        ("schwarzschild_horizon_scalar", C.c_float), ("schwarzschild_mass", C.c_float),
        ("kerr_horizon_scalar", C.c_float), ("kerr_mass", C.c_float), ("kerr_spin", C.c_float),
        ("active_camera", C.c_uint32), ("focal_length_mm", C.c_float), ("iso", C.c_float), ("fps", C.c_float),
        ("shutter_angle", C.c_float), ("sensor_diagonal_mm", C.c_float), ("x_resolution", C.c_uint32),
        ("y_resolution", C.c_uint32), ("position", C.c_float * 3), ("orientation", C.c_float * 9),
        ("n_isi_bin", C.c_uint32), ("isi_max_nm", C.c_float), ("isi_min_nm", C.c_float),
        ("redistribution_sigma_nm", C.c_float), ("cmf_type", C.c_int32), ("scene_colorspace", C.c_int32),
        ("view_transform", C.c_int32), ("display_colorspace", C.c_int32), ("output_format", C.c_int32),
        ("white_point", C.c_float), ("tint", C.c_float), ("reinhard_white_luminance", C.c_float),
        ("khronos_start_compression", C.c_float), ("khronos_desaturation", C.c_float), ("gt7_mode", C.c_int32),
        ("gt7_sdr_paper_white", C.c_float), ("gt7_reference_luminance", C.c_float),
        ("gt7_jzazbz_exponent_scale", C.c_float), ("agx_look", C.c_int32), ("n_geodesic_step_limit", C.c_uint32),
        ("n_reflected_limit", C.c_uint32), ("box_min", C.c_float * 3), ("box_max", C.c_float * 3),
        ("light_min", C.c_float * 3), ("light_max", C.c_float * 3), ("rendering", C.c_uint32),
        ("clear_requested", C.c_uint32), ("n_aov", C.c_uint32), ("aov", Aov * MAX_AOV),
    ]

    def aovs(self):
        return {bytes(a.name[:a.name_length]).decode(): a.channels for a in self.aov[:self.n_aov]}


class ManagerDescriptor(C.Structure):
    _fields_ = [("display_type", C.c_int32), ("user_device_id", C.c_uint32), ("user_stream", C.c_void_p),
                ("cqs_n_reserved_chunk", C.c_uint32), ("cqs_drop_overflow", C.c_bool)]


class RendererStatistics(C.Structure):
    _fields_ = [("x_sample", C.c_size_t), ("total_render_time_seconds", C.c_double),
                ("latest_render_loop_iteration_time_seconds", C.c_double),
                ("total_wavefront_sample_time_seconds", C.c_double),
                ("latest_wavefront_sample_time_seconds", C.c_double),
                ("latest_wavefront_history_length", C.c_size_t),
                ("h_latest_advance_A_queue_count_history", C.POINTER(C.c_uint32)),
                ("h_latest_advance_B_queue_count_history", C.POINTER(C.c_uint32)),
                ("h_latest_intersect_queue_count_history", C.POINTER(C.c_uint32)),
                ("h_latest_bxdf_queue_count_history", C.POINTER(C.c_uint32)),
                ("h_latest_redistribute_queue_count_history", C.POINTER(C.c_uint32)),
                ("h_latest_splat_queue_count_history", C.POINTER(C.c_uint32)),
                ("total_framebuffer_swapchain_size", C.c_size_t), ("total_wavefront_buffer_size", C.c_size_t)]


class HostConfig(C.Structure):
    _fields_ = [("x_resolution", C.c_uint32), ("y_resolution", C.c_uint32), ("channels", C.c_uint32),
                ("size_of_data", C.c_size_t), ("h_data", C.POINTER(C.c_float))]


assert C.sizeof(ManagerDescriptor) == 24 and C.sizeof(RendererStatistics) == 112 and C.sizeof(HostConfig) == 32


def _lib():
    from . import lib
    L = lib()
    if not getattr(L, "_manager_types", False):
        L.mgk_stage_defaults.argtypes = [C.POINTER(Stage)]
        L.mgk_stage_defaults.restype = None
        L.mgk_stage_apply.argtypes = [C.POINTER(Stage), C.c_void_p, C.c_uint32]
        L.mgk_command_size.argtypes = [C.c_int32]
        L.mgk_command_size.restype = C.c_uint32
        L.mgk_stage_scene.argtypes = [C.POINTER(Stage), C.c_uint64, C.POINTER(abi.Scene),
                                      C.POINTER(abi.DisplaySettings)]
        L.magik_render_manager_create.argtypes = [C.POINTER(C.c_void_p), ManagerDescriptor]
        L.magik_render_manager_destroy.argtypes = [C.c_void_p]
        L.magik_render_manager_fetch_error.argtypes = [C.c_void_p]
        L.magik_cqs_push_command.argtypes = [C.c_void_p, C.c_void_p]
        L.magik_cqs_dispatch_command_buffer.argtypes = [C.c_void_p, C.POINTER(C.c_bool)]
        L.magik_fetch_renderer_statistics.argtypes = [C.c_void_p, C.POINTER(C.c_bool), C.POINTER(RendererStatistics)]
        L.magik_destroy_renderer_statistics.argtypes = [C.POINTER(RendererStatistics)]
        L.magik_configure_framebuffer_collection.argtypes = [C.POINTER(C.c_void_p), C.c_int32]
        L.magik_framebuffer_collection_fetch.argtypes = [C.c_void_p, C.POINTER(C.c_bool), C.c_void_p]
        L.magik_extract_config_host.argtypes = [C.c_void_p, C.POINTER(HostConfig), C.c_void_p, C.c_char_p]
        L.magik_extract_config_opengl_interop.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_char_p]
        L.magik_destroy_framebuffer_collection.argtypes = [C.c_void_p]
        L.magik_gl_init.argtypes = [C.c_void_p]
        L.magik_get_version.argtypes = [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                        C.POINTER(C.c_char_p)]
        L._manager_types = True
    return L


def stage_defaults():
    s = Stage()
    _lib().mgk_stage_defaults(C.byref(s))
    return s


def stage_apply(stage, buf):
    """Applies a command buffer (uint32 array or bytes) to the stage; returns the result code."""
    a = np.ascontiguousarray(np.frombuffer(buf, dtype=np.uint32) if isinstance(buf, bytes) else buf, dtype=np.uint32)
    return _lib().mgk_stage_apply(C.byref(stage), a.ctypes.data, len(a))


def command_size(type_id):
    return _lib().mgk_command_size(type_id)


def stage_scene(stage, seed=0):
    """(result code, Scene, DisplaySettings) of one sample pass of the stage."""
    sc, ds = abi.Scene(), abi.DisplaySettings()
    rc = _lib().mgk_stage_scene(C.byref(stage), seed, C.byref(sc), C.byref(ds))
    return rc, sc, ds


class RenderManager:
    """A render manager (its worker thread renders on `device`)."""

    def __init__(self, device=0, n_chunks=4096, drop_overflow=False, headless=False):
        d = ManagerDescriptor(DISPLAY_HEADLESS if headless else DISPLAY_SWAPCHAIN, device, None, n_chunks,
                              drop_overflow)
        h = C.c_void_p()
        self.rc = _lib().magik_render_manager_create(C.byref(h), d)
        self.h = h if self.rc == SUCCESS else None
        self.fb = None

    def push(self, cmd):
        buf = (C.c_uint32 * (len(cmd) // 4)).from_buffer_copy(cmd)
        return _lib().magik_cqs_push_command(self.h, C.addressof(buf))

    def dispatch(self):
        ok = C.c_bool(False)
        rc = _lib().magik_cqs_dispatch_command_buffer(self.h, C.byref(ok))
        return rc, ok.value

    def error(self):
        return _lib().magik_render_manager_fetch_error(self.h)

    def fetch(self):
        """Fetches the newest frame into this manager's host collection; returns (rc, is_new)."""
        if self.fb is None:
            fb = C.c_void_p()
            rc = _lib().magik_configure_framebuffer_collection(C.byref(fb), CONFIG_HOST)
            assert rc == SUCCESS
            self.fb = fb
        new = C.c_bool(False)
        rc = _lib().magik_framebuffer_collection_fetch(self.h, C.byref(new), self.fb)
        return rc, new.value

    def aov(self, name):
        """The fetched AOV as a (y, x, channels) float32 array (None if absent)."""
        cfg = HostConfig()
        rc = _lib().magik_extract_config_host(self.h, C.byref(cfg), self.fb, name.encode())
        assert rc == SUCCESS, rc
        if not cfg.h_data:
            return None
        n = cfg.size_of_data // 4
        a = np.ctypeslib.as_array(cfg.h_data, shape=(n,)).copy()
        return a.reshape(cfg.y_resolution, cfg.x_resolution, cfg.channels)

    def statistics(self):
        st = RendererStatistics()
        new = C.c_bool(False)
        rc = _lib().magik_fetch_renderer_statistics(self.h, C.byref(new), C.byref(st))
        assert rc == SUCCESS
        n = st.latest_wavefront_history_length

        def arr(p):
            return [] if not p else [p[i] for i in range(n)]
        out = {k: getattr(st, k) for k, _ in RendererStatistics._fields_ if not k.startswith("h_")}
        for k, _ in RendererStatistics._fields_:
            if k.startswith("h_"):
                out[k] = arr(getattr(st, k))
        out["is_new"] = new.value
        _lib().magik_destroy_renderer_statistics(C.byref(st))
        return out

    def close(self):
        if self.fb is not None:
            _lib().magik_destroy_framebuffer_collection(self.fb)
            self.fb = None
        if self.h is not None:
            _lib().magik_render_manager_destroy(self.h)
            self.h = None
