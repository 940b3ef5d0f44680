"""ctypes mirror of include/mgk.h (the C ABI of libmgk.so).

Only plain C layouts live here; the loader and the Python-facing functions are
in magik_b200/__init__.py.
"""
import ctypes as C

SUCCESS = 0
ERROR_INVALID_POINTER = 2
ERROR_HOST_TRACE_ALLOCATED_STEPS_AND_CAPACITY_MISMATCH = 102
ERROR_UNKNOWN_METRIC = 707
ERROR_UNKNOWN = 10000
ERROR_INVALID_ARGUMENT = 10001
ERROR_CUDA = 10002
ERROR_NO_DEVICE = 10003
ERROR_DEVICE_STATUS = 10004

METRIC_MINKOWSKI, METRIC_SCHWARZSCHILD, METRIC_KERR = 0, 1, 2
PRECISION_REF32, PRECISION_MIXED, PRECISION_F64 = 0, 1, 2
RAY_ALIVE, RAY_DISK, RAY_ESCAPED, RAY_HORIZON, RAY_STEP_LIMIT, RAY_LIGHT = 0, 1, 2, 3, 4, 5
RAY_CLASSES = 6
CLASS_NAMES = {0: "alive", 1: "disk", 2: "escaped", 3: "horizon", 4: "step_limit", 5: "light"}
MASSIVE, MASSLESS = 0, 1
MAX_BINS = 64
PASS_HISTORY = 16
SPECTRAL_BINS, SPECTRAL_SAMPLED = 0, 1
CMF_ICDF_ENTRIES = 256
WIDE_BAND = 0.05
RESULT_BYTES = 128  # sizeof(mgk_ray_result)


class Scene(C.Structure):
    _fields_ = [
        ("metric", C.c_int32), ("precision", C.c_int32), ("time_reversed", C.c_int32),
        ("n_max_substep", C.c_uint32),
        ("spin", C.c_double), ("mass_sign", C.c_double), ("horizon_scalar", C.c_double),
        ("abs_tol", C.c_double), ("rel_tol", C.c_double), ("h_max", C.c_double),
        ("max_steps", C.c_uint32), ("n_bins", C.c_uint32),
        ("escape_radius", C.c_double), ("disk_r_in", C.c_double), ("disk_r_out", C.c_double),
        ("disk_T_in", C.c_double), ("cam_r", C.c_double), ("cam_incl_rad", C.c_double),
        ("focal_length_mm", C.c_double), ("sensor_diag_mm", C.c_double),
        ("width", C.c_uint32), ("height", C.c_uint32), ("spp", C.c_uint32), ("spectral_mode", C.c_uint32),
        ("seed", C.c_uint64), ("lambda_min_nm", C.c_double), ("lambda_max_nm", C.c_double),
        ("star_radius_rad", C.c_double),
        ("iso", C.c_double), ("fps", C.c_double), ("shutter_angle_deg", C.c_double),
        ("redistribution_sigma_nm", C.c_double),
        ("room_on", C.c_uint32), ("room_reflection_limit", C.c_uint32),
        ("room_min", C.c_double * 3), ("room_max", C.c_double * 3),
        ("light_min", C.c_double * 3), ("light_max", C.c_double * 3), ("light_scale", C.c_double),
        ("cam_explicit", C.c_uint32), ("sample_offset", C.c_uint32), ("cam_pos", C.c_double * 3),
        ("cam_axes", C.c_double * 9), ("cam_velocity", C.c_double * 3),
    ]

    def copy(self):
        s = Scene()
        C.pointer(s)[0] = self
        return s

    def __repr__(self):
        return "Scene(" + ", ".join(f"{n}={getattr(self, n)!r}" for n, _ in self._fields_) + ")"


SCENE_CS = dict(CIE_XYZ=0, CIE_RGB=1, LINEAR_REC709=2, LINEAR_REC2020=3, ACES_CG=4, ADOBE_RGB_1998=5)
DISPLAY_CS = dict(SRGB=0, REC709=1, REC2100_PQ=2, REC2100_HLG=3, DCI_P3_THEATRICAL_WHITE_POINT=4, DISPLAY_P3=5,
                  ADOBE_RGB=6)
VIEW_TRANSFORM = dict(NONE=0, REINHARD_SIMPLE=1, REINHARD_EXTENDED=2, GRAN_TURISMO_7=3, AGX=4, KHRONOS_PBR_NEUTRAL=5)
GT7_MODE = dict(ICTCP=0, JZAZBZ=1)
AGX_LOOK = dict(NONE=0, GOLDEN=1, PUNCHY=2)


class DisplaySettings(C.Structure):
    _fields_ = [("scene_colorspace", C.c_int32), ("view_transform", C.c_int32), ("display_colorspace", C.c_int32),
                ("gt7_mode", C.c_int32), ("agx_look", C.c_int32), ("reserved", C.c_int32),
                ("white_point_K", C.c_double), ("tint", C.c_double), ("reinhard_white_luminance", C.c_double),
                ("khronos_start_compression", C.c_double), ("khronos_desaturation", C.c_double),
                ("gt7_sdr_paper_white", C.c_double), ("gt7_reference_luminance", C.c_double),
                ("gt7_jzazbz_exponent_scale", C.c_double)]


class DisplayPipeline(C.Structure):
    _fields_ = [("view_transform", C.c_int32), ("display_colorspace", C.c_int32), ("gt7_mode", C.c_int32),
                ("agx_look", C.c_int32),
                ("xyz_to_scene", C.c_float * 9), ("scene_to_display", C.c_float * 9),
                ("vt_to_working", C.c_float * 9), ("vt_from_working", C.c_float * 9),
                ("agx_inset", C.c_float * 9), ("agx_outset", C.c_float * 9),
                ("luminance_weights", C.c_float * 3), ("reinhard_white_luminance", C.c_float),
                ("khronos_start_compression", C.c_float), ("khronos_desaturation", C.c_float),
                ("gt7_reference_luminance", C.c_float), ("gt7_jzazbz_exponent_scale", C.c_float),
                ("gt7_peak_intensity", C.c_float), ("gt7_alpha", C.c_float), ("gt7_mid_point", C.c_float),
                ("gt7_linear_section", C.c_float), ("gt7_toe_strength", C.c_float),
                ("gt7_kA", C.c_float), ("gt7_kB", C.c_float), ("gt7_kC", C.c_float),
                ("gt7_sdr_correction", C.c_float), ("gt7_fb_luminance_target", C.c_float),
                ("gt7_fb_luminance_target_ucs", C.c_float),
                ("gt7_blend_ratio", C.c_float), ("gt7_fade_start", C.c_float), ("gt7_fade_end", C.c_float),
                ("reserved", C.c_float * 3)]


class Star(C.Structure):
    _fields_ = [("dir", C.c_float * 3), ("amplitude", C.c_float), ("temperature", C.c_float),
                ("reserved", C.c_float * 3)]


class RayResult(C.Structure):
    _fields_ = [("x", C.c_double * 4), ("p", C.c_double * 4), ("z", C.c_double), ("r_hit", C.c_double),
                ("dir", C.c_double * 3), ("cls", C.c_uint32), ("steps", C.c_uint32),
                ("attempts", C.c_uint32), ("wide_attempts", C.c_uint32),
                ("refine_evals", C.c_uint32), ("bounces", C.c_uint32)]


class RenderStats(C.Structure):
    _fields_ = [("rays", C.c_uint64), ("attempts", C.c_uint64), ("steps", C.c_uint64),
                ("wide_attempts", C.c_uint64), ("refine_evals", C.c_uint64),
                ("class_count", C.c_uint64 * 6),
                ("integrate_ms", C.c_double), ("total_ms", C.c_double), ("crossings", C.c_uint64),
                ("resumed", C.c_uint64), ("fallback_rays", C.c_uint64), ("surrogate_ms", C.c_double),
                ("reflections", C.c_uint64), ("n_passes", C.c_uint32), ("reserved_passes", C.c_uint32),
                ("pass_rays", C.c_uint64 * PASS_HISTORY), ("pass_crossings", C.c_uint64 * PASS_HISTORY),
                ("pass_hits", C.c_uint64 * PASS_HISTORY), ("pass_continued", C.c_uint64 * PASS_HISTORY),
                ("pass_to_tail", C.c_uint64 * PASS_HISTORY)]


class SampleLabel(C.Structure):
    _fields_ = [("cls", C.c_int32), ("r", C.c_float), ("g", C.c_float), ("dir", C.c_float * 3),
                ("reserved", C.c_float * 2)]


class TrainConfig(C.Structure):
    _fields_ = [("batch", C.c_uint32), ("epochs", C.c_uint32), ("lr", C.c_float), ("beta1", C.c_float),
                ("beta2", C.c_float), ("eps", C.c_float), ("seed", C.c_uint64),
                ("w_cls", C.c_float), ("w_r", C.c_float), ("w_g", C.c_float), ("w_dir", C.c_float),
                ("w_conf", C.c_float), ("tol_r", C.c_float), ("tol_g", C.c_float), ("tol_dir", C.c_float),
                ("lr_final", C.c_float), ("reserved", C.c_uint32)]


assert C.sizeof(SampleLabel) == 32


class TraceMetricParams(C.Structure):
    _fields_ = [("metric_type", C.c_int32), ("time_reversed", C.c_bool), ("event_horizon_scalar", C.c_float),
                ("schwarzschild_mass", C.c_float), ("kerr_mass", C.c_float), ("kerr_spin", C.c_float)]


class TraceIntegratorParams(C.Structure):
    _fields_ = [("n_integrator_max_substep", C.c_uint), ("integrator_absolute_error_tolerance", C.c_float),
                ("integrator_relative_error_tolerance", C.c_float)]


class TraceInitialConditions(C.Structure):
    _fields_ = [("test_particle_type", C.c_int32),
                ("spatial_position_x", C.c_float), ("spatial_position_y", C.c_float),
                ("spatial_position_z", C.c_float),
                ("x_rotation", C.c_float), ("y_rotation", C.c_float), ("z_rotation", C.c_float),
                ("local_proper_velocity_x", C.c_float), ("local_proper_velocity_y", C.c_float),
                ("local_proper_velocity_z", C.c_float), ("massive_particle_speed", C.c_float)]


class TraceStep(C.Structure):
    _fields_ = [("four_position", C.c_float * 4), ("four_momentum", C.c_float * 4),
                ("moment_derivative", C.c_float * 4), ("four_vector_contraction", C.c_float),
                ("affine_parameter", C.c_float), ("delta_affine_parameter", C.c_float)]


class TraceContainer(C.Structure):
    _fields_ = [("capacity", C.c_uint64), ("n_allocated_step", C.c_uint32), ("n_written", C.c_uint32),
                ("steps", C.POINTER(TraceStep))]


assert C.sizeof(Scene) == 456, C.sizeof(Scene)
assert C.sizeof(Star) == 32
assert C.sizeof(RayResult) == 128
assert C.sizeof(TraceStep) == 60
assert C.sizeof(TraceMetricParams) == 24
