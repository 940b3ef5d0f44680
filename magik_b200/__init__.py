"""B200-native geodesic path: Python mirror of the C ABI in include/mgk.h.

The compute path is libmgk.so (hand-written sm_100a kernels behind a C ABI);
this module only loads it through ctypes and moves buffers.  There is no CPU
fallback: every compute entry point raises if the library or a B200 is not
available.  PyTorch is used for device memory and streams.
"""
import ctypes as C
import os

import numpy as np

from . import abi
from .abi import Scene, Star, RayResult, RenderStats  # noqa: F401

HERE = os.path.dirname(os.path.abspath(__file__))
# MGK_LIB selects another build of the library (e.g. a launch-shape variant)
LIB_PATH = os.environ.get("MGK_LIB", os.path.join(HERE, "libmgk.so"))

_lib = None

RESULT_DTYPE = np.dtype([("x", "<f8", 4), ("p", "<f8", 4), ("z", "<f8"), ("r_hit", "<f8"), ("dir", "<f8", 3),
                         ("cls", "<u4"), ("steps", "<u4"), ("attempts", "<u4"), ("wide_attempts", "<u4"),
                         ("refine_evals", "<u4"), ("bounces", "<u4")])
STAR_DTYPE = np.dtype([("dir", "<f4", 3), ("amplitude", "<f4"), ("temperature", "<f4"), ("reserved", "<f4", 3)])
STEP_DTYPE = np.dtype([("four_position", "<f4", 4), ("four_momentum", "<f4", 4), ("moment_derivative", "<f4", 4),
                       ("four_vector_contraction", "<f4"), ("affine_parameter", "<f4"),
                       ("delta_affine_parameter", "<f4")])
assert RESULT_DTYPE.itemsize == 128 and STAR_DTYPE.itemsize == 32 and STEP_DTYPE.itemsize == 60

EXPORTS = [
    "mgk_context_create", "mgk_context_destroy", "mgk_last_error", "mgk_scene_defaults", "mgk_isco_radius",
    "mgk_xyz_weights", "mgk_star_catalog", "mgk_scene_constants", "mgk_render", "mgk_render_host",
    "mgk_trace_rays", "mgk_shade_rays", "magik_trace_geodesic", "mgk_trace_geodesic_batch", "mgk_fp32_peak", "mgk_fp64_peak",
    "mgk_check_rounding", "mgk_cmf_inverse_cdf", "mgk_xyz_weights_analytic", "mgk_cmf_inverse_cdf_analytic", "mgk_display_defaults", "mgk_display_prepare", "mgk_display",
    "mgk_trace_rays_static", "mgk_train_defaults", "mgk_surrogate_param_count", "mgk_surrogate_create",
    "mgk_surrogate_destroy", "mgk_surrogate_get_params", "mgk_surrogate_set_params", "mgk_make_samples",
    "mgk_surrogate_forward", "mgk_surrogate_forward_tiled", "mgk_surrogate_status", "mgk_surrogate_gradient", "mgk_surrogate_train", "mgk_render_surrogate",
    "mgk_surrogate_shuffle", "mgk_surrogate_order", "mgk_surrogate_gradient_step", "mgk_surrogate_adam_step",
]


class MgkError(RuntimeError):
    def __init__(self, code, what, detail=""):
        super().__init__(f"{what} failed with code {code}" + (f": {detail}" if detail else ""))
        self.code = code


def lib():
    """The loaded libmgk.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m magik_b200.build`")
        L = C.CDLL(LIB_PATH)
        P = C.POINTER
        vp = C.c_void_p
        L.mgk_context_create.argtypes = [C.c_int32, P(vp)]
        L.mgk_context_destroy.argtypes = [vp]
        L.mgk_last_error.argtypes = [vp]
        L.mgk_last_error.restype = C.c_char_p
        L.mgk_scene_defaults.argtypes = [P(Scene)]
        L.mgk_scene_defaults.restype = None
        L.mgk_isco_radius.argtypes = [C.c_double]
        L.mgk_isco_radius.restype = C.c_double
        L.mgk_xyz_weights.argtypes = [C.c_uint32, C.c_double, C.c_double, P(C.c_float)]
        L.mgk_xyz_weights_analytic.argtypes = [C.c_uint32, C.c_double, C.c_double, P(C.c_float)]
        L.mgk_star_catalog.argtypes = [C.c_uint64, C.c_uint32, vp]
        L.mgk_scene_constants.argtypes = [P(Scene), P(C.c_double)]
        L.mgk_render.argtypes = [vp, P(Scene), vp, C.c_uint32, vp, vp, vp, P(RenderStats), vp]
        L.mgk_render_host.argtypes = [vp, P(Scene), vp, C.c_uint32, vp, vp, P(RenderStats), vp]
        L.mgk_trace_rays.argtypes = [vp, P(Scene), C.c_uint64, C.c_uint32, vp, vp]
        L.mgk_shade_rays.argtypes = [vp, P(Scene), vp, C.c_uint32, vp, C.c_uint64, C.c_uint32, vp, vp]
        L.magik_trace_geodesic.argtypes = [P(abi.TraceContainer), abi.TraceInitialConditions,
                                           abi.TraceMetricParams, abi.TraceIntegratorParams]
        L.magik_trace_geodesic.restype = C.c_int32
        L.mgk_trace_geodesic_batch.argtypes = [vp, P(abi.TraceContainer), P(abi.TraceInitialConditions),
                                               P(abi.TraceMetricParams), P(abi.TraceIntegratorParams), C.c_uint32]
        L.mgk_fp32_peak.argtypes = [vp, P(C.c_double)]
        L.mgk_fp64_peak.argtypes = [vp, P(C.c_double)]
        L.mgk_check_rounding.argtypes = [vp, P(C.c_uint64)]
        L.mgk_cmf_inverse_cdf.argtypes = [C.c_double, C.c_double, P(C.c_float)]
        L.mgk_cmf_inverse_cdf_analytic.argtypes = [C.c_double, C.c_double, P(C.c_float)]
        L.mgk_display_defaults.argtypes = [P(abi.DisplaySettings)]
        L.mgk_display_defaults.restype = None
        L.mgk_display_prepare.argtypes = [P(abi.DisplaySettings), P(abi.DisplayPipeline)]
        L.mgk_display.argtypes = [vp, P(abi.DisplayPipeline), vp, C.c_uint64, vp, vp]
        L.mgk_trace_rays_static.argtypes = [P(Scene), C.c_uint64, C.c_uint32, vp, vp]
        L.mgk_train_defaults.argtypes = [P(abi.TrainConfig)]
        L.mgk_train_defaults.restype = None
        L.mgk_surrogate_param_count.argtypes = []
        L.mgk_surrogate_param_count.restype = C.c_uint64
        L.mgk_surrogate_create.argtypes = [vp, C.c_uint64, P(vp)]
        L.mgk_surrogate_destroy.argtypes = [vp]
        L.mgk_surrogate_get_params.argtypes = [vp, P(C.c_float)]
        L.mgk_surrogate_set_params.argtypes = [vp, P(C.c_float)]
        L.mgk_make_samples.argtypes = [vp, P(Scene), C.c_uint64, C.c_uint32, C.c_uint32, vp, vp, vp]
        L.mgk_surrogate_forward.argtypes = [vp, vp, C.c_uint32, vp, vp]
        L.mgk_surrogate_forward_tiled.argtypes = [vp, vp, C.c_uint32, vp, vp]
        L.mgk_surrogate_status.argtypes = [vp, P(C.c_uint32)]
        L.mgk_surrogate_gradient.argtypes = [vp, P(abi.TrainConfig), vp, vp, C.c_uint32, P(C.c_float),
                                             P(C.c_float)]
        L.mgk_surrogate_train.argtypes = [vp, P(abi.TrainConfig), vp, vp, C.c_uint32, P(C.c_float), vp]
        L.mgk_surrogate_shuffle.argtypes = [vp, C.c_uint64, C.c_uint32, C.c_uint32, vp]
        L.mgk_surrogate_order.argtypes = [vp, P(C.c_uint32), C.c_uint32]
        L.mgk_surrogate_gradient_step.argtypes = [vp, P(abi.TrainConfig), vp, vp, C.c_uint32, C.c_uint32, vp, vp,
                                                  vp]
        L.mgk_surrogate_adam_step.argtypes = [vp, P(abi.TrainConfig), vp, C.c_float, C.c_double, vp]
        L.mgk_render_surrogate.argtypes = [vp, vp, P(Scene), vp, C.c_uint32, vp, C.c_float, C.c_float, vp,
                                           P(RenderStats), vp]
        for name in EXPORTS:
            fn = getattr(L, name)
            if fn.restype is C.c_int:  # ctypes default
                fn.restype = C.c_int32
        _lib = L
    return _lib


def _check(code, what, ctx=None):
    if code != abi.SUCCESS:
        detail = lib().mgk_last_error(ctx).decode() if ctx else ""
        raise MgkError(code, what, detail)


# ------------------------------------------------------------ host helpers
def scene_defaults(**overrides):
    s = Scene()
    lib().mgk_scene_defaults(C.byref(s))
    for k, v in overrides.items():
        if not hasattr(s, k):
            raise AttributeError(k)
        setattr(s, k, v)
    return s


def isco_radius(spin):
    return lib().mgk_isco_radius(float(spin))


def xyz_weights(n_bins, lambda_min_nm=380.0, lambda_max_nm=780.0, analytic=False):
    """mgk_xyz_weights: per-bin XYZ weights (n_bins x 3) from the tabulated
    CIE 1931 observer; `analytic` selects mgk_xyz_weights_analytic."""
    out = (C.c_float * (3 * n_bins))()
    fn = "mgk_xyz_weights_analytic" if analytic else "mgk_xyz_weights"
    _check(getattr(lib(), fn)(n_bins, lambda_min_nm, lambda_max_nm, out), fn)
    return np.frombuffer(out, dtype=np.float32).reshape(n_bins, 3).copy()


def cmf_inverse_cdf(lambda_min_nm=380.0, lambda_max_nm=780.0, analytic=False):
    """mgk_cmf_inverse_cdf: the sampled spectral mode's CIE inverse CDF table
    (256 wavelengths in nm); `analytic` selects the table of the analytic fit."""
    out = (C.c_float * abi.CMF_ICDF_ENTRIES)()
    fn = "mgk_cmf_inverse_cdf_analytic" if analytic else "mgk_cmf_inverse_cdf"
    _check(getattr(lib(), fn)(lambda_min_nm, lambda_max_nm, out), fn)
    return np.frombuffer(out, dtype=np.float32).copy()


def display_defaults(**overrides):
    """mgk_display_defaults (the reference's colour settings) with overrides;
    enum fields accept the names of abi.SCENE_CS / DISPLAY_CS / VIEW_TRANSFORM /
    GT7_MODE / AGX_LOOK."""
    d = abi.DisplaySettings()
    lib().mgk_display_defaults(C.byref(d))
    names = dict(scene_colorspace=abi.SCENE_CS, display_colorspace=abi.DISPLAY_CS, view_transform=abi.VIEW_TRANSFORM,
                 gt7_mode=abi.GT7_MODE, agx_look=abi.AGX_LOOK)
    for k, v in overrides.items():
        if not hasattr(d, k):
            raise AttributeError(k)
        setattr(d, k, names[k][v] if isinstance(v, str) else v)
    return d


def display_prepare(settings):
    """mgk_display_prepare: the display pipeline of the settings."""
    p = abi.DisplayPipeline()
    _check(lib().mgk_display_prepare(C.byref(settings), C.byref(p)), "mgk_display_prepare")
    return p


def star_catalog(seed, n):
    out = np.zeros(n, dtype=STAR_DTYPE)
    _check(lib().mgk_star_catalog(seed, n, out.ctypes.data_as(C.c_void_p)), "mgk_star_catalog")
    return out


def scene_constants(scene):
    out = (C.c_double * 32)()
    _check(lib().mgk_scene_constants(C.byref(scene), out), "mgk_scene_constants")
    return np.frombuffer(out, dtype=np.float64).copy()


def _stream_ptr(stream):
    if stream is None:
        import torch
        return C.c_void_p(torch.cuda.current_stream().cuda_stream)
    return C.c_void_p(getattr(stream, "cuda_stream", stream))


# ----------------------------------------------------------------- context
class Context:
    """A device context (mgk_context): kernels, scratch arena, events."""

    def __init__(self, device=0):
        h = C.c_void_p()
        _check(lib().mgk_context_create(device, C.byref(h)), "mgk_context_create")
        self.handle = h
        self.device = device

    def close(self):
        if self.handle:
            lib().mgk_context_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def fp32_peak(self):
        """Measured FP32 FLOP/s of this device (FMA probe)."""
        v = C.c_double(0)
        _check(lib().mgk_fp32_peak(self.handle, C.byref(v)), "mgk_fp32_peak", self.handle)
        return v.value

    def fp64_peak(self):
        """Measured FP64 FLOP/s of this device (double FMA probe)."""
        v = C.c_double(0)
        _check(lib().mgk_fp64_peak(self.handle, C.byref(v)), "mgk_fp64_peak", self.handle)
        return v.value

    def check_rounding(self):
        """mgk_check_rounding: (msqrt, mrcp) mismatch counts over all 2^32 floats."""
        out = (C.c_uint64 * 2)()
        _check(lib().mgk_check_rounding(self.handle, out), "mgk_check_rounding", self.handle)
        return int(out[0]), int(out[1])

    def display(self, pipeline, d_xyz, d_rgb, stream=None):
        """mgk_display: d_xyz (float32 CUDA tensor of n*3) -> d_rgb (same shape)."""
        n = d_xyz.numel() // 3
        _check(lib().mgk_display(self.handle, C.byref(pipeline), d_xyz.data_ptr(), n, d_rgb.data_ptr(),
                                 _stream_ptr(stream)), "mgk_display", self.handle)

    # -- device-buffer entry points (torch CUDA tensors)
    def render(self, scene, d_stars, d_film_xyz, d_weights=None, d_film_spectral=None, want_stats=True,
               stream=None):
        """mgk_render: d_stars (uint8/any CUDA tensor of n*32 bytes or None), d_film_xyz float32 [H*W*3]."""
        n_stars = 0 if d_stars is None else d_stars.numel() * d_stars.element_size() // 32
        st = RenderStats() if want_stats else None
        rc = lib().mgk_render(self.handle, C.byref(scene), None if d_stars is None else d_stars.data_ptr(),
                              n_stars, None if d_weights is None else d_weights.data_ptr(), d_film_xyz.data_ptr(),
                              None if d_film_spectral is None else d_film_spectral.data_ptr(),
                              C.byref(st) if st is not None else None, _stream_ptr(stream))
        _check(rc, "mgk_render", self.handle)
        return st

    def render_host(self, scene, h_stars, h_film_xyz, h_weights=None, want_stats=True, stream=None):
        """mgk_render_host: host pointers (numpy arrays or pinned torch tensors)."""
        def ptr(a):
            if a is None:
                return None
            return a.data_ptr() if hasattr(a, "data_ptr") else a.ctypes.data
        n_stars = 0 if h_stars is None else (h_stars.nbytes if hasattr(h_stars, "nbytes") else
                                             h_stars.numel() * h_stars.element_size()) // 32
        st = RenderStats() if want_stats else None
        rc = lib().mgk_render_host(self.handle, C.byref(scene), ptr(h_stars), n_stars, ptr(h_weights),
                                   ptr(h_film_xyz), C.byref(st) if st is not None else None, _stream_ptr(stream))
        _check(rc, "mgk_render_host", self.handle)
        return st

    def trace_rays(self, scene, first, n, stream=None):
        """Per-ray results of camera rays [first, first+n) as a numpy structured array."""
        import torch
        buf = torch.empty(max(n, 1) * 128, dtype=torch.uint8, device=f"cuda:{self.device}")
        _check(lib().mgk_trace_rays(self.handle, C.byref(scene), first, n, buf.data_ptr(), _stream_ptr(stream)),
               "mgk_trace_rays", self.handle)
        host = buf.cpu().numpy()
        return host[: n * 128].view(RESULT_DTYPE).copy()

    def shade_rays(self, scene, stars, weights, first, n, stream=None):
        """Per-ray XYZ of camera rays [first, first+n) as a float32 [n, 3] numpy array."""
        import torch
        dev = f"cuda:{self.device}"
        d_stars = None if stars is None or len(stars) == 0 else torch.from_numpy(
            np.ascontiguousarray(stars).view(np.uint8)).to(dev)
        d_w = None if weights is None else torch.from_numpy(np.ascontiguousarray(weights, np.float32).ravel()).to(dev)
        out = torch.empty(max(n, 1) * 3, dtype=torch.float32, device=dev)
        rc = lib().mgk_shade_rays(self.handle, C.byref(scene), None if d_stars is None else d_stars.data_ptr(),
                                  0 if d_stars is None else len(stars), None if d_w is None else d_w.data_ptr(),
                                  first, n, out.data_ptr(), _stream_ptr(stream))
        _check(rc, "mgk_shade_rays", self.handle)
        return out.cpu().numpy()[: 3 * n].reshape(n, 3)

    def trace_geodesic_batch(self, ics, mps, ips, n_steps):
        """Reference-compatible traces: one container of n_steps steps per geodesic."""
        n = len(ics)
        steps = [(abi.TraceStep * n_steps)() for _ in range(n)]
        cs = (abi.TraceContainer * n)()
        for i in range(n):
            cs[i] = abi.TraceContainer(C.sizeof(abi.TraceStep) * n_steps, n_steps, 0,
                                       C.cast(steps[i], C.POINTER(abi.TraceStep)))
        ic_a = (abi.TraceInitialConditions * n)(*ics)
        mp_a = (abi.TraceMetricParams * n)(*mps)
        ip_a = (abi.TraceIntegratorParams * n)(*ips)
        _check(lib().mgk_trace_geodesic_batch(self.handle, cs, ic_a, mp_a, ip_a, n), "mgk_trace_geodesic_batch",
               self.handle)
        out = []
        for i in range(n):
            a = np.frombuffer(steps[i], dtype=np.float32).reshape(n_steps, 15)
            out.append(a[: cs[i].n_written].copy())
        return out


STATIC_MAX_RAYS = 16384


def trace_rays_static(scene, first, n, d_out, stream=None):
    """mgk_trace_rays_static: traces camera rays [first, first+n) into the CUDA
    buffer d_out (n * 128 bytes) with no device allocation; n <= 16384."""
    if d_out.numel() * d_out.element_size() < n * abi.RESULT_BYTES:
        raise ValueError(f"d_out holds {d_out.numel() * d_out.element_size()} bytes, {n} records need "
                         f"{n * abi.RESULT_BYTES}")
    _check(lib().mgk_trace_rays_static(C.byref(scene), first, n, d_out.data_ptr(), _stream_ptr(stream)),
           "mgk_trace_rays_static")


def trace_geodesic(ic, mp, ip, n_steps=4096):
    """magik_trace_geodesic through libmgk (GPU).  Returns (code, steps[n_written, 15])."""
    steps = (abi.TraceStep * n_steps)()
    c = abi.TraceContainer(C.sizeof(abi.TraceStep) * n_steps, n_steps, 0, C.cast(steps, C.POINTER(abi.TraceStep)))
    rc = lib().magik_trace_geodesic(C.byref(c), ic, mp, ip)
    a = np.frombuffer(steps, dtype=np.float32).reshape(n_steps, 15)
    return rc, a[: c.n_written].copy()


# --------------------------------------------------------------- surrogate
LABEL_DTYPE = np.dtype([("cls", "<i4"), ("r", "<f4"), ("g", "<f4"), ("dir", "<f4", (3,)),
                        ("reserved", "<f4", (2,))])
assert LABEL_DTYPE.itemsize == 32


def train_defaults(**overrides):
    c = abi.TrainConfig()
    lib().mgk_train_defaults(C.byref(c))
    for k, v in overrides.items():
        setattr(c, k, v)
    return c


def surrogate_param_count():
    return int(lib().mgk_surrogate_param_count())


class Surrogate:
    """The deflection surrogate network (mgk_surrogate) on a context's device."""

    def __init__(self, ctx, seed=1):
        h = C.c_void_p()
        _check(lib().mgk_surrogate_create(ctx.handle, seed, C.byref(h)), "mgk_surrogate_create", ctx.handle)
        self.handle = h
        self.ctx = ctx

    def close(self):
        if self.handle:
            lib().mgk_surrogate_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def get_params(self):
        out = np.empty(surrogate_param_count(), np.float32)
        _check(lib().mgk_surrogate_get_params(self.handle, out.ctypes.data_as(C.POINTER(C.c_float))),
               "mgk_surrogate_get_params")
        return out

    def set_params(self, params):
        a = np.ascontiguousarray(params, np.float32)
        assert a.size == surrogate_param_count()
        _check(lib().mgk_surrogate_set_params(self.handle, a.ctypes.data_as(C.POINTER(C.c_float))),
               "mgk_surrogate_set_params")

    def forward(self, d_feat, stream=None):
        """d_feat: CUDA float32 [n, 7] -> CUDA float32 [n, 16]."""
        import torch
        n = d_feat.shape[0]
        out = torch.empty((max(n, 1), 16), dtype=torch.float32, device=d_feat.device)
        _check(lib().mgk_surrogate_forward(self.handle, d_feat.data_ptr(), n, out.data_ptr(), _stream_ptr(stream)),
               "mgk_surrogate_forward")
        return out[:n]

    def forward_tiled(self, d_feat, stream=None):
        """The forward pass on the training path's tiled GEMM kernels."""
        import torch
        n = d_feat.shape[0]
        out = torch.empty((max(n, 1), 16), dtype=torch.float32, device=d_feat.device)
        _check(lib().mgk_surrogate_forward_tiled(self.handle, d_feat.data_ptr(), n, out.data_ptr(),
                                                 _stream_ptr(stream)), "mgk_surrogate_forward_tiled")
        return out[:n]

    def status(self):
        v = C.c_uint32(0)
        _check(lib().mgk_surrogate_status(self.handle, C.byref(v)), "mgk_surrogate_status")
        return v.value

    def gradient(self, cfg, d_feat, d_lab):
        """Loss and gradient of one batch (host float32 vector)."""
        g = np.empty(surrogate_param_count(), np.float32)
        loss = C.c_float(0)
        _check(lib().mgk_surrogate_gradient(self.handle, C.byref(cfg), d_feat.data_ptr(), d_lab.data_ptr(),
                                            d_feat.shape[0], g.ctypes.data_as(C.POINTER(C.c_float)),
                                            C.byref(loss)), "mgk_surrogate_gradient")
        return float(loss.value), g

    def train(self, cfg, d_feat, d_lab, stream=None):
        """Adam training; returns the mean loss of each epoch."""
        losses = np.zeros(max(cfg.epochs, 1), np.float32)
        _check(lib().mgk_surrogate_train(self.handle, C.byref(cfg), d_feat.data_ptr(), d_lab.data_ptr(),
                                         d_feat.shape[0], losses.ctypes.data_as(C.POINTER(C.c_float)),
                                         _stream_ptr(stream)), "mgk_surrogate_train")
        return losses[: cfg.epochs]

    # one training step at a time, for data-parallel training (magik_b200.dist)
    @property
    def param_count(self):
        return surrogate_param_count()

    def shuffle(self, seed, epoch, n, stream=None):
        """The sample-set order of one epoch (mgk_surrogate_shuffle)."""
        _check(lib().mgk_surrogate_shuffle(self.handle, seed, epoch, n, _stream_ptr(stream)), "mgk_surrogate_shuffle")

    def order(self, n):
        """The first n entries of the latest sample order (mgk_surrogate_order)."""
        out = np.zeros(n, np.uint32)
        _check(lib().mgk_surrogate_order(self.handle, out.ctypes.data_as(C.POINTER(C.c_uint32)), n),
               "mgk_surrogate_order")
        return out

    def gradient_step(self, cfg, d_feat, d_lab, first, n, d_grad, d_loss_sum, stream=None):
        """Rows [first, first + n) of the order: gradient into d_grad, batch mean loss added to d_loss_sum."""
        _check(lib().mgk_surrogate_gradient_step(self.handle, C.byref(cfg), d_feat.data_ptr(), d_lab.data_ptr(),
                                                 first, n, d_grad.data_ptr(), d_loss_sum.data_ptr(),
                                                 _stream_ptr(stream)), "mgk_surrogate_gradient_step")

    def adam_step(self, cfg, d_grad, grad_scale, progress, stream=None):
        """One Adam step with gradient d_grad x grad_scale at schedule position progress."""
        _check(lib().mgk_surrogate_adam_step(self.handle, C.byref(cfg), d_grad.data_ptr(), grad_scale, progress,
                                             _stream_ptr(stream)), "mgk_surrogate_adam_step")


def make_samples(ctx, base, seed, n, n_spin_buckets=0, stream=None):
    """Training samples traced by the F64 integrator: (features [n, 7] float32,
    labels [n, 8] int32/float32 view of mgk_sample_label) as CUDA tensors."""
    import torch
    dev = f"cuda:{ctx.device}"
    feat = torch.empty((max(n, 1), 7), dtype=torch.float32, device=dev)
    lab = torch.empty((max(n, 1), 8), dtype=torch.int32, device=dev)
    _check(lib().mgk_make_samples(ctx.handle, C.byref(base), seed, n, n_spin_buckets, feat.data_ptr(),
                                  lab.data_ptr(), _stream_ptr(stream)), "mgk_make_samples", ctx.handle)
    return feat[:n], lab[:n]


def render_surrogate(ctx, net, scene, d_stars, d_film_xyz, conf_min=0.99, crit_frac=0.02, d_weights=None,
                     stream=None):
    """mgk_render_surrogate; returns the RenderStats."""
    n_stars = 0 if d_stars is None else d_stars.numel() * d_stars.element_size() // 32
    st = RenderStats()
    rc = lib().mgk_render_surrogate(ctx.handle, net.handle, C.byref(scene),
                                    None if d_stars is None else d_stars.data_ptr(), n_stars,
                                    None if d_weights is None else d_weights.data_ptr(), conf_min, crit_frac,
                                    d_film_xyz.data_ptr(), C.byref(st), _stream_ptr(stream))
    _check(rc, "mgk_render_surrogate", ctx.handle)
    return st


# the reference's render-manager API and the stage helpers (include/mgk_manager.h)
from . import manager  # noqa: E402
EXPORTS = EXPORTS + manager.MANAGER_EXPORTS
