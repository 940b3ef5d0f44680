"""ctypes loader of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Imported by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg.
liboracle.so is the C++ restatement (oracle.hpp, oracle_scene.hpp);
_ref/libmagikref.so is the reference's own CPU tracer compiled from its
sources by oracle/Makefile (only present where the reference was available
at build time).
"""
import ctypes as C
import importlib.util
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _load_abi():
    """The plain ctypes layouts of include/mgk.h (magik_b200/abi.py), loaded
    by path so that the oracle, and the CPU legs that use it, run without
    importing the magik_b200 package or loading libmgk.so.  The module is
    registered under its package name, so a later `import magik_b200` shares
    it (one set of ctypes classes)."""
    name = "magik_b200.abi"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, os.path.join(HERE, "..", "magik_b200", "abi.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


abi = _load_abi()
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libmagikref.so")

_lib = None
_ref = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build()
        L = C.CDLL(ORACLE_SO)
        L.orc_trace_geodesic.argtypes = [C.POINTER(abi.TraceContainer), abi.TraceInitialConditions,
                                         abi.TraceMetricParams, abi.TraceIntegratorParams, C.c_int]
        L.orc_trace_geodesic.restype = C.c_int
        L.orc_scene_constants.argtypes = [C.POINTER(abi.Scene), C.POINTER(C.c_double)]
        L.orc_scene_defaults.argtypes = [C.POINTER(abi.Scene)]
        L.orc_scene_defaults.restype = None
        L.orc_isco_radius.argtypes = [C.c_double]
        L.orc_isco_radius.restype = C.c_double
        L.orc_star_catalog.argtypes = [C.c_uint64, C.c_uint32, C.POINTER(abi.Star)]
        L.orc_star_catalog.restype = None
        L.orc_trace_rays.argtypes = [C.POINTER(abi.Scene), C.c_uint64, C.c_uint32, C.POINTER(abi.RayResult),
                                     C.c_int]
        L.orc_shade_rays.argtypes = [C.POINTER(abi.Scene), C.POINTER(abi.Star), C.c_uint32, C.POINTER(C.c_float),
                                     C.c_uint32, C.POINTER(abi.RayResult), C.c_uint64, C.POINTER(C.c_float),
                                     C.POINTER(C.c_double), C.c_int]
        L.orc_render_pixels.argtypes = [C.POINTER(abi.Scene), C.POINTER(abi.Star), C.c_uint32,
                                        C.POINTER(C.c_float), C.c_uint64, C.c_uint32, C.c_uint64,
                                        C.POINTER(C.c_float), C.POINTER(C.c_double), C.POINTER(C.c_uint64),
                                        C.POINTER(C.c_uint64), C.c_int]
        L.orc_count_ops.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_uint64)]
        D3 = C.POINTER(C.c_double)
        F4 = C.POINTER(C.c_float)
        L.orc_room_event.argtypes = [C.POINTER(abi.Scene), D3, D3, D3, C.POINTER(C.c_int)]
        L.orc_white_led.argtypes = [C.c_double]
        L.orc_white_led.restype = C.c_double
        L.orc_reflect_wall.argtypes = [C.POINTER(abi.Scene), F4, F4, C.c_int, C.c_int, C.c_float, C.c_uint32,
                                       C.c_uint64, F4, F4, F4]
        _lib = L
    return _lib


def ref_available():
    return os.path.exists(REF_SO)


def ref():
    global _ref
    if _ref is None:
        R = C.CDLL(REF_SO)
        R.ref_trace_geodesic.argtypes = [C.POINTER(abi.TraceContainer), abi.TraceInitialConditions,
                                         abi.TraceMetricParams, abi.TraceIntegratorParams]
        R.ref_trace_geodesic.restype = C.c_int
        R.ref_cmf_weights.argtypes = [C.c_uint, C.c_float, C.c_float, C.POINTER(C.c_float)]
        R.ref_cmf_inverse_cdf.argtypes = [C.c_float, C.c_float, C.POINTER(C.c_float)]
        R.ref_display_pipeline.argtypes = [C.POINTER(abi.DisplaySettings), C.POINTER(abi.DisplayPipeline)]
        R.ref_display_pixels.argtypes = [C.POINTER(abi.DisplaySettings), C.POINTER(C.c_float), C.c_uint32,
                                         C.POINTER(C.c_float)]
        R.ref_render_pixels.argtypes = [C.POINTER(abi.Scene), C.POINTER(abi.Star), C.c_uint32, C.POINTER(C.c_float),
                                        C.c_uint64, C.c_uint32, C.c_uint64, C.POINTER(C.c_double),
                                        C.POINTER(C.c_uint64), C.c_int]
        R.ref_render_pixels.restype = C.c_int
        R.ref_white_led.argtypes = [C.c_float]
        R.ref_white_led.restype = C.c_float
        F4 = C.POINTER(C.c_float)
        R.ref_reflect_mirror.argtypes = [C.POINTER(abi.Scene), F4, F4, F4, C.c_float, F4, F4]
        R.ref_reflect_mirror.restype = C.c_int
        _ref = R
    return _ref


def scene_defaults(**overrides):
    """The benchmark workload's scene (the oracle's restatement of
    mgk_scene_defaults), with field overrides."""
    s = abi.Scene()
    lib().orc_scene_defaults(C.byref(s))
    for k, v in overrides.items():
        if not hasattr(s, k):
            raise AttributeError(k)
        setattr(s, k, v)
    return s


def isco_radius(spin):
    return lib().orc_isco_radius(float(spin))


def star_catalog(seed, n):
    """The seeded star catalogue (the oracle's restatement of mgk_star_catalog)."""
    out = np.zeros(n, dtype=STAR_DTYPE)
    lib().orc_star_catalog(seed, n, out.ctypes.data_as(C.POINTER(abi.Star)))
    return out


STAR_DTYPE = np.dtype([("dir", "<f4", 3), ("amplitude", "<f4"), ("temperature", "<f4"), ("reserved", "<f4", 3)])


def new_container(n_steps):
    steps = (abi.TraceStep * n_steps)()
    c = abi.TraceContainer(C.sizeof(abi.TraceStep) * n_steps, n_steps, 0,
                           C.cast(steps, C.POINTER(abi.TraceStep)))
    return c, steps


def steps_array(container, steps):
    """(n_written, 15) float32 array of a filled container."""
    n = container.n_written
    a = np.frombuffer(steps, dtype=np.float32, count=15 * len(steps)).reshape(len(steps), 15)
    return a[:n].copy()


def trace_geodesic(ic, mp, ip, n_steps=4096, pow_in_double=False):
    c, steps = new_container(n_steps)
    rc = lib().orc_trace_geodesic(C.byref(c), ic, mp, ip, int(pow_in_double))
    return rc, steps_array(c, steps)


def ref_trace_geodesic(ic, mp, ip, n_steps=4096):
    c, steps = new_container(n_steps)
    rc = ref().ref_trace_geodesic(C.byref(c), ic, mp, ip)
    return rc, steps_array(c, steps)


def ref_cmf_weights(n_bins, lmin, lmax):
    out = (C.c_float * (3 * n_bins))()
    assert ref().ref_cmf_weights(n_bins, lmin, lmax, out) == 0
    return np.frombuffer(out, dtype=np.float32).reshape(n_bins, 3).copy()


def ref_cmf_inverse_cdf(lmin, lmax):
    out = (C.c_float * abi.CMF_ICDF_ENTRIES)()
    assert ref().ref_cmf_inverse_cdf(lmin, lmax, out) == abi.CMF_ICDF_ENTRIES
    return np.frombuffer(out, dtype=np.float32).copy()


def ref_display_pipeline(settings):
    """The reference's colour pipeline for the settings, in the library's
    mgk_display_pipeline layout."""
    p = abi.DisplayPipeline()
    assert ref().ref_display_pipeline(C.byref(settings), C.byref(p)) == 0
    return p


def ref_display_pixels(settings, xyz):
    """Display RGB of XYZ triples (float32 [n, 3]) by the reference's own colour code."""
    x = np.ascontiguousarray(xyz, dtype=np.float32).reshape(-1, 3)
    out = np.zeros_like(x)
    assert ref().ref_display_pixels(C.byref(settings), x.ctypes.data_as(C.POINTER(C.c_float)), len(x),
                                    out.ctypes.data_as(C.POINTER(C.c_float))) == 0
    return out


def scene_constants(scene):
    out = (C.c_double * 32)()
    lib().orc_scene_constants(C.byref(scene), out)
    return np.frombuffer(out, dtype=np.float64).copy()


RESULT_DTYPE = np.dtype([("x", "<f8", 4), ("p", "<f8", 4), ("z", "<f8"), ("r_hit", "<f8"), ("dir", "<f8", 3),
                         ("cls", "<u4"), ("steps", "<u4"), ("attempts", "<u4"), ("wide_attempts", "<u4"),
                         ("refine_evals", "<u4"), ("bounces", "<u4")])
assert RESULT_DTYPE.itemsize == C.sizeof(abi.RayResult)


def trace_rays(scene, first, n, nthreads=None):
    out = np.zeros(n, dtype=RESULT_DTYPE)
    lib().orc_trace_rays(C.byref(scene), first, n, out.ctypes.data_as(C.POINTER(abi.RayResult)),
                         nthreads or os.cpu_count())
    return out


def _icdf_ptr(scene, icdf):
    """The sampled spectral mode's inverse CDF table (256 float32) as a
    pointer, or None in the bin mode."""
    if scene.spectral_mode != abi.SPECTRAL_SAMPLED:
        return None, None
    if icdf is None:
        raise ValueError("the sampled spectral mode needs its inverse CDF table (icdf=...)")
    a = np.ascontiguousarray(icdf, dtype=np.float32)
    assert a.size == abi.CMF_ICDF_ENTRIES
    return a, a.ctypes.data_as(C.POINTER(C.c_float))


def shade_rays(scene, stars, weights, results, nthreads=None, first_ray=0, icdf=None):
    """XYZ of per-ray records of camera rays first_ray, first_ray + 1, ...
    (icdf: the inverse CDF table, sampled spectral mode only)."""
    stars = np.ascontiguousarray(stars)
    w = np.ascontiguousarray(weights, dtype=np.float32)
    out = np.zeros((len(results), 3), dtype=np.float64)
    keep, p = _icdf_ptr(scene, icdf)
    rc = lib().orc_shade_rays(C.byref(scene), stars.ctypes.data_as(C.POINTER(abi.Star)), len(stars),
                              w.ctypes.data_as(C.POINTER(C.c_float)), len(results),
                              np.ascontiguousarray(results).ctypes.data_as(C.POINTER(abi.RayResult)), first_ray, p,
                              out.ctypes.data_as(C.POINTER(C.c_double)), nthreads or os.cpu_count())
    assert rc == 0
    del keep
    return out


def render_pixels(scene, stars, weights, first_pixel, n_pixels, nthreads=None, stride=1, icdf=None):
    stars = np.ascontiguousarray(stars)
    w = np.ascontiguousarray(weights, dtype=np.float32)
    out = np.zeros((n_pixels, 3), dtype=np.float64)
    att, stp = C.c_uint64(0), C.c_uint64(0)
    keep, p = _icdf_ptr(scene, icdf)
    rc = lib().orc_render_pixels(C.byref(scene), stars.ctypes.data_as(C.POINTER(abi.Star)), len(stars),
                                 w.ctypes.data_as(C.POINTER(C.c_float)), first_pixel, n_pixels, stride, p,
                                 out.ctypes.data_as(C.POINTER(C.c_double)), C.byref(att), C.byref(stp),
                                 nthreads or os.cpu_count())
    assert rc == 0
    del keep
    return out, {"attempts": att.value, "steps": stp.value}


def ref_render_pixels(scene, stars, weights, first_pixel, n_pixels, nthreads=None, stride=1):
    """Pixels rendered with the reference's own RKF45 step (oracle/_ref) inside
    the oracle's camera, termination and spectral stages; REF32 semantics.
    Returns (xyz [n, 3] float64, {"attempts": None, "steps": accepted steps}):
    the reference reports no retries."""
    stars = np.ascontiguousarray(stars)
    w = np.ascontiguousarray(weights, dtype=np.float32)
    out = np.zeros((n_pixels, 3), dtype=np.float64)
    stp = C.c_uint64(0)
    rc = ref().ref_render_pixels(C.byref(scene), stars.ctypes.data_as(C.POINTER(abi.Star)), len(stars),
                                 w.ctypes.data_as(C.POINTER(C.c_float)), first_pixel, n_pixels, stride,
                                 out.ctypes.data_as(C.POINTER(C.c_double)), C.byref(stp), nthreads or os.cpu_count())
    assert rc == 0, rc
    return out, {"attempts": None, "steps": stp.value}


def count_ops(metric, fused):
    out = (C.c_uint64 * 2)()
    lib().orc_count_ops(metric, int(fused), out)
    return out[0], out[1]


def _fptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def room_event(scene, p0, p1):
    """First room event on the chord p0 -> p1: (t, axis, side, light)."""
    a0 = np.ascontiguousarray(p0, dtype=np.float64)
    a1 = np.ascontiguousarray(p1, dtype=np.float64)
    t = C.c_double()
    asl = (C.c_int * 3)()
    lib().orc_room_event(C.byref(scene), a0.ctypes.data_as(C.POINTER(C.c_double)),
                         a1.ctypes.data_as(C.POINTER(C.c_double)), C.byref(t), asl)
    return t.value, asl[0], asl[1], bool(asl[2])


def white_led(lam):
    return lib().orc_white_led(float(lam))


def reflect_wall(scene, x, p, axis, side, c0, bounce=0, ray_id=0):
    """One wall reflection of a float state: (x_out[4], p_out[4], c0_out)."""
    xi = np.ascontiguousarray(x, dtype=np.float32)
    pi = np.ascontiguousarray(p, dtype=np.float32)
    xo = np.zeros(4, np.float32)
    po = np.zeros(4, np.float32)
    co = C.c_float()
    lib().orc_reflect_wall(C.byref(scene), _fptr(xi), _fptr(pi), axis, side, c0, bounce, ray_id, _fptr(xo),
                           _fptr(po), C.byref(co))
    return xo, po, co.value


def ref_white_led(lam):
    return ref().ref_white_led(float(lam))


def ref_reflect_mirror(scene, x, p, n, c0):
    """The reference's mirror reflection: (p_out[4], c0_out)."""
    xi = np.ascontiguousarray(x, dtype=np.float32)
    pi = np.ascontiguousarray(p, dtype=np.float32)
    ni = np.ascontiguousarray(n, dtype=np.float32)
    po = np.zeros(4, np.float32)
    co = C.c_float()
    rc = ref().ref_reflect_mirror(C.byref(scene), _fptr(xi), _fptr(pi), _fptr(ni), c0, _fptr(po), C.byref(co))
    assert rc == 0
    return po, co.value
