"""Host-side checks that need no GPU: the C ABI library, host utilities, the
oracle's physics against analytic results, and the roofline op counts."""
import math
import os
import re

import numpy as np
import pytest

import magik_b200 as M
from magik_b200 import abi, flops
from oracle import oracle_py as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    names = []
    for h in ("mgk.h", "mgk_manager.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        names += re.findall(r"MGK_API\s+[\w\s\*]+?\b(\w+)\s*\(", text)
    return sorted(set(names))


def test_library_loads_and_exports_every_header_function():
    names = header_functions()
    assert "mgk_render" in names and "magik_trace_geodesic" in names
    L = M.lib()
    for n in names:
        assert hasattr(L, n), n
    assert set(names) == set(M.EXPORTS)


def test_context_reports_no_device_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(M.MgkError) as e:
        M.Context(0)
    assert e.value.code == abi.ERROR_NO_DEVICE


def test_scene_constants_match_oracle():
    for metric in (0, 1, 2):
        for precision in (0, 1, 2):
            s = M.scene_defaults(metric=metric, precision=precision, spin=0.9 if metric == 2 else 0.0)
            assert np.array_equal(M.scene_constants(s), O.scene_constants(s))


def test_isco_and_horizon():
    assert M.isco_radius(0.0) == pytest.approx(6.0, abs=1e-12)
    assert M.isco_radius(0.998) == pytest.approx(1.2370, abs=1e-4)
    assert M.isco_radius(0.9) == pytest.approx(2.3209, abs=1e-4)
    c = M.scene_constants(M.scene_defaults())
    assert c[28] == pytest.approx(1 + math.sqrt(1 - 0.81))  # r_plus


def test_star_catalogue_is_seeded_and_uniform():
    a = M.star_catalog(3, 20000)
    b = M.star_catalog(3, 20000)
    c = M.star_catalog(4, 20000)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    d = a["dir"].astype(np.float64)
    assert np.allclose(np.linalg.norm(d, axis=1), 1, atol=1e-6)
    assert np.abs(d.mean(0)).max() < 0.02  # uniform on the sphere
    assert ((a["temperature"] >= 3000) & (a["temperature"] <= 30000)).all()


def test_flop_counts_match_oracle_count():
    """The roofline's algorithmic work is the reference's expression tree
    (counted by the oracle's op-counting scalar); the fused formulation the
    kernels run is counted beside it."""
    for metric in (1, 2):
        rhs_f, att_f = O.count_ops(metric, False)
        assert flops.RHS[metric] == rhs_f
        assert flops.attempt_flops(metric) == att_f
        assert flops.IMPLEMENTATION[metric] == O.count_ops(metric, True)
        assert flops.IMPLEMENTATION[metric][1] < att_f


def test_scene_validation_rejects_bad_input():
    s = M.scene_defaults(n_bins=0)
    out = np.zeros(3, dtype=np.float32)
    # validation happens before any device work, so it runs without a GPU
    with pytest.raises(M.MgkError):
        M.xyz_weights(0)
    assert M.lib().mgk_xyz_weights(65, 380.0, 780.0, out.ctypes.data_as(__import__("ctypes").POINTER(
        __import__("ctypes").c_float))) == abi.ERROR_INVALID_ARGUMENT
    del s


# ------------------------------------------------------- oracle physics
def _trace(scene, n=None, first=0):
    n = n or scene.width * scene.height * scene.spp
    return O.trace_rays(scene, first, n)


def test_schwarzschild_shadow_edge_is_sqrt27():
    """Rays from far away with impact parameter b < sqrt(27) M are captured,
    b > sqrt(27) M escape (photon sphere at 3 M)."""
    b_crit = math.sqrt(27.0)
    r_cam = 1000.0
    # a one-row camera whose pixels sweep the impact parameter across b_crit
    w = 64
    s = M.scene_defaults(metric=abi.METRIC_SCHWARZSCHILD, spin=0.0, precision=abi.PRECISION_F64, width=w,
                         height=1, spp=1, cam_r=r_cam, cam_incl_rad=math.radians(90.0), disk_r_out=0.0,
                         escape_radius=2000.0, abs_tol=1e-12, rel_tol=1e-12)
    tan_half = 1.4 * b_crit / r_cam
    s.focal_length_mm = s.sensor_diag_mm / (2 * tan_half)
    r = _trace(s)
    c = M.scene_constants(s)
    px = np.arange(w)
    # camera x of each ray: (px + jx) * pix_a + pix_b with the seeded jitter
    jx = np.array([_jitter(s, p) for p in range(w)])
    sx = (px + jx) * c[24] + c[25]
    b = r_cam * np.abs(sx) / np.sqrt(1 + sx ** 2)
    captured = r["cls"] == abi.RAY_HORIZON
    escaped = r["cls"] == abi.RAY_ESCAPED
    assert (captured | escaped).all()
    margin = 0.02
    assert captured[b < b_crit * (1 - margin)].all()
    assert escaped[b > b_crit * (1 + margin)].all()


def _jitter(s, pixel, dim=0):
    # rng_unit(seed, sample=0, pixel, dim) of the oracle, restated
    def h32(x):
        x &= 0xFFFFFFFF
        x ^= x >> 17; x = (x * 0xED5AD4BB) & 0xFFFFFFFF
        x ^= x >> 11; x = (x * 0xAC4C1B51) & 0xFFFFFFFF
        x ^= x >> 15; x = (x * 0x31848BAB) & 0xFFFFFFFF
        x ^= x >> 14
        return x
    seed = s.seed
    v = h32((seed & 0xFFFFFFFF) ^ 0x9E3779B9)
    v = h32(v ^ (seed >> 32))
    v = h32(v ^ 0)
    v = h32(v ^ pixel)
    v = h32(v ^ ((dim * 0x85EBCA6B + 1) & 0xFFFFFFFF))
    return (v >> 8) / 16777216.0


def _inv_metric_norm(x, p, a):
    """H = g^{mu nu} p_mu p_nu for Kerr-Schild Kerr (spin axis y) at x."""
    X, Y, Z = x[..., 0], x[..., 1], x[..., 2]
    R = X * X + Y * Y + Z * Z - a * a
    r = np.sqrt(0.5 * R + 0.5 * np.sqrt(R * R + 4 * a * a * Y * Y))
    f = 2 * r ** 3 / (r ** 4 + a * a * Y * Y)
    kx = (r * X - a * Z) / (r * r + a * a)
    ky = Y / r
    kz = (r * Z + a * X) / (r * r + a * a)
    # g^{mu nu} = eta^{mu nu} - f k^mu k^nu, k^mu = (1, kx, ky, kz) with eta = diag(-1,1,1,1) and k_t = 1
    pt, px, py, pz = p[..., 3], p[..., 0], p[..., 1], p[..., 2]
    kp = -pt + kx * px + ky * py + kz * pz
    return -pt * pt + px * px + py * py + pz * pz - f * kp * kp


@pytest.mark.parametrize("precision", [abi.PRECISION_F64, abi.PRECISION_MIXED])
def test_null_condition_and_conserved_quantities(precision):
    """H = g^{mu nu} p_mu p_nu stays 0 and p_t, L_y stay constant, to the
    integration tolerance (1e-12 in F64, 1e-7 with FP32 state in MIXED)."""
    tol_kw = dict(rel_tol=1e-12, abs_tol=1e-12) if precision == abi.PRECISION_F64 else {}
    s = M.scene_defaults(width=32, height=18, spp=1, precision=precision, **tol_kw)
    a = -0.9  # the integrated (time-reversed) spin
    r = _trace(s)
    H = _inv_metric_norm(r["x"], r["p"], a)
    lit = (r["cls"] == abi.RAY_DISK) | (r["cls"] == abi.RAY_ESCAPED)
    tol = 1e-9 if precision == abi.PRECISION_F64 else 2e-5
    assert np.abs(H[lit]).max() < tol
    # p_t is conserved exactly; L_y = z p_x - x p_z is conserved by the Kerr flow
    init = O.trace_rays(M.scene_defaults(width=32, height=18, spp=1, precision=precision, max_steps=1, **tol_kw),
                        0, 32 * 18)
    Ly0 = init["x"][:, 2] * init["p"][:, 0] - init["x"][:, 0] * init["p"][:, 2]
    Ly1 = r["x"][:, 2] * r["p"][:, 0] - r["x"][:, 0] * r["p"][:, 2]
    assert np.array_equal(r["p"][:, 3], init["p"][:, 3])
    ok = lit & (init["steps"] == 1)
    rel = np.abs(Ly1[ok] - Ly0[ok]) / (np.abs(Ly0[ok]) + 1.0)
    assert rel.max() < (1e-8 if precision == abi.PRECISION_F64 else 1e-4)


def test_mixed_agrees_with_f64_physics():
    """MIXED (FP32 state and step control, FP64 attempts next to the horizon)
    against F64 on the same rays: termination class, located disk hits and
    escape directions."""
    kw = dict(width=64, height=36, spp=2)
    a = _trace(M.scene_defaults(precision=abi.PRECISION_MIXED, **kw))
    b = _trace(M.scene_defaults(precision=abi.PRECISION_F64, **kw))
    same = a["cls"] == b["cls"]
    assert same.mean() >= 0.999
    disk = same & (a["cls"] == abi.RAY_DISK)
    assert np.quantile(np.abs(a["r_hit"][disk] / b["r_hit"][disk] - 1), 0.99) < 1e-5
    assert np.quantile(np.abs(a["z"][disk] / b["z"][disk] - 1), 0.99) < 1e-5
    esc = same & (a["cls"] == abi.RAY_ESCAPED)
    # escape directions are taken on the escape sphere in both modes
    assert np.quantile(np.abs(a["dir"][esc] - b["dir"][esc]).max(1), 0.99) < 1e-6


def test_weak_field_deflection():
    """A ray passing a Schwarzschild mass at impact parameter b >> M bends by
    4M/b (Einstein), here over the straight-line chord from r_cam back out to
    r_cam: (4M/b) sqrt(1 - (b/r_cam)^2), plus a second-order term
    15 pi M^2 / (4 b^2) of 1.5 % at b = 200 M."""
    b = 200.0
    r_cam = 4000.0
    s = M.scene_defaults(metric=abi.METRIC_SCHWARZSCHILD, spin=0.0, precision=abi.PRECISION_F64, width=1, height=1,
                         spp=1, cam_r=r_cam, cam_incl_rad=math.radians(90.0), disk_r_out=0.0,
                         escape_radius=r_cam, abs_tol=1e-13, rel_tol=1e-13, h_max=200.0, max_steps=100000)
    # the single pixel's jittered direction is (t (2 jx - 1), t (1 - 2 jy), -1) for t = tan(fov/2)
    jx, jy = _jitter(s, 0, 0), _jitter(s, 0, 1)
    tan_b = b / math.sqrt(r_cam ** 2 - b ** 2)
    t = tan_b / math.hypot(2 * jx - 1, 1 - 2 * jy)
    s.focal_length_mm = s.sensor_diag_mm / (2 * t)
    r = _trace(s)
    assert r["cls"][0] == abi.RAY_ESCAPED
    # camera basis at 90 degrees inclination is the identity
    v_in = np.array([t * (2 * jx - 1), t * (1 - 2 * jy), -1.0])
    v_in /= np.linalg.norm(v_in)
    defl = math.acos(np.clip(np.dot(v_in, r["dir"][0]), -1, 1))
    expect = 4.0 / b * math.sqrt(1 - (b / r_cam) ** 2)
    assert abs(defl - expect) / expect < 0.03


def test_disk_emitter_is_normalised():
    """The Keplerian emitter's four-velocity has g(u, u) = -1 (checked through
    the redshift: a face-on ray's z follows from u)."""
    s = M.scene_defaults(width=48, height=27, spp=1, precision=abi.PRECISION_F64)
    r = _trace(s)
    disk = r["cls"] == abi.RAY_DISK
    assert disk.sum() > 50
    # redshift factor g = nu_obs / nu_em of a thin disk seen at 75 degrees lies in (0, ~1.6)
    assert (r["z"][disk] > 0).all() and (r["z"][disk] < 2).all()
    assert np.all((r["r_hit"][disk] >= s.disk_r_in) & (r["r_hit"][disk] <= s.disk_r_out))


def test_sampled_spectral_mode_oracle_splat():
    """The oracle's sampled spectral mode against a numpy restatement: a disk
    hit's wavelength from the inverse CDF table with u = rng(seed, sample,
    pixel, 2), throughput 1/pdf, the boosted blackbody there, the sensor gain,
    and the Gaussian spread over the bins, which with unit X weights sums to
    irradiance * (Phi(lambda_max) - Phi(lambda_min))."""
    s = M.scene_defaults(width=8, height=4, spp=2, precision=abi.PRECISION_F64,
                         spectral_mode=abi.SPECTRAL_SAMPLED, n_bins=24)
    icdf = M.cmf_inverse_cdf(s.lambda_min_nm, s.lambda_max_nm)
    n = 20
    rec = np.zeros(n, dtype=M.RESULT_DTYPE)
    rec["cls"] = abi.RAY_DISK
    rng = np.random.default_rng(5)
    rec["z"] = rng.uniform(0.5, 1.4, n)
    rec["r_hit"] = rng.uniform(s.disk_r_in, s.disk_r_out, n)
    w = np.zeros((s.n_bins, 3), dtype=np.float32)
    w[:, 0] = 1.0
    first = 3
    got = O.shade_rays(s, np.zeros(0, dtype=M.STAR_DTYPE), w, rec, first_ray=first, icdf=icdf)
    h, c, kb = 6.62607015e-34, 299792458.0, 1.380649e-23
    W, H = s.width, s.height
    inv_b = s.sensor_diag_mm / math.sqrt(W * W + H * H)
    gain = (W * inv_b) * (H * inv_b) / 1e6 / (W * H) * s.iso * 2 * math.pi / (360 * s.fps / s.shutter_angle_deg)
    for i in range(n):
        ray = first + i
        u = np.float32(_jitter_dim(s, ray // s.spp, ray % s.spp, 2))
        x = np.float32(u * np.float32(255))
        k = int(min(x, np.float32(254)))
        f = np.float32(x - np.float32(k))
        lam = float(np.float32(icdf[k] * (np.float32(1) - f)) + np.float32(icdf[k + 1] * f))
        tput = float(np.float32(255) * (icdf[k + 1] - icdf[k]))
        z, r = rec["z"][i], rec["r_hit"][i]
        T = s.disk_T_in * (r / s.disk_r_in) ** -0.75
        wl = z * lam * 1e-9
        rad = 2 * h * c * c / wl ** 5 / math.expm1(h * c / (wl * kb * T)) * z ** 5
        irr = rad * tput * gain
        sig = s.redistribution_sigma_nm * math.sqrt(2)
        phi = lambda e: 0.5 * (1 + math.erf((e - lam) / sig))
        expect = irr * (phi(s.lambda_max_nm) - phi(s.lambda_min_nm))
        assert got[i, 0] == pytest.approx(expect, rel=1e-9)
        assert got[i, 1] == 0 and got[i, 2] == 0


def _jitter_dim(s, pixel, sample, dim):
    """rng_unit(seed, sample, pixel, dim) of the library, restated."""
    def h32(x):
        x &= 0xFFFFFFFF
        x ^= x >> 17; x = (x * 0xED5AD4BB) & 0xFFFFFFFF
        x ^= x >> 11; x = (x * 0xAC4C1B51) & 0xFFFFFFFF
        x ^= x >> 15; x = (x * 0x31848BAB) & 0xFFFFFFFF
        x ^= x >> 14
        return x
    v = h32((s.seed & 0xFFFFFFFF) ^ 0x9E3779B9)
    v = h32(v ^ (s.seed >> 32))
    v = h32(v ^ sample)
    v = h32(v ^ pixel)
    v = h32(v ^ ((dim * 0x85EBCA6B + 1) & 0xFFFFFFFF))
    return (v >> 8) / 16777216.0


def test_oracle_scene_and_star_catalog_equal_the_library():
    """The CPU legs build the workload from oracle/ alone: its restated scene
    defaults, ISCO radius and star catalogue are the library's bytes."""
    assert bytes(O.scene_defaults()) == bytes(M.scene_defaults())
    assert O.isco_radius(0.998) == M.isco_radius(0.998)
    a = O.star_catalog(0x57A25, 5000)
    b = M.star_catalog(0x57A25, 5000)
    assert np.array_equal(a.view(np.uint8), b.view(np.uint8))


def test_reference_arm_loads_neither_the_package_nor_libmgk():
    """bench.py --impl reference runs the reference's code (or the oracle)
    only: a fresh process that imports no magik_b200 module and maps no
    libmgk.so, and reports a per-step time that its steps add up to."""
    import json
    import subprocess
    import sys
    code = ("import runpy, sys, json\n"
            "sys.argv = ['bench.py', '--impl', 'reference', '--steps', '2', '--warmup', '0', '--cpu-seconds', '0.2',\n"
            "            '--width', '64', '--height', '36', '--spp', '1']\n"
            "try:\n"
            "    runpy.run_path('bench.py', run_name='__main__')\n"
            "except SystemExit:\n"
            "    pass\n"
            "maps = open('/proc/self/maps').read()\n"
            "print(json.dumps({'libmgk': 'libmgk.so' in maps,\n"
            "                  'pkg': sorted(m for m in sys.modules if m.startswith('magik_b200'))}))\n")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    lines = [json.loads(x) for x in r.stdout.strip().splitlines()]
    line, probe = lines[0], lines[1]
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["package_imported"] is False and probe["libmgk"] is False
    assert probe["pkg"] in ([], ["magik_b200.abi"])  # the ctypes layouts, loaded by path
    assert line["ms_per_step"] > 0 and "REF32" in line["config"]["precision"]


def test_static_entry_refuses_a_short_output_buffer():
    """trace_rays_static checks d_out's size before it calls the library."""
    import torch
    s = M.scene_defaults(width=16, height=16, spp=1)
    with pytest.raises(ValueError):
        M.trace_rays_static(s, 0, 256, torch.empty(256 * 128 - 1, dtype=torch.uint8))
