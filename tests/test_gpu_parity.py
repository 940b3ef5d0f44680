"""GPU parity: libmgk's sm_100a kernels against the CPU oracle, through the C ABI.

REF32 and MIXED are defined so that the kernels and the oracle round every
operation identically, and F64 likewise; the per-ray records must therefore
match bit for bit.  The only tolerated difference is the last-bit rounding of
pow() in the step proposal (CUDA's double pow vs the C library's), which can
flip one float h in roughly 1e-8 of the attempts.
"""
import math

import numpy as np
import pytest

import magik_b200 as M
from magik_b200 import abi
from oracle import oracle_py as O
from tests.conftest import room_scene, small_scene

pytestmark = pytest.mark.gpu

FIELDS = ["cls", "steps", "attempts", "wide_attempts", "refine_evals", "bounces", "x", "p", "z", "r_hit", "dir"]


def scene_for(metric, precision, **kw):
    if metric == abi.METRIC_SCHWARZSCHILD:
        # the Schwarzschild workload: r = 30 M, 80 degrees, disk 6-20 M, 16 bins, rtol 1e-8 / atol 1e-10
        base = dict(metric=metric, spin=0.0, cam_r=30.0, cam_incl_rad=math.radians(80.0), disk_r_in=6.0,
                    n_bins=16, rel_tol=1e-8, abs_tol=1e-10 if precision == abi.PRECISION_F64 else 1e-7)
    elif metric == abi.METRIC_MINKOWSKI:
        base = dict(metric=metric, spin=0.0, disk_r_in=6.0)
    else:
        base = dict(metric=metric)
    base.update(precision=precision)
    base.update(kw)
    return small_scene(**base)


def compare_records(gpu, orc, allow_frac=1e-3):
    assert gpu.shape == orc.shape
    same = np.ones(len(gpu), dtype=bool)
    for f in FIELDS:
        a, b = gpu[f], orc[f]
        if a.dtype.kind == "f":
            eq = (a.view(np.uint64) == b.view(np.uint64)) | (np.isnan(a) & np.isnan(b))
        else:
            eq = a == b
        if eq.ndim > 1:
            eq = eq.all(axis=1)
        same &= eq
    n_bad = int((~same).sum())
    assert n_bad <= max(1, int(allow_frac * len(gpu))), f"{n_bad} of {len(gpu)} rays differ"
    # rays that differ (pow rounding) still agree in class: the 99.99 % bar
    assert np.mean(gpu["cls"] == orc["cls"]) >= 0.9999
    return n_bad


@pytest.mark.parametrize("metric", [abi.METRIC_KERR, abi.METRIC_SCHWARZSCHILD, abi.METRIC_MINKOWSKI])
@pytest.mark.parametrize("precision", [abi.PRECISION_REF32, abi.PRECISION_MIXED, abi.PRECISION_F64])
def test_trace_rays_bit_exact(ctx, metric, precision):
    s = scene_for(metric, precision)
    n = s.width * s.height * s.spp
    gpu = ctx.trace_rays(s, 0, n)
    orc = O.trace_rays(s, 0, n)
    compare_records(gpu, orc)
    assert (gpu["cls"] != abi.RAY_ALIVE).all()


def test_mixed_sqrt_and_reciprocal_match_their_definitions(ctx):
    """The MIXED fused RHS's square root and reciprocal (hardware approximation
    plus one FMA correction) equal their definitions, which the oracle
    restates, on every one of the 2^32 float inputs."""
    assert ctx.check_rounding() == (0, 0)


def test_peak_probes(ctx):
    """The roofline denominators: FP32 and FP64 FMA throughput of this device
    within the physical bounds of 148 SMs x 128 FP32 lanes at 2.1 GHz."""
    p32, p64 = ctx.fp32_peak(), ctx.fp64_peak()
    assert 1e13 < p32 < 148 * 128 * 2 * 2.1e9
    assert 1e11 < p64 <= p32


def test_trace_rays_offset_range(ctx):
    """A range that starts mid-frame and is not pixel aligned."""
    s = small_scene(spp=3)
    gpu = ctx.trace_rays(s, 1001, 777)
    orc = O.trace_rays(s, 1001, 777)
    compare_records(gpu, orc)


def test_mixed_band_and_refine_paths_exercised(ctx):
    """Rays that enter the FP64 band near the horizon and rays whose chord
    suggested the disk but missed it go through the tail kernel."""
    s = small_scene(width=96, height=54, spp=1, spin=0.998, disk_r_in=M.isco_radius(0.998), cam_r=20.0,
                    cam_incl_rad=math.radians(85.0))
    n = s.width * s.height
    gpu = ctx.trace_rays(s, 0, n)
    orc = O.trace_rays(s, 0, n)
    compare_records(gpu, orc)
    assert gpu["wide_attempts"].sum() > 0
    assert (gpu["refine_evals"] > 0).sum() > 0


def test_render_stats_match_per_ray_records(ctx):
    import torch
    s = small_scene()
    n = s.width * s.height * s.spp
    rec = ctx.trace_rays(s, 0, n)
    film = torch.empty(s.width * s.height * 3, dtype=torch.float32, device="cuda")
    st = ctx.render(s, None, film)
    assert st.rays == n
    assert st.attempts == int(rec["attempts"].sum())
    assert st.steps == int(rec["steps"].sum())
    assert st.refine_evals == int(rec["refine_evals"].sum())
    counts = np.bincount(rec["cls"], minlength=abi.RAY_CLASSES)
    assert list(st.class_count) == [int(c) for c in counts]


def _stars(n, seed=7):
    return M.star_catalog(seed, n)


def _film_rel_err(a, b):
    scale = np.maximum(np.abs(b), 1e-6 * np.abs(b).max())
    return np.abs(a - b) / scale


@pytest.mark.parametrize("precision", [abi.PRECISION_MIXED, abi.PRECISION_F64, abi.PRECISION_REF32])
def test_render_film_matches_oracle(ctx, precision):
    import torch
    s = small_scene(precision=precision, star_radius_rad=0.02)
    stars = _stars(20000)
    w = M.xyz_weights(s.n_bins)
    npix = s.width * s.height
    film = torch.empty(npix * 3, dtype=torch.float32, device="cuda")
    spec = torch.empty(npix * s.n_bins, dtype=torch.float32, device="cuda")
    d_stars = torch.from_numpy(stars.view(np.uint8)).cuda()
    d_w = torch.from_numpy(w.ravel()).cuda()
    ctx.render(s, d_stars, film, d_weights=d_w, d_film_spectral=spec)
    got = film.cpu().numpy().reshape(npix, 3).astype(np.float64)
    ref, _ = O.render_pixels(s, stars, w, 0, npix)
    err = _film_rel_err(got, ref)
    assert np.isfinite(got).all() and (got >= 0).all()
    assert err.max() <= 1e-4, err.max()
    # the spectral film integrates to the same XYZ with the bin weights
    sp = spec.cpu().numpy().reshape(npix, s.n_bins).astype(np.float64)
    xyz_from_spec = sp @ w.astype(np.float64)
    assert _film_rel_err(xyz_from_spec, got).max() <= 1e-4
    # some pixels see stars, some the disk
    assert (ref[:, 1] > 0).mean() > 0.2


@pytest.mark.parametrize("precision", [abi.PRECISION_MIXED, abi.PRECISION_F64])
def test_render_sampled_spectral_mode_matches_oracle(ctx, precision):
    """The reference's stochastic sensor (MGK_SPECTRAL_SAMPLED): one CIE
    inverse-CDF wavelength per ray, Gaussian redistribution over the bins."""
    import torch
    s = small_scene(precision=precision, star_radius_rad=0.02, spectral_mode=abi.SPECTRAL_SAMPLED, n_bins=24)
    stars = _stars(20000)
    w = M.xyz_weights(s.n_bins)
    icdf = M.cmf_inverse_cdf(s.lambda_min_nm, s.lambda_max_nm)
    npix = s.width * s.height
    film = torch.empty(npix * 3, dtype=torch.float32, device="cuda")
    spec = torch.empty(npix * s.n_bins, dtype=torch.float32, device="cuda")
    d_stars = torch.from_numpy(stars.view(np.uint8)).cuda()
    d_w = torch.from_numpy(w.ravel()).cuda()
    ctx.render(s, d_stars, film, d_weights=d_w, d_film_spectral=spec)
    got = film.cpu().numpy().reshape(npix, 3).astype(np.float64)
    ref, _ = O.render_pixels(s, stars, w, 0, npix, icdf=icdf)
    assert np.isfinite(got).all() and (got >= 0).all()
    assert _film_rel_err(got, ref).max() <= 1e-4
    sp = spec.cpu().numpy().reshape(npix, s.n_bins).astype(np.float64)
    assert _film_rel_err(sp @ w.astype(np.float64), got).max() <= 1e-4
    assert (ref[:, 1] > 0).mean() > 0.2
    # the per-ray path as well
    n = s.width * s.height * s.spp
    xyz = ctx.shade_rays(s, stars, w, 0, n).astype(np.float64)
    rec = O.trace_rays(s, 0, n)
    assert _film_rel_err(xyz, O.shade_rays(s, stars, w, rec, icdf=icdf)).max() <= 1e-4


def test_shade_rays_matches_oracle(ctx):
    s = small_scene(star_radius_rad=0.02)
    stars = _stars(20000)
    w = M.xyz_weights(s.n_bins)
    n = s.width * s.height * s.spp
    xyz = ctx.shade_rays(s, stars, w, 0, n).astype(np.float64)
    rec = O.trace_rays(s, 0, n)
    ref = O.shade_rays(s, stars, w, rec)
    assert _film_rel_err(xyz, ref).max() <= 1e-4


def test_render_host_equals_device_render(ctx):
    import torch
    s = small_scene()
    stars = _stars(5000)
    npix = s.width * s.height
    film = torch.empty(npix * 3, dtype=torch.float32, device="cuda")
    ctx.render(s, torch.from_numpy(stars.view(np.uint8)).cuda(), film)
    host = np.zeros(npix * 3, dtype=np.float32)
    ctx.render_host(s, stars, host)
    assert np.array_equal(host, film.cpu().numpy())


def _random_trace_inputs(rng, count):
    ics, mps, ips = [], [], []
    mass = 6.7329546075e26
    for trial in range(count):
        metric = trial % 3
        mps.append(abi.TraceMetricParams(metric, bool(rng.integers(0, 2)), 1.01,
                                         mass * (1 if rng.random() < 0.9 else -1), mass,
                                         float(rng.uniform(-0.999, 0.999))))
        ips.append(abi.TraceIntegratorParams(int(rng.integers(1, 60)), float(10 ** rng.uniform(-10, -3)),
                                             float(10 ** rng.uniform(-10, -3))))
        r = rng.uniform(3, 40)
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        ics.append(abi.TraceInitialConditions(
            abi.MASSLESS if rng.random() < 0.8 else abi.MASSIVE, *(d * r).astype(np.float32).tolist(),
            *rng.uniform(-math.pi, math.pi, 3).astype(np.float32).tolist(),
            *(rng.normal(size=3) * 1e7).astype(np.float32).tolist(), float(rng.uniform(0, 2e8))))
    return ics, mps, ips


def test_drop_in_trace_geodesic_batch(ctx):
    """The reference-compatible trace on the GPU equals the oracle step list
    bit for bit (pow in double, as the kernels round it)."""
    rng = np.random.default_rng(11)
    ics, mps, ips = _random_trace_inputs(rng, 240)
    gpu = ctx.trace_geodesic_batch(ics, mps, ips, 300)
    bad = 0
    for i in range(len(ics)):
        rc, orc = O.trace_geodesic(ics[i], mps[i], ips[i], 300, pow_in_double=True)
        assert rc == 0
        if not (orc.shape == gpu[i].shape and np.array_equal(orc.view(np.uint32), gpu[i].view(np.uint32))):
            bad += 1
    assert bad <= 1, bad


def test_drop_in_matches_reference_tracer(ctx):
    """Against the reference's own CPU tracer (built from its sources): the
    same accepted-step count and final state to 1e-5 on geodesics where
    glibc's powf rounds like the correctly rounded pow."""
    if not O.ref_available():
        pytest.skip("reference tracer not built")
    rng = np.random.default_rng(12)
    ics, mps, ips = _random_trace_inputs(rng, 120)
    gpu = ctx.trace_geodesic_batch(ics, mps, ips, 300)
    exact = 0
    for i in range(len(ics)):
        rc, ref = O.ref_trace_geodesic(ics[i], mps[i], ips[i], 300)
        assert rc == 0
        if ref.shape == gpu[i].shape and np.array_equal(ref.view(np.uint32), gpu[i].view(np.uint32)):
            exact += 1
    assert exact >= 0.7 * len(ics), exact


def test_magik_trace_geodesic_entry_point():
    ic = abi.TraceInitialConditions(abi.MASSLESS, 15.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0)
    mp = abi.TraceMetricParams(abi.METRIC_KERR, True, 1.01, 6.7329546075e26, 6.7329546075e26, 0.9)
    ip = abi.TraceIntegratorParams(56, 1e-3, 1e-10)
    rc, steps = M.trace_geodesic(ic, mp, ip, 512)
    assert rc == 0
    rc2, orc = O.trace_geodesic(ic, mp, ip, 512, pow_in_double=True)
    assert np.array_equal(steps.view(np.uint32), orc.view(np.uint32))
    # capacity mismatch is reported like the reference (magik.cpp:198-200)
    bad = abi.TraceContainer(7, 512, 0, None)
    assert M.lib().magik_trace_geodesic(bad, ic, mp, ip) == abi.ERROR_INVALID_POINTER


# ------------------------------------------------------------------ room
@pytest.mark.parametrize("metric", [abi.METRIC_KERR, abi.METRIC_SCHWARZSCHILD, abi.METRIC_MINKOWSKI])
@pytest.mark.parametrize("precision", [abi.PRECISION_REF32, abi.PRECISION_MIXED, abi.PRECISION_F64])
def test_room_trace_rays_bit_exact(ctx, metric, precision):
    """The box-and-light scene: wall and light crossings located on the
    geodesic, reflections in the wall's rest frame (mirror / Lambertian with
    the ray's own random numbers), the reflection cap; every record equal to
    the oracle's, bounces included."""
    s = room_scene(metric=metric, spin=0.9 if metric == abi.METRIC_KERR else 0.0, precision=precision)
    n = s.width * s.height * s.spp
    gpu = ctx.trace_rays(s, 0, n)
    orc = O.trace_rays(s, 0, n)
    compare_records(gpu, orc)
    counts = np.bincount(gpu["cls"], minlength=abi.RAY_CLASSES)
    assert counts[abi.RAY_ALIVE] == 0 and counts[abi.RAY_LIGHT] > 0
    assert gpu["bounces"].max() == s.room_reflection_limit + 1


def test_room_offset_range_and_disk(ctx):
    """A mid-frame range (the reflection random numbers follow the global ray
    index) in a room that also holds the disk (disk hits before wall exits)."""
    s = room_scene(disk_r_out=12.0, spp=3)
    gpu = ctx.trace_rays(s, 1001, 777)
    orc = O.trace_rays(s, 1001, 777)
    compare_records(gpu, orc)
    assert (gpu["cls"] == abi.RAY_DISK).any() and (gpu["cls"] == abi.RAY_LIGHT).any()


@pytest.mark.parametrize("sampled", [False, True])
@pytest.mark.parametrize("precision", [abi.PRECISION_MIXED, abi.PRECISION_F64])
def test_room_render_film_matches_oracle(ctx, precision, sampled):
    import torch
    kw = dict(spectral_mode=abi.SPECTRAL_SAMPLED, n_bins=24) if sampled else {}
    s = room_scene(precision=precision, **kw)
    w = M.xyz_weights(s.n_bins)
    icdf = M.cmf_inverse_cdf(s.lambda_min_nm, s.lambda_max_nm) if sampled else None
    npix = s.width * s.height
    film = torch.empty(npix * 3, dtype=torch.float32, device="cuda")
    st = ctx.render(s, None, film, d_weights=torch.from_numpy(w.ravel()).cuda())
    got = film.cpu().numpy().reshape(npix, 3).astype(np.float64)
    ref, _ = O.render_pixels(s, np.zeros(0, M.STAR_DTYPE), w, 0, npix, icdf=icdf)
    assert np.isfinite(got).all() and (got >= 0).all()
    assert _film_rel_err(got, ref).max() <= 1e-4
    assert (ref[:, 1] > 0).mean() > 0.1
    rec = ctx.trace_rays(s, 0, npix * s.spp)
    counts = np.bincount(rec["cls"], minlength=abi.RAY_CLASSES)
    assert list(st.class_count) == [int(c) for c in counts]
    # a ray stopped by the cap counts limit + 1 bounces but did not reflect the last time
    assert st.reflections == int(np.minimum(rec["bounces"], s.room_reflection_limit).sum())


def test_room_scene_validation(ctx):
    import torch
    film = torch.empty(48 * 27 * 3, dtype=torch.float32, device="cuda")
    bad = [dict(cam_r=60.0),                                   # camera outside the room
           dict(cam_r=19.5, cam_incl_rad=0.0),                 # camera inside the light
           dict(room_min=(40.0, -20.0, -40.0)),                # empty room
           dict(light_scale=float("nan")),
           dict(room_reflection_limit=5000)]
    for kw in bad:
        s = room_scene()
        for k, v in kw.items():
            if isinstance(v, tuple):
                getattr(s, k)[:] = v
            else:
                setattr(s, k, v)
        with pytest.raises(M.MgkError) as e:
            ctx.render(s, None, film)
        assert e.value.code == abi.ERROR_INVALID_ARGUMENT, kw


def test_render_pass_histories(ctx):
    """Per-pass statistics: without the room two passes (the disk misses take
    the second); with it one pass per reflection plus one; rays carried from
    each pass to the next, hits summing to the emitter classes, crossings and
    tail hand-offs summing to the totals."""
    import torch
    s = small_scene()
    film = torch.empty(s.width * s.height * 3, dtype=torch.float32, device="cuda")
    st = ctx.render(s, None, film)
    n = s.width * s.height * s.spp
    # the disk misses take one more pass of the integrator
    assert st.n_passes == 2 and st.pass_rays[0] == n and st.pass_rays[1] == st.pass_continued[0] > 0
    assert st.pass_continued[1] == 0
    assert sum(st.pass_to_tail[:2]) == st.resumed and sum(st.pass_crossings[:2]) == st.crossings
    r = room_scene()
    st = ctx.render(r, None, film)
    L = r.room_reflection_limit
    assert st.n_passes == L + 2 and st.pass_rays[0] == n
    for p in range(st.n_passes - 1):
        assert st.pass_rays[p + 1] == st.pass_continued[p]
    cls = st.class_count
    assert sum(st.pass_hits[:st.n_passes]) == cls[abi.RAY_LIGHT] + cls[abi.RAY_DISK] + cls[abi.RAY_ESCAPED]
    assert sum(st.pass_crossings[:st.n_passes]) == st.crossings
    assert sum(st.pass_to_tail[:st.n_passes]) == st.resumed


# --------------------------------------------------------------- edge cases
def test_empty_and_single_ray_calls(ctx):
    import torch
    s = small_scene()
    assert len(ctx.trace_rays(s, 0, 0)) == 0
    assert len(ctx.shade_rays(s, None, M.xyz_weights(s.n_bins), 5, 0)) == 0
    # the last ray of the frame alone
    n = s.width * s.height * s.spp
    compare_records(ctx.trace_rays(s, n - 1, 1), O.trace_rays(s, n - 1, 1))
    # past the frame: refused
    with pytest.raises(M.MgkError):
        ctx.trace_rays(s, n - 1, 2)
    # a 1 x 1 frame at one sample
    t = small_scene(width=1, height=1, spp=1)
    film = torch.empty(3, dtype=torch.float32, device="cuda")
    ctx.render(t, None, film)
    ref, _ = O.render_pixels(t, np.zeros(0, M.STAR_DTYPE), M.xyz_weights(t.n_bins), 0, 1)
    assert np.allclose(film.cpu().numpy().reshape(1, 3).astype(np.float64), ref, rtol=1e-4, atol=0.0)


@pytest.mark.parametrize("precision", [abi.PRECISION_REF32, abi.PRECISION_MIXED, abi.PRECISION_F64])
def test_step_cap_and_camera_in_the_disk_plane(ctx, precision):
    """Rays stopped by a small step cap, and a camera in the disk plane
    (rays that start with y = 0, where the disk's chord test sees no sign
    change): records equal to the oracle's."""
    s = small_scene(precision=precision, max_steps=7)
    n = s.width * s.height * s.spp
    gpu = ctx.trace_rays(s, 0, n)
    compare_records(gpu, O.trace_rays(s, 0, n))
    assert (gpu["cls"] == abi.RAY_STEP_LIMIT).mean() > 0.5 and gpu["steps"].max() <= 7
    e = small_scene(precision=precision, cam_incl_rad=math.pi / 2)
    compare_records(ctx.trace_rays(e, 0, n), O.trace_rays(e, 0, n))


def test_maximum_bins(ctx):
    """MGK_MAX_BINS spectral bins, with the spectral film."""
    import torch
    s = small_scene(n_bins=abi.MAX_BINS, star_radius_rad=0.02, width=32, height=18)
    stars = _stars(5000)
    w = M.xyz_weights(s.n_bins)
    npix = s.width * s.height
    film = torch.empty(npix * 3, dtype=torch.float32, device="cuda")
    spec = torch.empty(npix * s.n_bins, dtype=torch.float32, device="cuda")
    ctx.render(s, torch.from_numpy(stars.view(np.uint8)).cuda(), film,
               d_weights=torch.from_numpy(w.ravel()).cuda(), d_film_spectral=spec)
    ref, _ = O.render_pixels(s, stars, w, 0, npix)
    got = film.cpu().numpy().reshape(npix, 3).astype(np.float64)
    assert _film_rel_err(got, ref).max() <= 1e-4
    sp = spec.cpu().numpy().reshape(npix, s.n_bins).astype(np.float64)
    assert _film_rel_err(sp @ w.astype(np.float64), got).max() <= 1e-4
