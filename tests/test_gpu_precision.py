"""FP32 integrator against an FP64 run on the GPU, at a size the oracle could
not trace in seconds.

The MIXED mode (FP32 ray state, FP64 error estimate and FP64 attempts within
0.05 M of the horizon) and the F64 mode are both the library's own kernels;
F64 is pinned bit for bit to the CPU oracle by test_gpu_parity.  Here they
trace the same 518,400 camera rays of the Kerr benchmark view (a = 0.9,
r = 50 M, 75 degrees, rtol = atol = 1e-7), and

* the termination class agrees on at least 99.99 % of the rays;
* every ray whose class differs lies near a boundary where an error of the
  integration tolerance can flip it: its disk crossing within 1e-4 of an edge
  of the disk, or its conserved quantities within 2e-3 of the Kerr critical
  curve (the photon ring, where the geodesic flow amplifies a perturbation
  by about e^pi per half orbit);
* escape directions and escape points (on the escape sphere) agree to 1e-6
  at the 99th percentile and 2e-6 at the 99.9th (5.5e-7 and 9e-7 measured
  on the oracle); the rays beyond that are strongly deflected ones (50 or
  more steps, wrapping behind the hole), where the flow amplifies the FP32
  rounding;
* disk radii and redshifts agree to 1e-5 at the 99th percentile;
* against the converged solution (F64 at rtol = atol = 1e-11): MIXED's
  escape directions lie within 1e-6 at the 99th percentile, and its disk
  radii and redshifts within 3x of F64's own error at rtol = 1e-7 at every
  quantile up to the 99.9th (F64 at that tolerance is itself 1e-6 from the
  converged disk radii at the 99th percentile; the two modes take different
  step sequences, since at rtol = 1e-7 the FP32 stages' rounding moves the
  error estimate by several percent).
"""
import math

import numpy as np
import pytest

import magik_b200 as M
from magik_b200 import abi

pytestmark = pytest.mark.gpu

WIDTH, HEIGHT, SPP = 480, 270, 4


def critical_distance(x, p, a):
    """|b - b_c| / b_c of photons (rows of Kerr-Schild x, p; spin axis y, the
    integrated spin a) from the Kerr critical curve of spherical photon
    orbits (Bardeen 1973), vectorised: lambda = L/E, eta = Q/E^2 with
    L = z p_x - x p_z, E = -p_t and the Carter constant from the
    oblate-spheroidal theta (cos theta = y / r)."""
    x = np.asarray(x, np.float64)
    p = np.asarray(p, np.float64)
    X, Y, Z = x[:, 0], x[:, 1], x[:, 2]
    px, py, pz, pt = p[:, 0], p[:, 1], p[:, 2], p[:, 3]
    R = X * X + Y * Y + Z * Z - a * a
    r = np.sqrt(0.5 * R + 0.5 * np.sqrt(R * R + 4 * a * a * Y * Y))
    E, L = -pt, Z * px - X * pz
    ct = Y / r
    st2 = np.maximum(1e-300, 1 - ct * ct)
    st = np.sqrt(st2)
    pth = (ct / st) * (X * px + Z * pz) - r * st * py
    Q = pth * pth + ct * ct * (L * L / st2 - a * a * E * E)
    lam, eta = L / E, Q / (E * E)
    b = np.sqrt(np.maximum(0.0, eta + lam * lam))
    if abs(a) < 1e-3:
        return np.abs(b - math.sqrt(27.0)) / math.sqrt(27.0)
    aa = abs(a)
    r1 = np.full(len(x), 2 * (1 + math.cos(2 / 3 * math.acos(-aa))))
    r2 = np.full(len(x), 2 * (1 + math.cos(2 / 3 * math.acos(aa))))

    def lc(rr):
        return -(rr ** 3 - 3 * rr ** 2 + a * a * rr + a * a) / (a * (rr - 1))

    l1, l2 = lc(r1), lc(r2)
    inside = (lam - l1) * (lam - l2) <= 0
    for _ in range(60):
        rm = 0.5 * (r1 + r2)
        lm = lc(rm)
        left = (lm - lam) * (l1 - lam) > 0
        r1 = np.where(left, rm, r1)
        l1 = np.where(left, lm, l1)
        r2 = np.where(left, r2, rm)
    rs = 0.5 * (r1 + r2)
    etac = rs ** 3 * (4 * a * a - rs * (rs - 3) ** 2) / (a * a * (rs - 1) ** 2)
    bc = np.sqrt(np.maximum(1e-300, etac + lam * lam))
    return np.where(inside, np.abs(b - bc) / bc, np.inf)


def _equatorial_photon(lam, eta, z=1000.0):
    """A photon at (0, 0, z) with L/E = lam and Q/E^2 = eta (E = 1): in the
    equatorial plane p_theta = -r p_y, and L = z p_x."""
    x = np.array([[0.0, 0.0, z, 0.0]])
    p = np.array([[lam / z, -math.sqrt(eta) / z, -1.0, -1.0]])
    return x, p


def test_critical_distance_on_and_off_the_curve():
    """a = 0.9: the spherical photon orbit at r = 3 M has lambda = -1.8 and
    eta = 27 exactly; a photon with those constants lies on the curve (to
    4e-7: at (0, 0, 1000) the spheroidal r is sqrt(1000^2 - a^2), not 1000),
    one with eta 1 % larger does not."""
    a = 0.9
    x, p = _equatorial_photon(-1.8, 27.0)
    assert critical_distance(x, p, a)[0] < 1e-6
    x, p = _equatorial_photon(-1.8, 27.0 * 1.01)
    d = critical_distance(x, p, a)[0]
    assert 1e-3 < d < 1e-2
    # the Schwarzschild limit: the circle b = sqrt(27)
    x, p = _equatorial_photon(3.0, 18.0)
    assert critical_distance(x, p, 0.0)[0] < 1e-12


def test_mixed_against_f64_on_the_gpu(ctx):
    s32 = M.scene_defaults(width=WIDTH, height=HEIGHT, spp=SPP, precision=abi.PRECISION_MIXED)
    s64 = M.scene_defaults(width=WIDTH, height=HEIGHT, spp=SPP, precision=abi.PRECISION_F64)
    n = WIDTH * HEIGHT * SPP
    a = ctx.trace_rays(s32, 0, n)
    b = ctx.trace_rays(s64, 0, n)
    assert (a["cls"] != abi.RAY_ALIVE).all() and (b["cls"] != abi.RAY_ALIVE).all()
    assert (b["cls"] != abi.RAY_STEP_LIMIT).all()

    same = a["cls"] == b["cls"]
    n_diff = int((~same).sum())
    assert same.mean() >= 0.9999, f"{n_diff} of {n} rays change class"

    if n_diff:
        idx = np.nonzero(~same)[0]
        # conserved quantities from the start of each ray (one F64 step in)
        s1 = M.scene_defaults(width=WIDTH, height=HEIGHT, spp=SPP, precision=abi.PRECISION_F64, max_steps=1)
        start = np.concatenate([ctx.trace_rays(s1, int(i), 1) for i in idx])
        a_int = -s64.spin if s64.time_reversed else s64.spin  # the spin as integrated
        dc = critical_distance(start["x"], start["p"], a_int)
        r_hit = np.where(a["cls"][idx] == abi.RAY_DISK, a["r_hit"][idx], b["r_hit"][idx])
        edge = np.minimum(np.abs(r_hit / s64.disk_r_in - 1), np.abs(r_hit / s64.disk_r_out - 1))
        disk_involved = (a["cls"][idx] == abi.RAY_DISK) | (b["cls"][idx] == abi.RAY_DISK)
        near_edge = disk_involved & (edge < 1e-4)
        near_ring = dc < 2e-3
        bad = ~(near_edge | near_ring)
        assert not bad.any(), (
            f"class changes away from any boundary: rays {idx[bad][:8].tolist()}, "
            f"critical distance {dc[bad][:8].tolist()}, disk-edge distance {edge[bad][:8].tolist()}")

    disk = same & (a["cls"] == abi.RAY_DISK)
    esc = same & (a["cls"] == abi.RAY_ESCAPED)
    assert disk.sum() > 10000 and esc.sum() > 10000
    assert np.quantile(np.abs(a["r_hit"][disk] / b["r_hit"][disk] - 1), 0.99) < 1e-5
    assert np.quantile(np.abs(a["z"][disk] / b["z"][disk] - 1), 0.99) < 1e-5
    de = np.abs(a["dir"][esc] - b["dir"][esc]).max(1)
    xe = np.linalg.norm(a["x"][esc][:, :3] - b["x"][esc][:, :3], axis=1) / np.linalg.norm(b["x"][esc][:, :3], axis=1)
    print(f"escape direction MIXED vs F64: p99 {np.quantile(de, 0.99):.2e} p99.9 {np.quantile(de, 0.999):.2e} "
          f"p99.99 {np.quantile(de, 0.9999):.2e}; escape point p99 {np.quantile(xe, 0.99):.2e}")
    assert np.quantile(de, 0.99) <= 1e-6 and np.quantile(de, 0.999) <= 2e-6
    assert np.quantile(xe, 0.99) <= 1e-6 and np.quantile(xe, 0.999) <= 2e-6
    # the escape point lies on the escape sphere
    assert np.abs(np.linalg.norm(a["x"][esc][:, :3], axis=1) / s32.escape_radius - 1).max() < 1e-5
    # the FP64 band ran: MIXED took FP64 attempts near the horizon
    assert a["wide_attempts"].sum() > 0


def test_mixed_is_as_accurate_as_f64_at_the_same_tolerance(ctx):
    conv = M.scene_defaults(width=WIDTH, height=HEIGHT, spp=SPP, precision=abi.PRECISION_F64,
                            rel_tol=1e-11, abs_tol=1e-11)
    s32 = M.scene_defaults(width=WIDTH, height=HEIGHT, spp=SPP, precision=abi.PRECISION_MIXED)
    s64 = M.scene_defaults(width=WIDTH, height=HEIGHT, spp=SPP, precision=abi.PRECISION_F64)
    n = WIDTH * HEIGHT * SPP
    c = ctx.trace_rays(conv, 0, n)
    a = ctx.trace_rays(s32, 0, n)
    b = ctx.trace_rays(s64, 0, n)
    assert (c["cls"] != abi.RAY_STEP_LIMIT).all()
    same = (a["cls"] == c["cls"]) & (b["cls"] == c["cls"])
    assert same.mean() >= 0.9999
    disk = same & (c["cls"] == abi.RAY_DISK)
    esc = same & (c["cls"] == abi.RAY_ESCAPED)
    q = np.array([0.5, 0.9, 0.99, 0.999])

    def err(r, field, sel):
        if field == "dir":
            return np.abs(r["dir"][sel] - c["dir"][sel]).max(1)
        return np.abs(r[field][sel] / c[field][sel] - 1)

    de_m, de_f = np.quantile(err(a, "dir", esc), q), np.quantile(err(b, "dir", esc), q)
    print(f"dir vs converged: MIXED {np.array2string(de_m, precision=2)} F64@1e-7 {np.array2string(de_f, precision=2)}")
    assert de_m[2] <= 1e-6
    for field in ("r_hit", "z"):
        em, ef = np.quantile(err(a, field, disk), q), np.quantile(err(b, field, disk), q)
        print(f"{field} vs converged: MIXED {np.array2string(em, precision=2)} F64@1e-7 {np.array2string(ef, precision=2)}")
        assert np.all(em <= 3.0 * ef + 1e-8), (field, em.tolist(), ef.tolist())
