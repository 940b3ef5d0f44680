"""The room scene (the reference's box-and-light test stage) on the CPU: the
oracle's pieces against the reference's own code where it runs on the host
(the white-LED spectrum; the mirror reflection composed from its frame
functions), the chord test against brute force, the Lambertian directions
against their distribution, and whole rays against the scene's invariants."""
import math

import numpy as np
import pytest

import magik_b200 as M
from magik_b200 import abi
from oracle import oracle_py as O
from tests.conftest import room_scene

needs_ref = pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built (reference sources absent)")


@needs_ref
def test_white_led_matches_reference():
    for lam in np.linspace(300.0, 900.0, 601):
        want = O.ref_white_led(lam)
        assert O.white_led(lam) == pytest.approx(want, rel=2e-6, abs=1e-30)


def _wall_states(scene, rng, count, axis, side):
    """Null momenta at points of one wall: Lambertian reflections (the
    oracle's) of arbitrary states, so that p is null in the scene's metric."""
    out = []
    lo, hi = np.array(scene.room_min), np.array(scene.room_max)
    for i in range(count):
        x = np.zeros(4, np.float32)
        x[:3] = rng.uniform(lo * 0.9, hi * 0.9)
        x[axis] = hi[axis] if side else lo[axis]
        x[3] = rng.uniform(0, 100)
        p0 = np.array([*rng.normal(size=3), -1.0], np.float32)
        b = (axis + 1) % 3  # a Lambertian wall other than the mirror
        _, p, c0 = O.reflect_wall(scene, x, p0, b if b else 1, 0, 1.0, 0, 1000 + i)
        out.append((x, p, c0))
    return out


@needs_ref
@pytest.mark.parametrize("metric", [abi.METRIC_KERR, abi.METRIC_SCHWARZSCHILD])
def test_mirror_reflection_matches_reference(metric):
    """Walls normal to x mirror in their rest frame: the oracle's reflection
    against the reference's generate_material_context / vector_reflect /
    apply_reflected chain (its own compute_inv_g, tetrad and frame changes),
    in float."""
    s = room_scene(metric=metric, spin=0.9 if metric == abi.METRIC_KERR else 0.0, precision=abi.PRECISION_MIXED)
    rng = np.random.default_rng(5)
    worst = 0.0
    for side in (0, 1):
        for x, p, c0 in _wall_states(s, rng, 100, 0, side):
            xo, po, co = O.reflect_wall(s, x, p, 0, side, c0)
            n = np.array([-1.0 if side else 1.0, 0.0, 0.0], np.float32)
            pr, cr = O.ref_reflect_mirror(s, x, p, n, c0)
            scale = np.abs(pr).max()
            worst = max(worst, np.abs(po - pr).max() / scale, abs(co - cr) / abs(cr))
            # restart 1/256 inside the wall
            assert xo[0] == np.float32((s.room_max[0] - 1 / 256) if side else (s.room_min[0] + 1 / 256))
    assert worst < 2e-5, worst


def test_lambertian_is_cosine_weighted():
    """Flat space (rest frame = coordinate frame): floor reflections are
    distributed with density cos(theta) / pi about the normal, azimuth uniform."""
    s = room_scene(metric=abi.METRIC_MINKOWSKI, spin=0.0)
    x = np.array([3.0, s.room_min[1], -5.0, 0.0], np.float32)
    p_in = np.array([0.3, -0.8, 0.2, -1.0], np.float32)
    cos_t, phi = [], []
    for i in range(20000):
        _, p, _ = O.reflect_wall(s, x, p_in, 1, 0, 1.0, i % 7, i)
        d = p[:3] / np.linalg.norm(p[:3])
        cos_t.append(d[1])
        phi.append(math.atan2(d[2], d[0]))
    cos_t, phi = np.array(cos_t), np.array(phi)
    assert (cos_t >= 0).all()
    # CDF of cos(theta) under density 2 c on [0, 1] is c^2
    ks = np.abs(np.sort(cos_t) ** 2 - (np.arange(len(cos_t)) + 0.5) / len(cos_t)).max()
    assert ks < 0.015, ks
    assert abs(cos_t.mean() - 2 / 3) < 0.01
    hist = np.histogram(phi, bins=12, range=(-math.pi, math.pi))[0]
    assert hist.min() > 0.9 * hist.mean() and hist.max() < 1.1 * hist.mean()


def _brute_event(s, p0, p1, n=20001):
    t = np.linspace(0.0, 1.0, n)
    pts = p0[None, :] + t[:, None] * (p1 - p0)[None, :]
    lo, hi = np.array(s.room_min), np.array(s.room_max)
    llo, lhi = np.array(s.light_min), np.array(s.light_max)
    out = ((pts < lo) | (pts > hi)).any(axis=1)
    inl = ((pts >= llo) & (pts <= lhi)).all(axis=1)
    tw = t[np.argmax(out)] if out.any() else 2.0
    tl = t[np.argmax(inl)] if inl.any() else 2.0
    return tw, tl


def test_room_chord_event_against_brute_force():
    s = room_scene()
    rng = np.random.default_rng(11)
    lo, hi = np.array(s.room_min), np.array(s.room_max)
    checked = {"wall": 0, "light": 0, "none": 0}
    for _ in range(3000):
        p0 = rng.uniform(lo, hi)
        if (p0 >= np.array(s.light_min)).all() and (p0 <= np.array(s.light_max)).all():
            continue
        p1 = p0 + rng.normal(size=3) * rng.choice([2.0, 20.0, 80.0])
        t, axis, side, light = O.room_event(s, p0, p1)
        tw, tl = _brute_event(s, p0, p1)
        if axis < 0:
            assert tw == 2.0 and tl == 2.0
            checked["none"] += 1
            continue
        if light:
            assert abs(t - tl) <= 1e-4 and tl <= tw + 1e-4
            plane = s.light_max[axis] if side else s.light_min[axis]
            checked["light"] += 1
        else:
            assert abs(t - tw) <= 1e-4 and tw <= tl + 1e-4
            plane = s.room_max[axis] if side else s.room_min[axis]
            checked["wall"] += 1
        assert abs(p0[axis] + t * (p1[axis] - p0[axis]) - plane) <= 1e-9 * max(1.0, abs(plane))
    assert min(checked.values()) > 50, checked


@pytest.mark.parametrize("precision", [abi.PRECISION_MIXED, abi.PRECISION_F64, abi.PRECISION_REF32])
def test_room_rays_respect_the_scene(precision):
    s = room_scene(precision=precision, width=40, height=24, spp=1)
    r = O.trace_rays(s, 0, s.width * s.height)
    cls = r["cls"]
    counts = np.bincount(cls, minlength=abi.RAY_CLASSES)
    # nothing escapes the room; the light, the horizon and the reflection cap end rays
    assert counts[abi.RAY_ESCAPED] == 0 and counts[abi.RAY_ALIVE] == 0
    assert counts[abi.RAY_LIGHT] > 0 and counts[abi.RAY_HORIZON] > 0
    assert r["bounces"].max() == s.room_reflection_limit + 1
    capped = (cls == abi.RAY_STEP_LIMIT) & (r["steps"] < s.max_steps)
    assert (r["bounces"][capped] == s.room_reflection_limit + 1).all()
    assert (r["bounces"] <= s.room_reflection_limit + 1).all()
    # every ray ends inside the room (walls restart 1/256 inside, hits lie on faces)
    lo, hi = np.array(s.room_min), np.array(s.room_max)
    x = r["x"][:, :3]
    assert ((x >= lo - 1e-3) & (x <= hi + 1e-3)).all()
    lit = cls == abi.RAY_LIGHT
    assert np.isfinite(r["z"][lit]).all() and (r["z"][lit] > 0).all()
    # light hits lie on a face of the light box
    xl = x[lit]
    on_face = np.zeros(len(xl), bool)
    for a in range(3):
        for b in (s.light_min[a], s.light_max[a]):
            on_face |= np.abs(xl[:, a] - b) < 1e-3
    assert on_face.all()


def test_room_reflection_limit_zero_ends_rays_at_the_first_wall():
    s = room_scene(room_reflection_limit=0, width=24, height=16, spp=1)
    r = O.trace_rays(s, 0, s.width * s.height)
    assert r["bounces"].max() == 1
    assert set(np.unique(r["cls"])) <= {abi.RAY_LIGHT, abi.RAY_HORIZON, abi.RAY_STEP_LIMIT}


def test_room_light_emission_is_the_boosted_led():
    """The light's XYZ: LED(z lambda) * scale * z^5 through the bin weights."""
    s = room_scene(width=24, height=16, spp=1)
    n = s.width * s.height
    r = O.trace_rays(s, 0, n)
    w = M.xyz_weights(s.n_bins)
    xyz = O.shade_rays(s, None, w, r)
    lit = np.flatnonzero(r["cls"] == abi.RAY_LIGHT)
    assert len(lit) > 0
    dl = (s.lambda_max_nm - s.lambda_min_nm) / s.n_bins
    lam = s.lambda_min_nm + (np.arange(s.n_bins) + 0.5) * dl
    for i in lit[:20]:
        z = r["z"][i]
        spec = np.array([O.white_led(z * l) for l in lam]) * s.light_scale * z ** 5
        assert np.allclose(spec @ w.astype(np.float64), xyz[i], rtol=1e-5)
    dark = r["cls"] != abi.RAY_LIGHT
    assert (xyz[dark] == 0).all()
