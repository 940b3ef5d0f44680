"""Pins the CPU oracle to the reference.

The reference ships no tests or known-answer vectors, so the pins are:
  * the reference's own CPU tracer (src/renderer/relativity/host_trace_geodesic.cu,
    compiled unchanged from its sources into oracle/_ref) run here on seeded
    initial conditions: the oracle's REF32 restatement must reproduce its step
    lists bit for bit;
  * golden fixtures of that tracer and of the reference's colour weights,
    generated by tests/golden/make_golden.py, which travel with the repository.
"""
import math
import os

import numpy as np
import pytest

from magik_b200 import abi
from oracle import oracle_py as O
from tests.golden.make_golden import to_structs

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_oracle_reproduces_golden_reference_traces():
    g = np.load(os.path.join(GOLD, "ref_traces.npz"))
    cases, steps, n_written = g["cases"], g["steps"], g["n_written"]
    assert len(cases) >= 40
    for i, c in enumerate(cases):
        rc, a = O.trace_geodesic(*to_structs(c), n_steps=steps.shape[1])
        assert rc == 0
        ref = steps[i, : n_written[i]]
        assert a.shape == ref.shape, (i, a.shape, ref.shape)
        assert np.array_equal(a.view(np.uint32), ref.view(np.uint32)), i


def _random_inputs(rng, count):
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


@pytest.mark.skipif(not O.ref_available(), reason="reference tracer not built (needs the reference sources)")
def test_oracle_bit_exact_with_reference_tracer():
    rng = np.random.default_rng(5)
    ics, mps, ips = _random_inputs(rng, 600)
    for ic, mp, ip in zip(ics, mps, ips):
        rc1, ref = O.ref_trace_geodesic(ic, mp, ip, 300)
        rc2, orc = O.trace_geodesic(ic, mp, ip, 300)
        assert rc1 == rc2 == 0
        assert ref.shape == orc.shape
        assert np.array_equal(ref.view(np.uint32), orc.view(np.uint32))


def test_pow_in_double_stays_close_to_reference():
    """REF32 on the GPU rounds pow() in double; glibc's powf is not always
    correctly rounded, so a few geodesics differ in the last bits of one step
    size.  Those geodesics must stay close to the reference's."""
    g = np.load(os.path.join(GOLD, "ref_traces.npz"))
    exact = 0
    for i, c in enumerate(g["cases"]):
        rc, a = O.trace_geodesic(*to_structs(c), n_steps=g["steps"].shape[1], pow_in_double=True)
        ref = g["steps"][i, : g["n_written"][i]]
        if a.shape == ref.shape and np.array_equal(a.view(np.uint32), ref.view(np.uint32)):
            exact += 1
            continue
        n = min(len(a), len(ref))
        assert abs(len(a) - len(ref)) <= max(2, len(ref) // 10)
        # the first steps agree to a few ulp
        rel = np.abs(a[: min(n, 5), :8] - ref[: min(n, 5), :8]) / (np.abs(ref[: min(n, 5), :8]) + 1e-30)
        assert np.nanmax(rel) < 1e-4
    assert exact >= 0.6 * len(g["cases"])


def test_reference_colour_weights_golden():
    import magik_b200 as M
    g = np.load(os.path.join(GOLD, "ref_cmf_weights.npz"))
    for key in g.files:
        n, lo, hi = key[1:].split("_")
        ref = g[key]
        ours = M.xyz_weights(int(n), float(lo), float(hi))
        # the tabulated CIE 1931 observer, integrated in float as the
        # reference integrates it: the same floats
        assert ours.shape == ref.shape
        assert np.array_equal(ours, ref), key
        # the opt-in analytic fit stays within 1% of the peak weight
        fit = M.xyz_weights(int(n), float(lo), float(hi), analytic=True)
        assert np.abs(fit - ref).max() <= 0.01 * np.abs(ref).max(), key
        # all are normalised so that a flat spectrum has Y = 1 / bin width
        width = (float(hi) - float(lo)) / int(n)
        for w in (ref, ours, fit):
            assert abs(w[:, 1].sum() * width - 1.0) < 1e-5


@pytest.mark.skipif(not O.ref_available(), reason="reference tracer not built (needs the reference sources)")
@pytest.mark.parametrize("metric", [abi.METRIC_KERR, abi.METRIC_SCHWARZSCHILD])
def test_oracle_render_matches_reference_step_render(metric):
    """The oracle's REF32 render against the same render driven by the
    reference's own compiled RKF45 step: the two differ only where the
    reference's powf and the oracle's double pow round a step size apart."""
    import magik_b200 as M
    s = M.scene_defaults(width=48, height=27, spp=1, precision=abi.PRECISION_REF32, metric=metric)
    stars = M.star_catalog(0x57A25, 20000)
    w = M.xyz_weights(s.n_bins)
    n = s.width * s.height
    a, ca = O.render_pixels(s, stars, w, 0, n, nthreads=4)
    b, cb = O.ref_render_pixels(s, stars, w, 0, n, nthreads=4)
    assert np.mean(np.all(a == b, axis=1)) >= 0.98
    assert np.abs(a - b).sum() <= 1e-5 * np.abs(a).sum()
    # the step totals the CPU baselines report: the per-ray records summed
    rec = O.trace_rays(s, 0, n)
    assert ca["steps"] == int(rec["steps"].sum()) and ca["attempts"] == int(rec["attempts"].sum())
    assert abs(cb["steps"] - ca["steps"]) <= 1e-3 * ca["steps"]


def test_reference_inverse_cdf_golden():
    """The sampled spectral mode's CIE inverse CDF table against the
    reference's own (compute_tabulated_cmf_inverse_cdf on its tabulated CIE
    1931 data): the library builds it the same way from the same table, in
    float, so the wavelengths are the same floats."""
    import magik_b200 as M
    g = np.load(os.path.join(GOLD, "ref_cmf_icdf.npz"))
    for key in g.files:
        lo, hi = map(float, key.split("_")[1:])
        ref = g[key]
        ours = M.cmf_inverse_cdf(lo, hi)
        assert ours.shape == ref.shape == (256,)
        assert ours[0] == lo and ours[-1] == hi
        assert np.all(np.diff(ours) >= 0)
        assert np.array_equal(ours, ref), key
        # the opt-in analytic fit: 0.12 nm on average, up to 3 nm in the last
        # entries, where the CMFs vanish and the inverse CDF is steep
        fit = M.cmf_inverse_cdf(lo, hi, analytic=True)
        d = np.abs(fit.astype(np.float64) - ref)
        assert d.mean() < 0.25 and d.max() < 4.0, key


def _display_golden():
    g = np.load(os.path.join(GOLD, "ref_display.npz"))
    from magik_b200 import abi
    settings = [abi.DisplaySettings.from_buffer_copy(s.tobytes()) for s in g["settings"]]
    pipes = [abi.DisplayPipeline.from_buffer_copy(p.tobytes()) for p in g["pipelines"]]
    return g, settings, pipes


def test_display_pipeline_against_reference_golden():
    """mgk_display_prepare against the reference's colour pipeline
    (color_pipeline_descriptor_t::create and the view transforms'
    make_params, from oracle/_ref): every matrix and parameter is the same
    float, the white-balance matrix included (its white point integrates the
    blackbody against the same tabulated CIE 1931 functions in float)."""
    import ctypes as C
    import magik_b200 as M
    from magik_b200 import abi
    g, settings, pipes = _display_golden()
    names = []
    for f, t in abi.DisplayPipeline._fields_[4:]:
        names += [f] * (C.sizeof(t) // 4)
    names = np.array(names)
    for combo, ds, ref in zip(g["combos"], settings, pipes):
        ours = np.frombuffer(bytes(M.display_prepare(ds)), dtype=np.float32)[4:]
        theirs = np.frombuffer(bytes(ref), dtype=np.float32)[4:]
        assert np.array_equal(ours, theirs), (combo, sorted(set(names[ours != theirs])))
