"""Generates the golden fixtures of the reference's own CPU code.

Run in a container where the reference sources are present (oracle/Makefile
builds oracle/_ref/libmagikref.so from them):

    make -C oracle && python tests/golden/make_golden.py

Writes
  ref_traces.npz       step lists of magik_trace_geodesic (the reference's
                       host_trace_geodesic.cu) for seeded initial conditions
                       over the three metrics, photons and massive particles
  ref_cmf_weights.npz  the reference's per-bin CIE 1931 XYZ weights
                       (compute_normalized_isi_cmf_weights) for the bin
                       layouts the workloads use
  ref_display.npz      the reference's colour resolve: for combinations of
                       scene colourspace, view transform, display colourspace,
                       GT7 mode and AgX look, its pipeline (in the library's
                       mgk_display_pipeline layout) and the display RGB of a
                       seeded set of XYZ colours by its own functions
  ref_cmf_icdf.npz     the reference's CIE inverse CDF table of its
                       stochastic spectral mode
                       (compute_tabulated_cmf_inverse_cdf) for the same
                       wavelength ranges
"""
import ctypes as C
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from magik_b200 import abi  # noqa: E402
from oracle import oracle_py as O  # noqa: E402

N_CASES = 48
N_STEPS = 160

IC_DTYPE = np.dtype([("test_particle_type", "<i4"), ("spatial_position", "<f4", 3), ("rotation", "<f4", 3),
                     ("local_proper_velocity", "<f4", 3), ("massive_particle_speed", "<f4"),
                     ("metric_type", "<i4"), ("time_reversed", "?"), ("event_horizon_scalar", "<f4"),
                     ("schwarzschild_mass", "<f4"), ("kerr_mass", "<f4"), ("kerr_spin", "<f4"),
                     ("n_max", "<u4"), ("atol", "<f4"), ("rtol", "<f4")])


def cases(seed=2024):
    rng = np.random.default_rng(seed)
    out = np.zeros(N_CASES, dtype=IC_DTYPE)
    mass = 6.7329546075e26
    for i in range(N_CASES):
        r = rng.uniform(3, 40)
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        out[i]["test_particle_type"] = abi.MASSLESS if i % 5 else abi.MASSIVE
        out[i]["spatial_position"] = d * r
        out[i]["rotation"] = rng.uniform(-math.pi, math.pi, 3)
        out[i]["local_proper_velocity"] = rng.normal(size=3) * 1e7
        out[i]["massive_particle_speed"] = rng.uniform(0, 2e8)
        out[i]["metric_type"] = i % 3
        out[i]["time_reversed"] = bool(i % 2)
        out[i]["event_horizon_scalar"] = 1.01
        out[i]["schwarzschild_mass"] = mass * (-1 if i % 11 == 7 else 1)
        out[i]["kerr_mass"] = mass
        out[i]["kerr_spin"] = rng.uniform(-0.999, 0.999)
        out[i]["n_max"] = int(rng.integers(1, 60))
        out[i]["atol"] = 10 ** rng.uniform(-10, -3)
        out[i]["rtol"] = 10 ** rng.uniform(-10, -3)
    return out


def to_structs(c):
    ic = abi.TraceInitialConditions(int(c["test_particle_type"]), *map(float, c["spatial_position"]),
                                    *map(float, c["rotation"]), *map(float, c["local_proper_velocity"]),
                                    float(c["massive_particle_speed"]))
    mp = abi.TraceMetricParams(int(c["metric_type"]), bool(c["time_reversed"]), float(c["event_horizon_scalar"]),
                               float(c["schwarzschild_mass"]), float(c["kerr_mass"]), float(c["kerr_spin"]))
    ip = abi.TraceIntegratorParams(int(c["n_max"]), float(c["atol"]), float(c["rtol"]))
    return ic, mp, ip


def main():
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libmagikref.so is missing: build it with `make -C oracle` next to the reference")
    cs = cases()
    steps = np.zeros((N_CASES, N_STEPS, 15), dtype=np.float32)
    n_written = np.zeros(N_CASES, dtype=np.int32)
    for i, c in enumerate(cs):
        rc, a = O.ref_trace_geodesic(*to_structs(c), n_steps=N_STEPS)
        assert rc == 0
        steps[i, : len(a)] = a
        n_written[i] = len(a)
    np.savez_compressed(os.path.join(HERE, "ref_traces.npz"), cases=cs, steps=steps, n_written=n_written)
    w = {f"w{n}_{int(lo)}_{int(hi)}": O.ref_cmf_weights(n, lo, hi)
         for n, lo, hi in [(16, 380.0, 780.0), (32, 380.0, 780.0), (24, 360.0, 830.0)]}
    np.savez_compressed(os.path.join(HERE, "ref_cmf_weights.npz"), **w)
    icdf = {f"icdf_{int(lo)}_{int(hi)}": O.ref_cmf_inverse_cdf(lo, hi) for lo, hi in [(380.0, 780.0), (360.0, 830.0)]}
    np.savez_compressed(os.path.join(HERE, "ref_cmf_icdf.npz"), **icdf)
    combos, settings, pipes, outs = display_golden()
    xyz = display_inputs()
    np.savez_compressed(os.path.join(HERE, "ref_display.npz"), combos=np.array(combos), settings=settings,
                        pipelines=pipes, xyz=xyz, rgb=outs)
    print("wrote", N_CASES, "traces,", len(w), "weight tables,", len(icdf), "inverse CDF tables and",
          len(combos), "display pipelines")


def display_inputs(n=384, seed=77):
    """XYZ colours for the display fixtures: luminance log-uniform over
    1e-4 .. 30 at chromaticities inside the spectral locus (x, y drawn in the
    triangle of the Rec.2020 primaries), and a few exact blacks."""
    rng = np.random.default_rng(seed)
    prim = np.array([[0.708, 0.292], [0.170, 0.797], [0.131, 0.046]])
    w = rng.dirichlet([1.0, 1.0, 1.0], n)
    xy = w @ prim
    Y = 10 ** rng.uniform(-4, math.log10(30.0), n)
    X = xy[:, 0] / xy[:, 1] * Y
    Z = (1 - xy[:, 0] - xy[:, 1]) / xy[:, 1] * Y
    xyz = np.stack([X, Y, Z], 1).astype(np.float32)
    xyz[:4] = 0.0
    return xyz


def display_golden():
    import ctypes as C
    import magik_b200 as M
    combos = []
    for vt in abi.VIEW_TRANSFORM:
        for dc in abi.DISPLAY_CS:
            combos.append(("LINEAR_REC709", vt, dc, "JZAZBZ", "GOLDEN"))
    for sc in abi.SCENE_CS:
        if sc != "LINEAR_REC709":
            combos.append((sc, "GRAN_TURISMO_7", "REC709", "JZAZBZ", "GOLDEN"))
            combos.append((sc, "AGX", "SRGB", "JZAZBZ", "GOLDEN"))
    for dc in ("REC709", "REC2100_PQ"):
        combos.append(("LINEAR_REC709", "GRAN_TURISMO_7", dc, "ICTCP", "GOLDEN"))
    for look in ("NONE", "PUNCHY"):
        combos.append(("LINEAR_REC709", "AGX", "SRGB", "JZAZBZ", look))
    xyz = display_inputs()
    settings, pipes, outs = [], [], []
    for sc, vt, dc, mode, look in combos:
        ds = M.display_defaults(scene_colorspace=sc, view_transform=vt, display_colorspace=dc, gt7_mode=mode,
                                agx_look=look)
        settings.append(np.frombuffer(bytes(ds), dtype=np.uint8))
        pipes.append(np.frombuffer(bytes(O.ref_display_pipeline(ds)), dtype=np.uint8))
        outs.append(O.ref_display_pixels(ds, xyz))
    return ["/".join(c) for c in combos], np.stack(settings), np.stack(pipes), np.stack(outs)


if __name__ == "__main__":
    main()
