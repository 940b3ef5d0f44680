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
    print("wrote", N_CASES, "traces,", len(w), "weight tables and", len(icdf), "inverse CDF tables")


if __name__ == "__main__":
    main()
