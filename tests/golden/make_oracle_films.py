"""Generates golden films of the FP64 oracle for the two render workloads at
reduced size (the oracle alone, no reference sources needed):

    python tests/golden/make_oracle_films.py

Writes oracle_films.npz with, for each workload (prefix c1_ / c2_), the
per-pixel XYZ film (float64, [height, width, 3]) and the per-ray termination
class and accepted-step count of the same frame.

  c1  the Schwarzschild CPU workload: M = 1, pinhole camera at r = 30 M,
      inclination 80 deg, 60 deg field of view, 1 jittered sample per pixel,
      disk 6-20 M at 1e4 K inner temperature, 16 bins over 380-780 nm, black
      background, escape at 1000 M, rtol 1e-8, atol 1e-10, <= 1e4 steps per
      ray, FP64 state; 64 x 64 pixels instead of 256 x 256 (same field of
      view, every fourth pixel pitch).
  c2  the Kerr benchmark frame: a = 0.9, r = 50 M, inclination 75 deg, disk
      from the ISCO, 32 bins, 1e5 seeded stars, rtol = atol = 1e-7, in FP64
      (the oracle the MIXED mode is checked against); 96 x 54 pixels x 2
      samples instead of 1920 x 1080 x 16.
  c2conv  the same frame in FP64 at rtol = atol = 1e-11: the converged
      image (its steps are 1e-10 apart from rtol 1e-12), against which the
      error of the rtol = 1e-7 renders, FP64 and MIXED alike, is measured.

tests/test_oracle_films.py checks that the oracle still renders these films
(CPU) and that the library's F64 and MIXED renders agree with them (GPU).
"""
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

PATH = os.path.join(HERE, "oracle_films.npz")
STAR_SEED = 0x57A25
N_STARS = 100_000


def workloads():
    """{name: (scene, stars)} of the two workloads at fixture size."""
    import magik_b200 as M
    from magik_b200 import abi
    c1 = M.scene_defaults(metric=abi.METRIC_SCHWARZSCHILD, spin=0.0, precision=abi.PRECISION_F64,
                          cam_r=30.0, cam_incl_rad=math.radians(80.0), disk_r_in=6.0, disk_r_out=20.0,
                          disk_T_in=1e4, n_bins=16, lambda_min_nm=380.0, lambda_max_nm=780.0,
                          escape_radius=1000.0, rel_tol=1e-8, abs_tol=1e-10, max_steps=10_000,
                          width=64, height=64, spp=1)
    c2 = M.scene_defaults(precision=abi.PRECISION_F64, width=96, height=54, spp=2)
    c2conv = M.scene_defaults(precision=abi.PRECISION_F64, width=96, height=54, spp=2, rel_tol=1e-11,
                              abs_tol=1e-11)
    stars = M.star_catalog(STAR_SEED, N_STARS)
    return {"c1": (c1, np.zeros(0, M.STAR_DTYPE)), "c2": (c2, stars), "c2conv": (c2conv, stars)}


def render(scene, stars):
    """(film [h, w, 3] float64, records) of the FP64 oracle."""
    import magik_b200 as M
    from oracle import oracle_py as O
    npix = scene.width * scene.height
    film, _ = O.render_pixels(scene, stars, M.xyz_weights(scene.n_bins), 0, npix)
    rec = O.trace_rays(scene, 0, npix * scene.spp)
    return film.reshape(scene.height, scene.width, 3), rec


def main():
    out = {}
    for name, (scene, stars) in workloads().items():
        film, rec = render(scene, stars)
        out[f"{name}_xyz"] = film
        out[f"{name}_cls"] = rec["cls"].astype(np.int8)
        out[f"{name}_steps"] = rec["steps"].astype(np.uint32)
    np.savez_compressed(PATH, **out)
    print(f"wrote {PATH}: " + ", ".join(f"{k} {v.shape}" for k, v in out.items()))


if __name__ == "__main__":
    main()
