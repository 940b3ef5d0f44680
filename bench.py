#!/usr/bin/env python
"""Geodesics/s of the Kerr render workload on B200s (and the CPU reference arm).

Workload (one "step" = one frame): Kerr a = 0.9, camera at r = 50 M and 75
degrees inclination, 60 degree horizontal field of view, 1920x1080 pixels at
16 samples per pixel (33,177,600 geodesics), thin Keplerian disk from the ISCO
to 20 M at T_in = 1e4 K, 32 spectral bins over 380-780 nm, 10^5 seeded
background stars, adaptive RKF45 at rtol = atol = 1e-7, FP32 ray state and
step control with FP64 attempts next to the horizon (MIXED), escape radius
1000 M.  Synthetic, seeded input.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Under torchrun the ranks share the one frame (--split spp, the default): rank
r renders a contiguous slice of the 16 samples per pixel (all pixels, the same
seed), and the films, weighted by their share of the samples, are
sum-reduced into rank 0 inside the timed region; the total work is fixed, so
scaling is strong.  --split seeds renders all 16 samples on every rank with
its own seed instead (weak scaling: N x 16 samples per pixel).  The value is
the geodesics of all ranks per second.  Rank 0 prints one JSON line.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# DRAM bytes per ray of k_integrate and per row of the fused inference, from one
# ncu capture each of a smaller case (640x360x16 rays; 2^20 rows); the
# traffic grows with the units, so the roofline scales it to the launch.
INTEGRATE_DRAM_BYTES_PER_RAY = 617.4e6 / 3_686_400
MLP_DRAM_BYTES_PER_ROW = 44.2e6 / 1_048_576
N_STARS = 100_000
STAR_SEED = 0x57A25
WORKLOAD = "kerr_a0.9_r50M_i75_fov60_1920x1080_16spp_32bins_1e5stars_rtol1e-7"
METRIC = "geodesics/s on 1 B200: RKF45 FP32 vs surrogate+fallback at <=1e-3 XYZ error"
UNIT = "geodesics/s"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mgk", choices=["mgk", "reference"])
    ap.add_argument("--split", default="spp", choices=["spp", "seeds"],
                    help="multi-GPU split: sample slices of one frame (strong) or one frame per rank (weak)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="CPU sample budget per measurement")
    # frame-size overrides for profiling captures (the default is the benchmark workload)
    ap.add_argument("--width", type=int, default=None)
    ap.add_argument("--height", type=int, default=None)
    ap.add_argument("--spp", type=int, default=None)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-surrogate", action="store_true", help="skip the surrogate+fallback leg")
    ap.add_argument("--surrogate-samples", type=int, default=1 << 24)
    ap.add_argument("--surrogate-epochs", type=int, default=20)
    ap.add_argument("--no-stress", action="store_true", help="skip the refill-stress frame (Kerr a=0.998)")
    ap.add_argument("--stress-spp", type=int, default=64)
    ap.add_argument("--c5-spp", type=int, default=256,
                    help="samples per pixel of the 3840x2160 surrogate render (0 skips it)")
    ap.add_argument("--surrogate-kernels", action="store_true",
                    help="time only the surrogate's training loop and fused inference (for profiling their kernels)")
    return ap.parse_args()


ARGS = None


def scene_config(M, rank=0, world=1):
    """The scene a rank renders: the whole frame at one rank; with --split
    spp its slice of the frame's samples, with --split seeds the whole frame
    under its own seed."""
    from magik_b200.dist import frame_seed, sample_slice
    s = M.scene_defaults()
    _resize(s)
    if ARGS is not None and ARGS.split == "seeds":
        s.seed = frame_seed(0x5EED, rank)
    else:
        s.seed = 0x5EED
        s.sample_offset, s.spp = sample_slice(s.spp, rank, world)
    return s


def _resize(s):
    if ARGS is not None:
        for k in ("width", "height", "spp"):
            v = getattr(ARGS, k)
            if v:
                setattr(s, k, v)


MIXED_PRECISION = "mixed (fp32 state and step control, fp64 attempts within 0.05 M of the horizon)"


def config_dict(s, extra=None, precision=MIXED_PRECISION):
    name = WORKLOAD if (s.width, s.height, s.spp) == (1920, 1080, 16) else f"{WORKLOAD} resized to {s.width}x{s.height}x{s.spp}spp (profiling size)"
    d = {"workload": name, "metric_tensor": "kerr", "spin": s.spin, "width": s.width, "height": s.height,
         "spp": s.spp, "rays_per_frame": s.width * s.height * s.spp, "n_bins": s.n_bins, "stars": N_STARS,
         "rel_tol": s.rel_tol, "abs_tol": s.abs_tol,
         "precision": precision,
         "l2": "a 512 MiB buffer is written between timed frames (frame traffic is also > L2)"}
    if extra:
        d.update(extra)
    return d


# ------------------------------------------------------------------ clocks
class Clocks:
    """Samples SM clocks and throttle reasons with nvidia-smi while timing."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.path = tempfile.mktemp(prefix="mgk_clocks_", suffix=".csv")
        self.proc = None

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.f.close()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax = float(parts[2])
                except ValueError:
                    continue
                for n, v in zip(names, parts[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
        os.unlink(self.path)
        loaded = [v for v in sm if smax and v > 0.3 * smax] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------------------- CPU legs
def cpu_render_sample(s, stars, w, seconds, precision, reference=False):
    """Renders a strided sample of the frame's pixels on the host cores and
    returns (geodesics/s, accepted RKF45 steps/s, threads, description).  The
    sample is sized from a short calibration run so that it takes about
    `seconds`."""
    from oracle import oracle_py as O
    s = s.copy()
    s.precision = precision
    threads = os.cpu_count() or 1
    npix = s.width * s.height
    render = O.ref_render_pixels if reference else O.render_pixels
    n_cal = min(npix, 64 * threads)
    stride = max(1, npix // n_cal)
    t0 = time.perf_counter()
    render(s, stars, w, 0, n_cal, nthreads=threads, stride=stride)
    dt = time.perf_counter() - t0
    rate = n_cal / max(dt, 1e-6)
    n = int(min(npix, max(n_cal, rate * seconds)))
    stride = max(1, npix // n)
    t0 = time.perf_counter()
    _, counts = render(s, stars, w, 0, n, nthreads=threads, stride=stride)
    dt = time.perf_counter() - t0
    rays = n * s.spp
    desc = (f"{n} of {npix} pixels (every {stride}th) x {s.spp} spp = {rays} geodesics, "
            f"{counts['steps']} steps in {dt:.1f} s")
    cpu_render_sample.last_ms = dt * 1e3
    return rays / dt, counts["steps"] / dt, threads, desc


# ------------------------------------------------------------------ arms
def run_reference(args, rank, world):
    """The reference arm: the reference's own RKF45 (metric_kerr.cuh /
    internal_math.h compiled from its sources into oracle/_ref) per camera
    ray on all host cores, with the reference's own CIE weights.  Everything
    it needs comes from oracle/: the scene (the oracle's restatement of the
    workload's defaults), the star catalogue and, where oracle/_ref is
    absent, the oracle port in the reference's arithmetic.  It neither
    imports the magik_b200 package nor loads libmgk.so.  Rank 0 alone runs."""
    if rank != 0:
        return None
    from oracle import oracle_py as O
    abi = O.abi
    s = O.scene_defaults()
    _resize(s)
    stars = O.star_catalog(STAR_SEED, N_STARS)
    use_ref = O.ref_available() and hasattr(O, "ref_render_pixels")
    if use_ref:
        w = O.ref_cmf_weights(s.n_bins, s.lambda_min_nm, s.lambda_max_nm)
    else:
        w = np.load(os.path.join(ROOT, "tests", "golden", "ref_cmf_weights.npz"))[
            f"w{s.n_bins}_{int(s.lambda_min_nm)}_{int(s.lambda_max_nm)}"]
    kind = "reference" if use_ref else "port"
    per = max(2.0, min(args.cpu_seconds, 120.0 / max(1, args.steps + args.warmup)))
    vals, svals, step_ms, desc, threads = [], [], [], "", 1
    for i in range(args.warmup + args.steps):
        v, sv, threads, desc = cpu_render_sample(s, stars, w, per, abi.PRECISION_REF32, reference=use_ref)
        if i >= args.warmup:
            vals.append(v)
            svals.append(sv)
            step_ms.append(cpu_render_sample.last_ms)
    value = statistics.mean(vals)
    rays = s.width * s.height * s.spp
    what = ("the reference's own RKF45 (metric_kerr.cuh / internal_math.h compiled from its sources) per camera "
            "ray, with the disk, escape, star and spectral stages of the CPU oracle, which the reference lacks, "
            "and the reference's own CIE 1931 bin weights"
            if use_ref else "the CPU oracle in REF32 arithmetic (the reference's operation order)")
    precision = "fp32 (REF32: the reference's arithmetic and step control)"
    return {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            # each step renders a strided pixel sample of the frame (cpu_baseline.sample)
            "ms_per_step": statistics.mean(step_ms), "ms_per_frame_equivalent": rays / value * 1e3,
            "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "fp32", "data": "synthetic (seeded)",
            "config": config_dict(s, precision=precision),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                             "sample": desc + "; a step is one such sample; ms_per_frame_equivalent is the "
                                       "time the whole frame takes at the sample's rate",
                             "what": what, "steps_per_s": statistics.mean(svals)},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "package_imported": "magik_b200" in sys.modules}


# The pool's earlier measurement of HBM copy bandwidth and cuBLAS BF16 burst
# throughput, used only when MEASURED_PEAKS.json is absent.
FALLBACK_PEAKS = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}


def measured_peaks():
    """(peaks, source): MEASURED_PEAKS.json when present ("of measured"), else
    the fallback figures ("of fallback")."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        if d.get("hbm_gbs") and d.get("bf16_tflops"):
            return d, "of measured"
    except (OSError, ValueError):
        pass
    return dict(FALLBACK_PEAKS), "of fallback"



def run_surrogate(args, ctx, s, d_stars, d_w, film_mixed_ms, steps):
    """Surrogate + RKF45 fallback on the same frame, after training the
    network on the GPU as specified: 2^24 rays with observers uniform in r
    [10, 100] M and inclination [0, 90] deg, spins uniform in [0, 0.998]
    (16 launches), FP64 RKF45 labels, Adam lr 1e-3, batch 65536, 20 epochs.
    Routing: confidence < 0.99 or impact parameter within 2% of the critical
    curve go to the FP32 RKF45 fallback.  Errors are the mean absolute XYZ
    difference over the image divided by the mean absolute XYZ of the FP64
    image."""
    import torch
    import magik_b200 as M
    dev = f"cuda:{ctx.device}"
    npix = s.width * s.height
    rays = npix * s.spp
    f64 = M.scene_defaults(width=s.width, height=s.height, spp=s.spp, precision=M.abi.PRECISION_F64)
    f64.seed = s.seed
    ref = torch.empty(npix * 3, dtype=torch.float32, device=dev)
    ctx.render(f64, d_stars, ref, d_weights=d_w, want_stats=False)
    scale = float(ref.abs().mean())
    # the converged image: FP64 at rtol = atol = 1e-11
    conv = M.scene_defaults(width=s.width, height=s.height, spp=s.spp, precision=M.abi.PRECISION_F64,
                            rel_tol=1e-11, abs_tol=1e-11)
    conv.seed = s.seed
    ref_conv = torch.empty_like(ref)
    ctx.render(conv, d_stars, ref_conv, d_weights=d_w, want_stats=False)
    scale_conv = float(ref_conv.abs().mean())
    err_f64_conv = float((ref - ref_conv).abs().mean()) / scale_conv
    film = torch.empty_like(ref)

    def timed(fn):
        fn()
        ts = []
        for _ in range(steps):
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            st = fn()
            e1.record()
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        return statistics.mean(ts), st

    ctx.render(s, d_stars, film, d_weights=d_w, want_stats=False)
    err_plain = float((film - ref).abs().mean()) / scale
    err_plain_conv = float((film - ref_conv).abs().mean()) / scale_conv

    t0 = time.time()
    feat, lab = M.make_samples(ctx, f64, 0x5A3B, args.surrogate_samples, n_spin_buckets=16)
    torch.cuda.synchronize()
    t_samples = time.time() - t0
    # the training kernels' first use in this process (module loading, kernel
    # attributes) outside the timed region: one epoch of a separate network;
    # the timed run still sizes its own buffers and captures its own graph
    warm = M.Surrogate(ctx, seed=5)
    warm.train(M.train_defaults(epochs=1), feat, lab)
    warm.close()
    torch.cuda.synchronize()
    net = M.Surrogate(ctx, seed=3)
    cfg = M.train_defaults(epochs=args.surrogate_epochs)
    t0 = time.time()
    losses = net.train(cfg, feat, lab)
    t_train = time.time() - t0
    steps_train = args.surrogate_epochs * (args.surrogate_samples // cfg.batch)
    train_flop = steps_train * cfg.batch * 3 * 400_896  # forward + two backward GEMMs per layer
    # the same training on the mma.sync GEMM path, one epoch, for comparison
    os.environ["MGK_SURROGATE_TRAIN"] = "mma"
    try:
        net_mma = M.Surrogate(ctx, seed=3)
    finally:
        del os.environ["MGK_SURROGATE_TRAIN"]
    cfg1 = M.train_defaults(epochs=1)
    torch.cuda.synchronize()
    t0 = time.time()
    net_mma.train(cfg1, feat, lab)
    t_mma = time.time() - t0
    net_mma.close()
    mma_tflops = (args.surrogate_samples // cfg1.batch) * cfg1.batch * 3 * 400_896 / t_mma / 1e12

    # fused inference kernel alone (tensor-core roofline)
    x = feat[: 1 << 22].contiguous()
    n_rows = int(x.shape[0])
    fwd_ms, _ = timed(lambda: net.forward(x))
    fwd_tflops = n_rows * 400_896 / (fwd_ms * 1e-3) / 1e12
    peaks, peak_src = measured_peaks()
    bf16_peak = peaks.get("bf16_tflops")

    points = []
    for name, cm, cf in (("spec routing: conf<0.99 or |b-b_c|/b_c<2% -> RKF45", 0.99, 0.02),
                         ("network only (no fallback)", -1.0, 0.0)):
        ms, st = timed(lambda: M.render_surrogate(ctx, net, s, d_stars, film, conf_min=cm, crit_frac=cf,
                                                  d_weights=d_w))
        err = float((film - ref).abs().mean()) / scale
        err_conv = float((film - ref_conv).abs().mean()) / scale_conv
        points.append({"routing": name, "conf_min": cm, "crit_frac": cf, "value": rays / (ms * 1e-3),
                       "unit": UNIT, "ms_per_frame": ms, "fallback_fraction": st.fallback_rays / rays,
                       "network_and_routing_ms": st.surrogate_ms, "rkf45_ms": st.integrate_ms,
                       "xyz_rel_err_vs_fp64": err, "xyz_rel_err_vs_fp64_converged": err_conv,
                       "meets_1e-3": err <= 1e-3,
                       "speedup_vs_plain_rkf45": film_mixed_ms / ms})
    config5 = None if args.c5_spp <= 0 else run_config5(args, ctx, net, d_stars, d_w)
    assert net.status() == 0
    net.close()
    return {
        "config5": config5,
        "value": points[0]["value"], "unit": UNIT, "xyz_rel_err_vs_fp64": points[0]["xyz_rel_err_vs_fp64"],
        "plain_rkf45_xyz_rel_err_vs_fp64": err_plain, "plain_rkf45_xyz_rel_err_vs_fp64_converged": err_plain_conv,
        "fp64_same_tolerance_xyz_rel_err_vs_converged": err_f64_conv,
        "error_definition": "mean |XYZ - XYZ_ref| over the frame / mean |XYZ_ref|; fp64 = F64 at the same "
                            "rtol 1e-7, fp64_converged = F64 at rtol = atol = 1e-11",
        "points": points,
        "training": {"samples": args.surrogate_samples, "epochs": args.surrogate_epochs, "batch": cfg.batch,
                     "sample_generation_s": t_samples, "train_s": t_train,
                     "timed": "the whole run of a fresh network: its buffers, first epoch, graph capture, replays "
                              "and loss read-back (one epoch of another network loaded the kernels before)",
                     "train_tflops": train_flop / t_train / 1e12, "epoch_loss": [float(v) for v in losses],
                     "path": "tcgen05 (one kernel per tile: forward with stash and loss, then the input-"
                             "gradient chain; split-K weight gradients; Adam on device-side step counters; "
                             "one CUDA graph per epoch)",
                     "mma_sync_path_tflops": mma_tflops,
                     "flop_count": "3 x 400,896 FLOP per sample per step (forward, input and weight gradients)",
                     "distribution": "observer r U[10,100] M, inclination U[0,90] deg, spin U[0,0.998] "
                                     "(16 launches), directions uniform on the forward hemisphere"},
        "inference_roofline": {"bound": "tensor", "kernel": "k_mlp_chain_tc<INFER> (tcgen05, fused 5 layers)",
                               "achieved": fwd_tflops, "peak": bf16_peak, "unit": "TFLOP/s",
                               "frac": (fwd_tflops / bf16_peak) if bf16_peak else None,
                               "traffic": MLP_DRAM_BYTES_PER_ROW * n_rows,
                               "peak_source": f"MEASURED_PEAKS.json bf16_tflops (cuBLAS burst), {peak_src}",
                               "flop_per_ray": 400_896, "rows": n_rows, "ms": fwd_ms},
    }


def run_surrogate_kernels(args, device):
    """The surrogate's kernels alone: the training loop on
    --surrogate-samples FP64-labelled samples of the training distribution
    (one warm-up epoch, then --surrogate-epochs timed epochs at batch 65536 on
    the default tcgen05 path; 3 x 400,896 FLOP per sample per step), then the
    fused inference on 2^22 rows of the same samples (400,896 FLOP per row,
    CUDA events over 5 launches after one)."""
    import torch
    import magik_b200 as M
    torch.cuda.set_device(device)
    with M.Context(device) as ctx:
        s = M.scene_defaults(width=1920, height=1080, spp=1, precision=M.abi.PRECISION_F64)
        feat, lab = M.make_samples(ctx, s, 0x5A3B, args.surrogate_samples, n_spin_buckets=16)
        net = M.Surrogate(ctx, seed=3)
        # warm-up: a run of 2 epochs sets up the kernels and captures the
        # graph of one epoch, which the timed run reuses
        net.train(M.train_defaults(epochs=2), feat, lab)
        cfg = M.train_defaults(epochs=args.surrogate_epochs)
        torch.cuda.synchronize()
        t0 = time.time()
        losses = net.train(cfg, feat, lab)
        torch.cuda.synchronize()
        dt = time.time() - t0
        x = feat[: min(1 << 22, feat.shape[0])].contiguous()
        net.forward(x)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(5):
            net.forward(x)
        e1.record()
        e1.synchronize()
        infer_ms = e0.elapsed_time(e1) / 5
        assert net.status() == 0
        net.close()
    steps = args.surrogate_epochs * (args.surrogate_samples // cfg.batch)
    return {"metric": "surrogate training FLOP/s", "value": steps * cfg.batch * 3 * 400_896 / dt / 1e12,
            "unit": "TFLOP/s", "higher_is_better": True, "steps": steps, "us_per_step": dt / steps * 1e6,
            "batch": cfg.batch, "samples": args.surrogate_samples, "epochs": args.surrogate_epochs,
            "final_loss": float(losses[-1]), "dtype": "bf16", "data": "synthetic",
            "inference": {"rows": int(x.shape[0]), "ms": infer_ms,
                          "tflops": int(x.shape[0]) * 400_896 / (infer_ms * 1e-3) / 1e12}}


def run_config5(args, ctx, net, d_stars, d_w):
    """The surrogate inference render of the specification: the benchmark's
    Kerr a = 0.9 view at 3840x2160 and 256 spp (2,123,366,400 geodesics),
    32 bins, rendered with plain RKF45 (MIXED), with the specified routing
    (confidence < 0.99 or impact parameter within 2 % of the critical curve
    -> FP32 RKF45) and with the network alone, each once after the frames
    above warmed the kernels.  Errors: mean |XYZ - XYZ_F64| over the frame /
    mean |XYZ_F64|, against the full-RKF45 FP64 render of the same samples."""
    import torch
    import magik_b200 as M
    dev = f"cuda:{ctx.device}"
    s = M.scene_defaults(width=3840, height=2160, spp=args.c5_spp)
    f64 = M.scene_defaults(width=3840, height=2160, spp=args.c5_spp, precision=M.abi.PRECISION_F64)
    rays = s.width * s.height * s.spp
    npix = s.width * s.height
    ref = torch.empty(npix * 3, dtype=torch.float32, device=dev)
    ctx.render(f64, d_stars, ref, d_weights=d_w, want_stats=False)
    scale = float(ref.abs().mean())
    film = torch.empty_like(ref)

    def once(fn):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        st = fn()
        e1.record()
        e1.synchronize()
        return e0.elapsed_time(e1), st

    plain_ms, _ = once(lambda: ctx.render(s, d_stars, film, d_weights=d_w, want_stats=False))
    plain_err = float((film - ref).abs().mean()) / scale
    out = {"workload": f"kerr_a0.9_r50M_i75_fov60_3840x2160_{s.spp}spp_32bins_1e5stars_rtol1e-7",
           "rays": rays, "plain_rkf45": {"value": rays / (plain_ms * 1e-3), "unit": UNIT, "ms_per_frame": plain_ms,
                                         "xyz_rel_err_vs_fp64": plain_err},
           "points": []}
    for name, cm, cf in (("spec routing: conf<0.99 or |b-b_c|/b_c<2% -> RKF45", 0.99, 0.02),
                         ("network only (no fallback)", -1.0, 0.0)):
        ms, st = once(lambda: M.render_surrogate(ctx, net, s, d_stars, film, conf_min=cm, crit_frac=cf,
                                                 d_weights=d_w))
        err = float((film - ref).abs().mean()) / scale
        out["points"].append({"routing": name, "value": rays / (ms * 1e-3), "unit": UNIT, "ms_per_frame": ms,
                              "fallback_fraction": st.fallback_rays / rays, "xyz_rel_err_vs_fp64": err,
                              "meets_1e-3": err <= 1e-3, "speedup_vs_plain_rkf45": plain_ms / ms,
                              "meets_5x_at_1e-3": err <= 1e-3 and plain_ms / ms >= 5.0})
    return out


def split_rooflines(metric, st, integrate_ms, peaks):
    """The integrator's two roofline lines for one frame: FP32 work (the
    attempts taken in FP32 and the crossing sub-steps) over the FP32 peak, and
    the FP64 attempts next to the horizon over the FP64 peak.  Both run inside
    the same kernels, so the FP64 line gives the time its work needs at the
    FP64 peak, its share of the integration time, and the fraction of the
    combined bound (FP32 work / FP32 peak + FP64 work / FP64 peak)."""
    from magik_b200 import flops as FL
    t = integrate_ms * 1e-3
    f32 = FL.render_flops(metric, st.attempts - st.wide_attempts, st.refine_evals)
    f64 = st.wide_attempts * FL.attempt_flops(metric)
    r32 = {"bound": "fp32", "achieved": f32 / t / 1e12, "peak": peaks["fp32"] / 1e12, "unit": "TFLOP/s",
           "frac": f32 / t / peaks["fp32"]}
    t64 = f64 / peaks["fp64"]
    r64 = {"bound": "fp64", "flop": f64, "attempts": st.wide_attempts, "peak": peaks["fp64"] / 1e12,
           "unit": "TFLOP/s", "ms_at_peak": t64 * 1e3, "share_of_integrate_time_at_peak": t64 / t,
           "combined_frac": (f32 / peaks["fp32"] + t64) / t,
           "peak_source": "measured in this run by mgk_fp64_peak (double FMA probe kernel)"}
    return r32, r64


def run_stress(args, ctx, d_stars, d_w, peaks):
    """BASELINE's refill-stress configuration: Kerr a = 0.998, observer at
    r = 20 M and 85 degrees, 3840x2160 at 64 spp (530,841,600 geodesics),
    up to 5e4 steps per ray, FP32 integration with the FP64 band near the
    horizon.  One warm-up and one timed frame; reports geodesics/s, the
    fraction of attempts taken in FP64 and the FP32 roofline."""
    import torch
    import magik_b200 as M
    s = M.scene_defaults(width=3840, height=2160, spp=args.stress_spp, spin=0.998, cam_r=20.0,
                         cam_incl_rad=85.0 * 3.141592653589793 / 180.0, max_steps=50_000)
    s.disk_r_in = M.isco_radius(0.998)
    film = torch.empty(s.width * s.height * 3, dtype=torch.float32, device=f"cuda:{ctx.device}")
    ctx.render(s, d_stars, film, d_weights=d_w, want_stats=False)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    st = ctx.render(s, d_stars, film, d_weights=d_w, want_stats=True)
    e1.record()
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    rays = s.width * s.height * s.spp
    r32, r64 = split_rooflines(s.metric, st, st.integrate_ms, peaks)
    return {"workload": f"kerr_a0.998_r20M_i85_fov60_3840x2160_{s.spp}spp_32bins_1e5stars_rtol1e-7",
            "value": rays / (ms * 1e-3), "unit": UNIT, "ms_per_frame": ms, "rays": rays,
            "attempts_per_ray": st.attempts / rays, "max_steps": s.max_steps,
            "fp64_attempt_fraction": st.wide_attempts / max(1, st.attempts),
            "rays_resumed_in_tail": st.resumed, "step_limit_rays": int(st.class_count[4]),
            "classes": dict(zip(["alive", "disk", "escaped", "horizon", "step_limit", "light"],
                                [int(c) for c in st.class_count])),
            "roofline": r32, "roofline_fp64": r64}


def run_room(args, ctx, d_w, peaks):
    """The reference's box-and-light stage around the Kerr a = 0.9 hole
    (walls at x, z = +-40 M, floor and ceiling at y = -+20 M, white-LED light
    straddling the ceiling, up to 10 reflections, mirror walls normal to x,
    Lambertian elsewhere), camera 18 M out and 10 degrees above the equator,
    1920x1080 at 4 spp, MIXED precision.  One warm-up and three timed frames;
    geodesics/s (camera rays), path segments/s (rays + reflections), the
    FP32 roofline of the integration and the oracle port on a strided sample
    of the same frame on the host cores."""
    import torch
    import magik_b200 as M
    s = M.scene_defaults(width=1920, height=1080, spp=4, room_on=1, cam_r=18.0,
                         cam_incl_rad=80.0 * 3.141592653589793 / 180.0, disk_r_out=0.0)
    film = torch.empty(s.width * s.height * 3, dtype=torch.float32, device=f"cuda:{ctx.device}")
    ctx.render(s, None, film, d_weights=d_w, want_stats=False)
    torch.cuda.synchronize()
    reps = 3
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        st = ctx.render(s, None, film, d_weights=d_w, want_stats=True)
    e1.record()
    e1.synchronize()
    ms = e0.elapsed_time(e1) / reps
    rays = s.width * s.height * s.spp
    r32, r64 = split_rooflines(s.metric, st, st.integrate_ms, peaks)
    out = {"workload": "room_kerr_a0.9_r18M_i80_fov60_1920x1080_4spp_32bins_10reflections",
           "value": rays / (ms * 1e-3), "unit": UNIT, "ms_per_frame": ms, "rays": rays,
           "segments_per_s": (rays + st.reflections) / (ms * 1e-3),
           "reflections_per_ray": st.reflections / rays, "attempts_per_ray": st.attempts / rays,
           "classes": dict(zip(["alive", "disk", "escaped", "horizon", "step_limit", "light"],
                               [int(c) for c in st.class_count])),
           "film_finite": bool(torch.isfinite(film).all().item()),
           "roofline": r32, "roofline_fp64": r64}
    if not args.no_cpu_baseline:
        v, sv, thr, desc = cpu_render_sample(s, np.zeros(0, M.STAR_DTYPE), M.xyz_weights(s.n_bins), 3.0,
                                             M.abi.PRECISION_MIXED)
        out["cpu_port"] = {"value": v, "unit": UNIT, "cores": thr, "kind": "port", "sample": desc,
                           "steps_per_s": sv}
    return out


def run_display(args, ctx):
    """The colour resolve after the film (mgk_display) over 16.8 M seeded XYZ
    pixels (403 MB moved per launch, above the 126 MB L2): the reference's
    default settings (linear Rec.709 scene, white balance 5600 K, the GT7 tone
    mapper in Jzazbz, Rec.709 display), which spend ~36 float transcendentals
    per pixel and are compute-bound, and the same resolve without a view
    transform to sRGB, which is HBM-bound (24 bytes per pixel)."""
    import torch
    import magik_b200 as M
    n = 1 << 24
    dev = f"cuda:{ctx.device}"
    g = torch.Generator(device=dev)
    g.manual_seed(0xD15)
    xyz = torch.rand(n * 3, generator=g, device=dev) * 4.0
    rgb = torch.empty_like(xyz)
    peaks, peak_src = measured_peaks()
    peak = peaks.get("hbm_gbs")

    def timed(pipe, reps=20):
        for _ in range(3):
            ctx.display(pipe, xyz, rgb)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            ctx.display(pipe, xyz, rgb)
        e1.record()
        e1.synchronize()
        return e0.elapsed_time(e1) / reps

    out = {}
    for key, ds, what in (("gt7", M.display_defaults(),
                           "GT7 (Jzazbz) view transform, Rec.709 scene and display"),
                          ("none_srgb", M.display_defaults(view_transform="NONE", display_colorspace="SRGB"),
                           "no view transform, Rec.709 scene, sRGB display")):
        ms = timed(M.display_prepare(ds))
        gbs = 24.0 * n / (ms * 1e-3) / 1e9
        out[key] = {"workload": f"{what}, 16,777,216 XYZ pixels", "value": n / (ms * 1e-3), "unit": "pixels/s",
                    "ms_per_launch": ms,
                    "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s",
                                 "frac": gbs / peak if peak else None,
                                 "peak_source": f"MEASURED_PEAKS.json hbm_gbs, {peak_src}",
                                 "note": "instruction-bound, not HBM-bound: ncu 90 % issue, 3.7 % DRAM"
                                         if key == "gt7" else
                                         ("24 bytes per pixel moved; three full-accuracy powf per pixel (the sRGB "
                                          "encode) set the time, not the bytes")}}
    return out


def run_gpu(args, rank, world, local_rank):
    import torch
    import magik_b200 as M
    from magik_b200 import flops as FL

    from magik_b200.dist import reduce_film, reduce_slices
    torch.cuda.set_device(local_rank)
    dev = f"cuda:{local_rank}"
    ctx = M.Context(local_rank)
    strong = args.split == "spp"
    s = scene_config(M, rank, world)       # what this rank renders
    s_frame = scene_config(M, 0, 1)        # the frame
    rays = s.width * s.height * s.spp     # this rank's geodesics per step
    npix = s.width * s.height
    total_rays = s_frame.width * s_frame.height * s_frame.spp * (1 if strong else world)

    def combine(f):
        # the one exchange step: the ranks' films into rank 0's
        if world > 1:
            if strong:
                reduce_slices(f, s.spp, s_frame.spp)
            else:
                reduce_film(f)
    stars = M.star_catalog(STAR_SEED, N_STARS)
    w = M.xyz_weights(s.n_bins)
    d_stars = torch.from_numpy(stars.view(np.uint8)).to(dev)
    d_w = torch.from_numpy(w.ravel()).to(dev)
    film = torch.empty(npix * 3, dtype=torch.float32, device=dev)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=dev)
    peak = ctx.fp32_peak()
    peaks_fp = {"fp32": peak, "fp64": ctx.fp64_peak()}

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    for _ in range(args.warmup):
        ctx.render(s, d_stars, film, d_weights=d_w, want_stats=False)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()

    clocks = Clocks(local_rank)
    clocks.start()
    times, integ, flop = [], [], []
    st_last = None
    for _ in range(args.steps):
        flush.fill_(1)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        st = ctx.render(s, d_stars, film, d_weights=d_w, want_stats=True)
        combine(film)
        e1.record()
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
        integ.append(st.integrate_ms)
        flop.append(FL.render_flops(s.metric, st.attempts - st.wide_attempts, st.refine_evals))
        st_last = st
    torch.cuda.synchronize()
    clk = clocks.stop()
    barrier()

    # end to end through the host-buffer entry point: pinned inputs in, film out
    h_stars = torch.from_numpy(stars.view(np.uint8).copy()).pin_memory()
    h_w = torch.from_numpy(w.ravel().copy()).pin_memory()
    h_film = torch.empty(npix * 3, dtype=torch.float32).pin_memory()
    e2e_times = []
    d_tmp = torch.empty_like(film) if world > 1 else None

    def render_e2e():
        ctx.render_host(s, h_stars, h_film, h_weights=h_w, want_stats=False)
        if world > 1:  # the host film through the same exchange step, back to rank 0's host
            d_tmp.copy_(h_film, non_blocking=True)
            combine(d_tmp)
            if rank == 0:
                h_film.copy_(d_tmp, non_blocking=True)

    if not args.no_e2e:
        render_e2e()
        for _ in range(max(1, min(args.steps, 3))):
            flush.fill_(1)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            render_e2e()
            e1.record()
            e1.synchronize()
            e2e_times.append(e0.elapsed_time(e1))
        film_ok = bool(torch.isfinite(h_film).all().item())
    else:
        e2e_times = [float("nan")]
        film_ok = bool(torch.isfinite(film).all().item())

    ms = statistics.mean(times)
    e2e_ms = statistics.mean(e2e_times)
    ms_int = statistics.mean(integ)
    steps_all = float(st_last.steps)
    if world > 1:
        from magik_b200.dist import max_over_ranks, sum_over_ranks
        ms, e2e_ms, ms_int = max_over_ranks([ms, e2e_ms, ms_int], device=dev)
        steps_all = sum_over_ranks([steps_all], device=dev)[0]
    if rank != 0:
        return None

    achieved = statistics.mean(f / (t * 1e-3) for f, t in zip(flop, integ))
    out = {
        "metric": METRIC, "value": total_rays / (ms * 1e-3), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "strong" if strong else "weak", "vs_baseline": None,
        "dtype": "fp32 (fp64 attempts next to the horizon)",
        "data": "synthetic (seeded camera jitter and star catalogue)",
        # one camera geodesic per pixel sample: samples/s equals geodesics/s
        "samples_per_s": total_rays / (ms * 1e-3),
        "config": config_dict(s_frame, {"parallelism": (
            f"{world} GPU(s): each renders {s.spp} of the frame's {s_frame.spp} samples per pixel "
            f"(sample slices of one frame), films weighted and sum-reduced into rank 0 (strong)") if strong else (
            f"{world} GPU(s): each renders the whole frame with its own seed, films averaged into rank 0 "
            f"(weak: {world} x {s_frame.spp} samples per pixel)")}),
        "e2e": {"value": total_rays / (e2e_ms * 1e-3), "unit": UNIT,
                "h2d_bytes_per_step": int(h_stars.numel() + h_w.numel() * 4),
                "d2h_bytes_per_step": int(h_film.numel() * 4)},
        "roofline": {"bound": "fp32", "kernel": "k_integrate + k_refine + k_tail (one chunk)",
                     "achieved": achieved / 1e12, "peak": peak / 1e12, "unit": "TFLOP/s",
                     "frac": achieved / peak, "traffic": INTEGRATE_DRAM_BYTES_PER_RAY * rays,
                     "traffic_note": "bytes per launch of k_integrate: ncu DRAM bytes per ray of a "
                                     "640x360x16 capture x rays of this frame",
                     "peak_source": "measured in this run by mgk_fp32_peak (FMA probe kernel); "
                                    "MEASURED_PEAKS.json has no FP32 figure",
                     "flop_per_attempt": FL.attempt_flops(s.metric),
                     "flop_per_crossing_substep": FL.substep_flops(s.metric),
                     "integrate_ms": ms_int,
                     "work": "attempts taken in FP32 and crossing sub-steps; the FP64 attempts are in roofline_fp64"},
        "roofline_fp64": split_rooflines(s.metric, st_last, ms_int, peaks_fp)[1],
        "steps_per_s": steps_all / (ms * 1e-3),
        "stats": {"attempts": st_last.attempts, "steps": st_last.steps, "refine_evals": st_last.refine_evals,
                  "wide_attempts": st_last.wide_attempts, "crossings": st_last.crossings,
                  "resumed": st_last.resumed,
                  "classes": dict(zip(["alive", "disk", "escaped", "horizon", "step_limit", "light"],
                                      [int(c) for c in st_last.class_count])),
                  "attempts_per_ray": st_last.attempts / rays},
        "clocks": clk,
        # per frame: generate, integrate, refine, tail, shade, resolve; next-pass,
        # integrate and refine for each continuation pass; four star-grid kernels
        "gpu_launches": (6 + 3 * (int(st_last.n_passes) - 1) + 4) * args.steps,
        "film_finite": film_ok,
    }
    if world == 1 and not args.no_stress:
        out["refill_stress"] = run_stress(args, ctx, d_stars, d_w, peaks_fp)
    if world == 1:
        out["room"] = run_room(args, ctx, d_w, peaks_fp)
        out["display"] = run_display(args, ctx)
    if world == 1 and not args.no_surrogate:
        # runs after the timed region; its own timings are inside "surrogate"
        out["surrogate"] = run_surrogate(args, ctx, s, d_stars, d_w, ms, max(1, min(args.steps, 3)))
    if world == 1 and not args.no_cpu_baseline:
        from oracle import oracle_py as O
        use_ref = O.ref_available()
        v, sv, thr, desc = cpu_render_sample(s, stars, w, args.cpu_seconds,
                                             M.abi.PRECISION_REF32 if use_ref else M.abi.PRECISION_MIXED,
                                             reference=use_ref)
        out["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": thr, "kind": "reference" if use_ref else "port",
                               "sample": desc, "steps_per_s": sv}
    return out


def main():
    global ARGS
    args = parse_args()
    ARGS = args
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.surrogate_kernels:
        print(json.dumps(run_surrogate_kernels(args, local_rank)), flush=True)
        return 0
    if args.impl == "reference":
        out = run_reference(args, rank, world)
        if out is not None:
            print(json.dumps(out), flush=True)
        return 0
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device(f"cuda:{local_rank}"))
    try:
        out = run_gpu(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
    if out is not None:
        print(json.dumps(out), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
