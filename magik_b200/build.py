"""Builds libmgk.so in-tree with nvcc for sm_100a.

    python -m magik_b200.build

The kernels are compiled with -fmad=false: every fused multiply-add is
written explicitly (mad()), which is what lets the REF32 and MIXED modes be
checked bit for bit against the CPU oracle.  The CUDA runtime is linked
statically so the library does not depend on which libcudart a host process
already loaded.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libmgk.so")
SOURCES = ["kernels.cu", "api.cu", "static_scratch.cu", "mlp.cu", "mlp_tc.cu", "mlp_train_tc.cu", "surrogate.cu", "display.cu",
           "manager.cu"]
HEADERS = ["dev_physics.cuh", "dev_pair.cuh", "dev_scene.cuh", "internal.h", "cie1931_2deg.inc", "mlp.h", "mlp_loss.cuh", "mlp_act.cuh", "tc_sm100.cuh",
           os.path.join("..", "src", "renderer", "relativity", "metric.cuh"),
           os.path.join("..", "src", "renderer", "relativity", "metric_kerr.cuh"),
           os.path.join("..", "src", "renderer", "relativity", "metric_schwarzschild.cuh"),
           os.path.join("..", "src", "renderer", "relativity", "metric_minkowski.cuh"),
           os.path.join("..", "src", "renderer", "bxdf", "matter.cuh"), os.path.join("..", "..", "include", "mgk.h"),
           os.path.join("..", "..", "include", "mgk_manager.h")]

NVCC_FLAGS = [
    "-std=c++17", "-O3", "-lineinfo",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-fmad=false",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-fvisibility=hidden",
    "-Xptxas", "-v",
]


def nvcc():
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [os.path.abspath(__file__)]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, out=None, defines=()):
    """Compiles libmgk.so (or `out`, with extra -D `defines`); the sources
    compile in parallel."""
    from concurrent.futures import ThreadPoolExecutor
    lib = out or LIB
    if not force and out is None and not _stale():
        return LIB
    bdir = os.path.join(os.path.dirname(lib) if out else HERE, "_build")
    os.makedirs(bdir, exist_ok=True)

    def compile_one(src):
        obj = os.path.join(bdir, src.replace(".cu", ".o"))
        cmd = [nvcc(), *NVCC_FLAGS, *[f"-D{d}" for d in defines], "-c", os.path.join(CSRC, src), "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
        if verbose:
            sys.stderr.write(r.stderr)
        with open(obj + ".ptxas.txt", "w") as f:
            f.write(r.stderr)
        return obj

    with ThreadPoolExecutor(max_workers=min(len(SOURCES), os.cpu_count() or 1)) as pool:
        objs = list(pool.map(compile_one, SOURCES))
    tmp = lib + ".tmp"
    cmd = [nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-cudart", "static",
           *objs, "-o", tmp]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, lib)
    return lib


# A variant of the library with a user metric plugin compiled in (the
# contract of src/renderer/relativity/metric.cuh): the test plugin of
# tests/plugin/metric_schwarzschild_user.cuh under tag 16.
USER_METRIC_HEADER = os.path.join(HERE, "..", "tests", "plugin", "metric_schwarzschild_user.cuh")
USER_METRIC_LIB = os.path.join(HERE, "..", "tests", "plugin", "libmgk_user_metric.so")


def user_metric_build(force=False):
    """Builds USER_METRIC_LIB (when missing or older than its sources)."""
    lib = os.path.abspath(USER_METRIC_LIB)
    header = os.path.abspath(USER_METRIC_HEADER)
    if not force and os.path.exists(lib):
        t = os.path.getmtime(lib)
        deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [header, os.path.abspath(__file__)]
        if all(os.path.getmtime(d) <= t for d in deps):
            return lib
    return build(out=lib, defines=(f'MGK_USER_METRIC_HEADER="{header}"',))


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
