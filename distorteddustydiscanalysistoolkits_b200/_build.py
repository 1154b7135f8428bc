"""Build libpartia_b200.so in-tree with nvcc for sm_100a.

Each CUDA translation unit is compiled separately so that the FP64 units that must
reproduce the reference's IEEE results bit for bit get -fmad=false (no FMA contraction),
while the FP32-compensated unit keeps FMA.  Objects go to <repo>/_build/, the shared
library next to this file.  The line-integrated kernel tables are regenerated from the
kernel formulas first (csrc/gen_line_tables.py).
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(REPO, "include")
OBJDIR = os.path.join(REPO, "_build")
LIB = os.path.join(PKG, "libpartia_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", CSRC, "-I", INCLUDE,
                 "-Xptxas", "-warn-spills"]
UNITS = {
    "pb_build.cu": ["-fmad=false"],
    "pb_interp64.cu": ["-fmad=false"],
    "pb_query.cu": ["-fmad=false"],
    "pb_walk.cu": ["-fmad=false"],
    "pb_sched.cu": ["-fmad=false"],
    "pb_interp32.cu": ["-fmad=false"],   # FMAs only where written (fmaf): bits independent of code shape
    "pb_capi.cu": [],
    "pb_noalloc.cu": ["-fmad=false"],
    "pb_input.cu": ["-fmad=false"],
    "pb_batch.cu": ["-fmad=false"],
}
HEADERS = ["pb_device.cuh", "pb_internal.h", "pb_interp_impl.cuh", "pb_fp32_impl.cuh", "pb_fp64_impl.cuh", "pb_walk_impl.cuh",
           "line_tables.h"]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def gen_tables(force=False):
    out = os.path.join(CSRC, "line_tables.h")
    gen = os.path.join(CSRC, "gen_line_tables.py")
    if force or _newer(out, [gen]):
        subprocess.check_call([sys.executable, gen, out])
    return out


def build(verbose=False, force=False, extra=()):
    """Compile every unit and link the shared library; returns its path."""
    gen_tables()
    os.makedirs(OBJDIR, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "partia_b200.h")]
    jobs = []
    for unit, flags in UNITS.items():
        src = os.path.join(CSRC, unit)
        obj = os.path.join(OBJDIR, unit.replace(".cu", ".o"))
        if force or _newer(obj, [src] + hdrs):
            jobs.append([NVCC] + COMMON + list(flags) + list(extra) + ["-c", src, "-o", obj])

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed:\n%s\n%s\n%s" % (" ".join(cmd), r.stdout, r.stderr))
        return r.stderr

    with ThreadPoolExecutor(max_workers=len(UNITS)) as ex:
        logs = list(ex.map(run, jobs))
    if verbose:
        for log in logs:
            sys.stderr.write(log)
    objs = [os.path.join(OBJDIR, u.replace(".cu", ".o")) for u in UNITS]
    if force or jobs or _newer(LIB, objs):
        subprocess.check_call([NVCC] + ARCH + ["-shared", "-o", LIB] + objs)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print(LIB)
