"""Builds libmbt.so in place: the C host (gcc) and the sm_100a CUDA kernels
with the C-ABI (nvcc), linked into one shared library next to this file.

Run as ``python -m mbtrack_b200.build``; __graft_entry__.build() calls it.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libmbt.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

# Multiply-adds contract to FMA; the expressions whose rounding the parity
# bars depend on (betatron phase, RF argument, bin index) are written with
# explicit round-to-nearest intrinsics in the kernels.
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
                     "-Xcompiler", "-fPIC", "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]
# host C: no contraction of multiply-adds, as in the reference's x86-64 build
CC_FLAGS = ["-O2", "-fPIC", "-std=gnu11", "-Wall", "-ffp-contract=off", "-I" + os.path.join(ROOT, "include")]

CU_SOURCES = ["mbt_runtime.cu", "mbt_step.cu", "mbt_fields.cu", "mbt_mlp.cu", "mbt_tune.cu", "mbt_ws.cu"]
# per-file extra flags: w(z) and the BE field keep every multiply and add
# separately rounded, as the reference's x86-64 build does
CU_EXTRA = {"mbt_fields.cu": ["-fmad=false"], "mbt_ws.cu": ["-fmad=false"]}
C_SOURCES = ["mbt_host.c", "mbt_beam.c", "mbt_output.c", "mbt_ws_output.c"]
# the drop-in executable for mbtrack-mpi's weak-weak runs
CLI_SOURCE = "mbtrack_gpu.c"
CLI = os.path.join(HERE, "mbtrack-gpu")
HEADERS = ["mbt_beamion.cuh", "mbt_common.cuh", "mbt_gauss.cuh", "mbt_device.cuh", "mbt_kernels.cuh", "mbt_mlp.cuh", "mbt_philox.cuh",
           "mbt_wofz.cuh"]


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose_ptxas=False, force=False):
    os.makedirs(BUILD, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", h) for h in ("mbt.h", "mbt_ws.h")]
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if force or _stale(o, [s] + hdrs):
            extra = (["-Xptxas", "-v"] if verbose_ptxas else []) + CU_EXTRA.get(src, [])
            _run([NVCC] + NVCC_FLAGS + extra + ["-c", s, "-o", o])
        objs.append(o)
    for src in C_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if force or _stale(o, [s] + hdrs):
            _run(["gcc"] + CC_FLAGS + ["-c", s, "-o", o])
        objs.append(o)
    if force or _stale(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart", "-lm"])
    cli_src = os.path.join(CSRC, CLI_SOURCE)
    if force or _stale(CLI, [cli_src, LIB] + hdrs):
        _run(["gcc"] + CC_FLAGS + [cli_src, "-o", CLI, "-L" + HERE, "-lmbt", "-lpthread", "-lm",
                                   "-Wl,-rpath,$ORIGIN"])
    return LIB


if __name__ == "__main__":
    build(verbose_ptxas="-v" in sys.argv, force="-f" in sys.argv)
