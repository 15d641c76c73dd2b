"""Build the native parts in-tree.

    libipole_b200.so   ipole_b200/_build/   CUDA kernels for sm_100a + host C
    ipole_b200         ipole_b200/bin/      the command-line program

nvcc compiles the kernels (``-gencode arch=compute_100a,code=sm_100a``),
gcc the host C with ``-ffp-contract=off`` so that host set-up arithmetic
(camera tetrad, derived fluid fields) keeps the reference's operation order.
Run ``python -m ipole_b200.build`` or call :func:`build`.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
HOST = os.path.join(CSRC, "host")
BUILD = os.path.join(HERE, "_build")
BIN = os.path.join(HERE, "bin")
INC = os.path.join(ROOT, "include")
LIB = os.path.join(BUILD, "libipole_b200.so")
CLI = os.path.join(BIN, "ipole_b200")

NVCC_FLAGS = ["-std=c++17", "-O3", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
              "-Xcompiler", "-fPIC,-ffp-contract=off", "-Xptxas", "-v"]
CC_FLAGS = ["-std=gnu99", "-O2", "-fPIC", "-ffp-contract=off", "-fopenmp", "-Wall", "-Wno-unused-result"]
CU_EXTRA = ["ipg_refine.cu"]
HOST_SRC = ["ipgc.c", "h5lite.c", "plugins.c", "trace.c", "coords.c", "par.c", "model_iharm.c", "camera.c", "render.c",
            "model_api.c"]


def _nvcc() -> str:
    for c in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _cc() -> str:
    return shutil.which("gcc") or "gcc"


def _sources():
    srcs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cuh", ".h"))]
    srcs += [os.path.join(HOST, f) for f in os.listdir(HOST) if f.endswith((".c", ".h"))]
    srcs += [os.path.join(INC, f) for f in os.listdir(INC) if f.endswith(".h")]
    return srcs


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, log):
    if log:
        print(" ".join(cmd), file=log)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build step failed ({r.returncode}): {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return r.stdout + r.stderr


def build(force: bool = False, verbose: bool = False, defines=(), out_dir: str | None = None) -> str:
    """Compile the kernels and host library (and the CLI) if sources changed.
    Returns the path of libipole_b200.so.  ``defines`` (e.g.
    ["IPG_XFER_MINB=2"]) and ``out_dir`` build a variant library elsewhere
    (no CLI) for code-generation experiments."""
    log = sys.stderr if verbose else None
    bdir = out_dir or BUILD
    lib = os.path.join(bdir, "libipole_b200.so")
    os.makedirs(bdir, exist_ok=True)
    os.makedirs(BIN, exist_ok=True)
    deps = _sources()
    if force or out_dir or _stale(lib, deps) or _stale(CLI, deps + [lib]):
        objs = []
        ko = os.path.join(bdir, "ipg_kernels.o")
        dflags = [f"-D{d}" for d in defines]
        out = _run([_nvcc(), *NVCC_FLAGS, *dflags, "-I", INC, "-c", os.path.join(CSRC, "ipg_kernels.cu"), "-o", ko],
                   log)
        with open(os.path.join(bdir, "ptxas.txt"), "w") as f:
            f.write(out)
        objs.append(ko)
        for cu in CU_EXTRA:
            o = os.path.join(bdir, cu[:-3] + ".o")
            # no multiply-add contraction: the image driver must round as the host driver does
            out = _run([_nvcc(), *NVCC_FLAGS, "-fmad=false", *dflags, "-I", INC, "-c", os.path.join(CSRC, cu),
                        "-o", o], log)
            with open(os.path.join(bdir, f"ptxas_{cu[:-3]}.txt"), "w") as f:
                f.write(out)
            objs.append(o)
        for s in HOST_SRC:
            o = os.path.join(bdir, s[:-2] + ".o")
            _run([_cc(), *CC_FLAGS, "-I", INC, "-c", os.path.join(HOST, s), "-o", o], log)
            objs.append(o)
        tmp = lib + ".tmp"
        _run([_nvcc(), "-shared", "-Xcompiler", "-fPIC,-fopenmp", "-o", tmp, *objs, "-lz", "-lm"], log)
        os.replace(tmp, lib)
        if not out_dir:
            _run([_cc(), *CC_FLAGS, "-I", INC, os.path.join(HOST, "main.c"), "-o", CLI, "-L", BUILD,
                  "-lipole_b200", "-Wl,-rpath,$ORIGIN/../_build", "-lm"], log)
    return lib


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
