"""Build recipe for the package's native libraries (sm_100a only).

Produces, inside the package directory (so they travel with the source tree):
  libbgk3d_b200.so        the library (C ABI of include/bgk3d_b200.h)
  libbgk3d_dropin_sp.so   reference-named symbols, real_t = float
  libbgk3d_dropin_dp.so   reference-named symbols, real_t = double
All CUDA code is compiled with --fmad=false: every add and multiply rounds
separately, in the reference's source order, which makes FP32/FP64 results
bit-identical to a strict IEEE restatement of the reference loops.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "--fmad=false", "-std=c++17",
    "-Xcompiler", "-fPIC",
    "-I" + INCLUDE, "-I" + CSRC,
]

LIB_SOURCES = ["bgk_api.cu", "lattice.cu", "lattice_io.cu", "diag.cu", "batch.cu", "noalloc.cu", "devmem.cu"] + [
    f"inst_{kind}_{group}.cu" for kind in ("f64", "f32", "f16", "bf16", "f32f64") for group in ("ab", "aa", "batch", "misc")]
LIB = "libbgk3d_b200.so"
DROPIN_SP = "libbgk3d_dropin_sp.so"
DROPIN_DP = "libbgk3d_dropin_dp.so"


def _nvcc() -> str:
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(exe):
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build bgk3d_gpu_b200")
    return exe


def _run(cmd: list[str]) -> None:
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + res.stdout + res.stderr)


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _deps() -> list[str]:
    out = []
    for d in (CSRC, INCLUDE):
        for f in os.listdir(d):
            if f.endswith((".cu", ".cuh", ".h")):
                out.append(os.path.join(d, f))
    out.append(os.path.abspath(__file__))
    return out


def build(force: bool = False, verbose: bool = False) -> dict:
    """Compile every native library of the package; returns their paths."""
    nvcc = _nvcc()
    deps = _deps()
    lib = os.path.join(PKG, LIB)
    objs = []
    jobs = []
    for src in LIB_SOURCES:
        srcp = os.path.join(CSRC, src)
        if not os.path.exists(srcp):
            continue
        obj = os.path.join(PKG, "_build", src.replace(".cu", ".o"))
        objs.append(obj)
        if force or _stale(obj, deps):
            jobs.append([nvcc, *NVCC_FLAGS, "-c", srcp, "-o", obj])
    os.makedirs(os.path.join(PKG, "_build"), exist_ok=True)
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        for cmd in jobs:
            if verbose:
                print(" ".join(cmd), file=sys.stderr)
        list(ex.map(_run, jobs))
    if force or jobs or _stale(lib, objs):
        _run([nvcc, *ARCH, "-shared", "-o", lib, *objs, "-lcudart"])
    out = {"lib": lib}
    dropin_jobs = []
    for name, extra in ((DROPIN_SP, []), (DROPIN_DP, ["-DDOUBLE_P"])):
        tgt = os.path.join(PKG, name)
        out[name] = tgt
        if force or _stale(tgt, deps + [lib]):
            dropin_jobs.append([nvcc, *NVCC_FLAGS, *extra, "-shared", os.path.join(CSRC, "dropin.cu"),
                                "-o", tgt, "-L" + PKG, "-lbgk3d_b200", "-Xlinker", "-rpath=$ORIGIN",
                                "-lcudart"])
    with ThreadPoolExecutor(max_workers=2) as ex:
        list(ex.map(_run, dropin_jobs))
    return out


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
