"""Build recipe for libgabe_b200.so (sm_100a) -- run `python -m gabe_b200.build`.

The library is a plain C-ABI shared object (include/gabe.h) built in-tree by
nvcc so that it travels with the source tree.  kernels_f64.cu is compiled
with -fmad=false: the FP64 path rounds every multiply and add separately,
like the reference's x86-64 build.  kernels_f32.cu and api.cu use the
default contraction.
"""
from __future__ import annotations

import concurrent.futures
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(ROOT, "_build", "gabe_b200")
LIB = os.path.join(HERE, "libgabe_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I" + os.path.join(ROOT, "include")]
UNITS = [
    ("api.cu", []),
    ("kernels_f64.cu", ["-fmad=false"]),
    ("kernels_f32.cu", []),
    ("fft3d.cu", []),
    ("fftt.cu", []),
    ("noalloc.cu", ["-fmad=false"]),
    ("ensemble.cu", []),
    ("slab.cu", []),
    ("mlp.cu", []),
    ("probe.cu", []),
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _deps() -> list[str]:
    out = []
    for d in (CSRC, os.path.join(ROOT, "include")):
        for f in os.listdir(d):
            if f.endswith((".cu", ".cuh", ".h")):
                out.append(os.path.join(d, f))
    return out


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(p) <= t for p in _deps() + [__file__])


def build(force: bool = False, verbose: bool = False, ptxas_v: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    nv = nvcc()

    def compile_unit(unit):
        src, extra = unit
        obj = os.path.join(BUILD, src.replace(".cu", ".o"))
        cmd = [nv, *ARCH, *COMMON, *extra, "-c", os.path.join(CSRC, src), "-o", obj]
        if ptxas_v:
            cmd += ["-Xptxas", "-v"]
        return obj, cmd, subprocess.run(cmd, capture_output=True, text=True)

    # the units are independent: compile them side by side, report in order
    workers = max(1, min(len(UNITS), os.cpu_count() or 1))
    with concurrent.futures.ThreadPoolExecutor(max_workers=workers) as pool:
        results = list(pool.map(compile_unit, UNITS))
    objs = []
    for (src, _), (obj, cmd, r) in zip(UNITS, results):
        if verbose:
            print(" ".join(cmd), flush=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
        if ptxas_v or verbose:
            sys.stdout.write(r.stderr)
        objs.append(obj)
    tmp = LIB + ".tmp"
    cmd = [nv, *ARCH, "-shared", "-o", tmp, *objs, "-lcufft", "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_v="--ptxas-v" in sys.argv)
    print(LIB)
