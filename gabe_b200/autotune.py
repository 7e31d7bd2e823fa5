"""Stencil tile autotuner.

The two sweeps (include/gabe.h: tile_shape, tile_ci) are launched on a grid
of TJ x TK column tiles that each march `ci` planes along i.  The best pair
depends on N, the precision and whether the GW sources are written.  This
module times candidates on the current GPU with the library's own per-phase
CUDA events (gabe_profile_steps) and keeps the fastest per
(GPU name, N, precision, GWs) in a JSON cache, which `Lattice(...,
tile_shape="auto")` consults.

    python -m gabe_b200.autotune 64 128 256 512 --gws 1 --precision fp32
"""
from __future__ import annotations

import argparse
import json
import os

import numpy as np

from . import FP32, FP64, GabeError, Lattice

SHAPES = {0: (32, 8), 1: (16, 16), 2: (32, 4), 3: (16, 8), 4: (8, 8), 5: (4, 4)}  # FP64 sweeps
# ensemble work items (sites along k x j, 256-thread blocks): ens_tile_k/j in csrc/ensemble.cuh
ENS_SHAPES = {0: (64, 8), 1: (32, 16), 2: (16, 16)}
# FP32 single-lattice sweeps (two sites per thread along k): kShapes32 in csrc/launch.h
SHAPES32 = {0: (64, 8), 1: (64, 4), 2: (128, 4), 3: (32, 8), 4: (64, 16), 5: (32, 4), 6: (16, 8)}


def shapes_for(precision: int) -> dict:
    return SHAPES32 if precision == FP32 else SHAPES
CACHE = os.environ.get("GABE_TILE_CACHE", os.path.join(os.path.dirname(os.path.abspath(__file__)), "tiles.json"))


def _gpu_name() -> str:
    try:
        import torch

        return torch.cuda.get_device_name(0)
    except Exception:
        return "unknown"


def _key(N: int, precision: int, gws: bool) -> str:
    return f"{_gpu_name()}|N={N}|{'fp32' if precision == FP32 else 'fp64'}|gws={int(gws)}"


def load_cache() -> dict:
    if os.path.exists(CACHE):
        with open(CACHE) as fh:
            return json.load(fh)
    return {}


def lookup(N: int, precision: int, gws: bool):
    """(tile_shape, tile_ci) from the cache, or None."""
    e = load_cache().get(_key(N, precision, gws))
    return (e["shape"], e["ci"]) if e else None


def lookup_ensemble(N: int):
    """(shape, ci) for ensemble lattices of size N, or None."""
    e = load_cache().get(f"{_gpu_name()}|ens32|N={N}")
    return (e["shape"], e["ci"]) if e else None


def tune_ensemble(sizes, steps: int = 6, verbose: bool = True) -> dict:
    """Ensemble tiles per lattice size: every shape of ENS_SHAPES that
    divides N and ci in {8, 16, 32, 64}, timed (CUDA events on the
    ensemble's stream) on an ensemble of ~32M sites of lattices of that size."""
    import torch

    from . import Ensemble

    out = {}
    cache = load_cache()
    for N in sizes:
        nl = max(1, (1 << 25) // N ** 3)
        best = None
        for shape, (tk, tj) in ENS_SHAPES.items():
            if N % tk or N % tj:
                continue
            for ci in (8, 16, 32, 64):
                if ci > N:
                    continue
                with Ensemble([N] * nl, [100.0] * nl, [1.0] * nl, list(range(nl)), nlog=8,
                              tiles=([shape] * nl, [ci] * nl)) as ens:
                    ens.init()
                    ens.step(2)
                    st = torch.cuda.ExternalStream(ens.stream_ptr)
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record(st)
                    ens.step(steps)
                    e1.record(st)
                    e1.synchronize()
                    t = e0.elapsed_time(e1) / steps
                if verbose:
                    print(f"ens N={N} x {nl} shape {ENS_SHAPES[shape]} ci {ci}: {t:.4f} ms/step", flush=True)
                if best is None or t < best[2]:
                    best = (shape, ci, t)
        cache[f"{_gpu_name()}|ens32|N={N}"] = {"shape": best[0], "ci": best[1], "step_ms": best[2],
                                               "lattices": nl, "tile": ENS_SHAPES[best[0]]}
        out[N] = best
    with open(CACHE, "w") as fh:
        json.dump(cache, fh, indent=1, sort_keys=True)
    return out


def candidates(N: int, precision: int = FP32):
    out = []
    for s, (tk, tj) in shapes_for(precision).items():
        if tk > N or tj > N or N % tk or N % tj:
            continue
        for ci in (16, 32, 64, 128, 256, 512):
            if ci <= N:
                out.append((s, ci))
    return out


def tune(N: int, precision: int = FP32, gws: bool = True, steps: int = 3, verbose: bool = True) -> dict:
    """Times every candidate on a random state; returns and caches the best."""
    rng = np.random.default_rng(0)
    f = 0.342 + 1e-6 * rng.standard_normal((2, N, N, N))
    f[1] -= 0.342
    d = 1e-6 * rng.standard_normal((2, N, N, N))
    results = []
    table = shapes_for(precision)
    for shape, ci in candidates(N, precision):
        try:
            with Lattice(N, gws=gws, precision=precision, tile_shape=shape, tile_ci=ci) as lat:
                lat.upload_state(f, d, a0=1.0, adot0=0.5)
                lat.profile_steps(1)
                ph = lat.profile_steps(steps)
        except GabeError as e:
            if verbose:
                print(f"shape {table[shape]} ci {ci}: {e}")
            continue
        t = ph["stage1"] + ph["stage2"]
        results.append({"shape": shape, "ci": ci, "sweeps_ms": t, "stage1": ph["stage1"], "stage2": ph["stage2"]})
        if verbose:
            print(f"shape {table[shape]} ci {ci:4d}: sweep A {ph['stage1']:.3f} ms  sweep B {ph['stage2']:.3f} ms",
                  flush=True)
    best = min(results, key=lambda r: r["sweeps_ms"])
    cache = load_cache()
    cache[_key(N, precision, gws)] = {"shape": best["shape"], "ci": best["ci"], "sweeps_ms": best["sweeps_ms"],
                                      "tile": table[best["shape"]]}
    with open(CACHE, "w") as fh:
        json.dump(cache, fh, indent=1, sort_keys=True)
    return {"best": best, "all": results}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("N", type=int, nargs="+")
    ap.add_argument("--gws", type=int, default=1)
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--ensemble", action="store_true", help="tune the ensemble's work-item tiles instead")
    a = ap.parse_args()
    if a.ensemble:
        return tune_ensemble(a.N, a.steps)
    out = {}
    for N in a.N:
        r = tune(N, FP32 if a.precision == "fp32" else FP64, bool(a.gws), a.steps)
        out[N] = r["best"]
        print(json.dumps({"N": N, "best": r["best"]}), flush=True)
    return out


if __name__ == "__main__":
    main()
