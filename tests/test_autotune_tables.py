"""The autotuner's tile tables against the library's, and its committed
cache (gabe_b200/tiles.json), on the CPU: the FP32 shapes are launch.h's
kShapes32, the FP64 ones the cases of kernels_f64.cu's sweep_f64, the
ensemble ones ensemble.cuh's ens_tile_k/j; every cached choice names a
shape of its table that tiles its N, with ci <= N."""
import json
import os
import re

import pytest

from gabe_b200 import FP32, FP64, autotune

CSRC = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "gabe_b200", "csrc")


def _src(name):
    return open(os.path.join(CSRC, name)).read()


def test_fp32_shapes_are_launch_h_kShapes32():
    m = re.search(r"kShapes32\[kNumShapes32\]\[2\]\s*=\s*\{(.*?)\};", _src("launch.h"), re.S)
    pairs = [tuple(int(v) for v in p) for p in re.findall(r"\{(\d+),\s*(\d+)\}", m.group(1))]
    assert pairs == [autotune.SHAPES32[s] for s in range(len(pairs))]


def test_fp64_shapes_are_the_sweep_f64_cases():
    cases = re.findall(r"case (\d+): return sweep_shape<(\d+), (\d+)>", _src("kernels_f64.cu"))
    assert {int(s): (int(k), int(j)) for s, k, j in cases} == autotune.SHAPES


def test_ensemble_shapes_are_ens_tile_k_and_j():
    src = _src("ensemble.cuh")
    tk = re.search(r"ens_tile_k\(int shape\) \{ return shape == 0 \? (\d+) : \(shape == 1 \? (\d+) : (\d+)\); \}", src)
    tj = re.search(r"ens_tile_j\(int shape\) \{ return shape == 0 \? (\d+) : (\d+); \}", src)
    k = [int(v) for v in tk.groups()]
    j = [int(tj.group(1)), int(tj.group(2)), int(tj.group(2))]
    assert {s: (k[s], j[s]) for s in range(3)} == autotune.ENS_SHAPES


def _cache_entries():
    with open(os.path.join(os.path.dirname(CSRC), "tiles.json")) as fh:
        return sorted(json.load(fh).items())


@pytest.mark.parametrize("key,entry", _cache_entries())
def test_cached_choices_tile_their_lattice(key, entry):
    N = int(re.search(r"N=(\d+)", key).group(1))
    if "|ens32|" in key:
        table = autotune.ENS_SHAPES
    else:
        table = autotune.shapes_for(FP32 if "|fp32|" in key else FP64)
    tk, tj = table[entry["shape"]]
    assert list(entry["tile"]) == [tk, tj]
    assert N % tk == 0 and N % tj == 0 and 1 <= entry["ci"] <= N


@pytest.mark.parametrize("N", [32, 48, 64, 96, 128, 512])
@pytest.mark.parametrize("precision", [FP32, FP64])
def test_candidates_only_name_tiles_that_fit(N, precision):
    cands = autotune.candidates(N, precision)
    assert cands
    for s, ci in cands:
        tk, tj = autotune.shapes_for(precision)[s]
        assert N % tk == 0 and N % tj == 0 and ci <= N
