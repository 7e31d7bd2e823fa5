"""The C-ABI library: it loads, exports every entry point include/*.h
declares, and rejects bad input before touching a GPU.  No compute calls
here -- those are the gpu-marked tests."""
import ctypes
import glob
import os
import re
import subprocess
import sys

import pytest

import gabe_b200 as gb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for hdr in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(hdr).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(gabe_[a-z0-9_]+)\s*\(", src, re.M):
            names.add(m.group(1))
    # static inline helpers of the dump format are not library exports
    return sorted(n for n in names if not n.startswith("gabe_dump_"))


def test_library_exports_every_declared_symbol():
    lib = gb.library()
    names = declared_functions()
    assert "gabe_step" in names and "gabe_create" in names
    out = subprocess.run(["nm", "-D", "--defined-only", gb.lib_path()], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (gabe_\w+)", out))
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    for n in names:
        getattr(lib, n)


def test_python_constants_match_the_header_enums():
    """Every GABE_FLAG_*, GABE_FP* and GABE_MODEL_* value of include/gabe.h
    has the same value in gabe_b200 (FLAG_*, FP*, MODEL_*)."""
    src = re.sub(r"/\*.*?\*/", "", open(os.path.join(ROOT, "include", "gabe.h")).read(), flags=re.S)
    enums = dict((m.group(1), int(m.group(2))) for m in re.finditer(r"\bGABE_((?:FLAG|MODEL)_\w+|FP32|FP64)\s*=\s*(\d+)",
                                                                     src))
    assert {"FLAG_OWN_FFT", "FLAG_CUFFT_3D", "FP32", "MODEL_LPHI4"} <= set(enums)
    for name, value in enums.items():
        assert getattr(gb, name) == value, name


def test_params_struct_matches_header():
    lib = gb.library()
    p = gb.Params()
    lib.gabe_default_params(ctypes.byref(p), 64)
    assert p.struct_size == ctypes.sizeof(gb.Params)
    assert p.N == 64 and p.nflds == 2 and p.expansion == 1
    assert gb.numbins(64) == lib.gabe_spectra_numbins(64) == 56
    assert gb.numbins(256) == 222 and gb.numbins(512) == 444 and gb.numbins(1024) == 887


@pytest.mark.parametrize("field,value", [("N", 63), ("N", 2), ("N", 6), ("N", 1290), ("nflds", 3), ("expansion", 3),
                                         ("expansion", -1), ("model", 7), ("precision", 5), ("dt", -1.0),
                                         ("gws_on", 2)])
def test_create_rejects_bad_params(field, value):
    lib = gb.library()
    p = gb.Params()
    lib.gabe_default_params(ctypes.byref(p), 32)
    setattr(p, field, value)
    h = ctypes.c_void_p()
    rc = lib.gabe_create(ctypes.byref(p), ctypes.byref(h))
    assert rc == 1 and not h.value
    assert lib.gabe_last_error(None)


@pytest.mark.parametrize("N,precision", [(6, 0), (10, 0), (1290, 0), (24, 1), (40, 1)])
def test_create_rejects_lattices_no_stencil_tile_divides(N, precision):
    """Even N that no stencil tile divides (FP64 tiles need N % 4 == 0, FP32
    tiles N % 16 == 0) are refused with a message, before any device work."""
    lib = gb.library()
    p = gb.Params()
    lib.gabe_default_params(ctypes.byref(p), N)
    p.precision = precision
    h = ctypes.c_void_p()
    assert lib.gabe_create(ctypes.byref(p), ctypes.byref(h)) == 1 and not h.value
    assert b"no stencil tile divides N" in lib.gabe_last_error(None)


@pytest.mark.parametrize("field,value", [("N", 6), ("N", 1290), ("model", 7), ("dt", float("nan")),
                                         ("L", float("inf")), ("expansion", 5)])
def test_energy_noalloc_rejects_bad_params_before_device_work(field, value):
    """gabe_energy_noalloc checks its parameters as gabe_create does and
    refuses untileable N; the refusal comes before any CUDA call (the device
    pointers here are never touched)."""
    lib = gb.library()
    p = gb.Params()
    lib.gabe_default_params(ctypes.byref(p), 32)
    setattr(p, field, value)
    dummy = ctypes.c_void_p(0x1000)
    assert lib.gabe_energy_noalloc(ctypes.byref(p), dummy, dummy, 1.0, dummy, None) == 1
    p2 = gb.Params()
    lib.gabe_default_params(ctypes.byref(p2), 32)
    p2.model, p2.model_c[0] = gb.MODEL_QUADRATIC, 0.0  # mphi = 0: the model constants divide by it
    assert lib.gabe_energy_noalloc(ctypes.byref(p2), dummy, dummy, 1.0, dummy, None) == 1


def test_null_handles_are_errors_not_crashes():
    lib = gb.library()
    assert lib.gabe_destroy(None) == 0
    assert lib.gabe_step(None, 1) == 1
    assert lib.gabe_sync(None) == 1
    out = (ctypes.c_double * 4)()
    assert lib.gabe_profile_steps(None, 1, out) == 1
    assert lib.gabe_profile_fft_passes(None, 1, out) == 1


def test_bench_counts_each_fft_pass_and_the_step_once():
    """bench.py's byte model: each pass of the library's FFT reads and
    writes its ten arrays once; the step's algorithmic bytes hold the
    transforms once -- in FP32 with GWs 56 (sweep A) + 32 (sweep B) +
    4 x 10 (1 + 2M/N^3) (one transform pass) + 4 x 36 M/N^3 (k-space) B per
    site-update, about 240 B for the device's five traceless components
    and four TT amplitudes (the reference's formulation, 336 B, is reported
    separately) -- and ncu traffic of the column passes scales with the
    k-points."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    N, w = 512, 4
    n3, M = N ** 3, N * N * (N // 2 + 1)
    b = bench.algorithmic_bytes(N, w, True)
    assert b["fft_rows"] == b["fft"] == 10 * (n3 + 2 * M) * w
    assert b["fft_j"] == b["fft_i"] == 10 * 4 * M * w
    assert b["fft_i_kspace"] == b["kspace"] == 36 * M * w
    step = sum(v for k, v in b.items() if k in ("stage1", "fft", "kspace", "stage2"))
    assert step == (56 + 32) * n3 + 40 * (n3 + 2 * M) + 144 * M
    assert abs(step / n3 - 240.4) < 0.1
    assert bench.reference_formulation_bytes(w, True) == 336
    assert set(bench.algorithmic_bytes(N, w, False)) == {"stage1", "stage2"}
    # the ensemble's step counts the transforms once (one pass), not once per pass on top
    for n in (32, 48, 64, 96, 128):
        n3e, Me = n ** 3, n * n * (n // 2 + 1)
        assert bench.ensemble_step_bytes(n) == (56 + 32) * n3e + 40 * (n3e + 2 * Me) + 144 * Me
    t256 = bench.traffic_scaled("fft_i_kspace", "fp32", 256)
    t512 = bench.traffic_scaled("fft_i_kspace", "fp32", 512)
    assert t256 and abs(t512 / t256 - M / (256 * 256 * 129)) < 1e-12


def test_oracle_library_loads():
    from oracle import pyoracle as po
    assert po.numbins(64) == 56


def test_bench_reference_arm_line():
    """bench.py --impl reference: the reference's own step() (or the oracle
    port when its binary is not built) prints one JSON line with the arm's
    contract keys on rank 0; other ranks print nothing and exit 0."""
    import json as _json

    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1", "--warmup", "0",
           "--ref-N", "128"]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    line = _json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["unit"] == "site-updates/s" and line["value"] > 0
    assert line["higher_is_better"] is True and line["metric"].startswith("site-updates/s")
    assert line["cpu_baseline"]["kind"] in ("reference", "port") and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    env = dict(os.environ, RANK="1", WORLD_SIZE="2")
    other = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT, env=env)
    assert other.returncode == 0 and not other.stdout.strip()


def test_wait_probe_refuses_bad_limits_before_any_device_call():
    """gabe_wait_probe checks its limit on the host (no GPU needed here)."""
    import gabe_b200 as gb

    assert gb.wait_probe(0)[0] == 1
    assert gb.wait_probe(-5)[0] == 1
    assert gb.wait_probe(20_000_000_000)[0] == 1
