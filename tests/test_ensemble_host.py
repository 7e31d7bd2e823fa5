"""Host-side logic of the batched ensemble, on the CPU: parameter checks of
gabe_ensemble_create (made before any CUDA call), the sweep's parameter
draw, the sum-N^3 partition over ranks and the gather of per-lattice rows
through a world-size-2 gloo process group."""
import ctypes
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import gabe_b200 as gb
from gabe_b200 import ensemble as ge


def _params(N, g=None, amp=None, seed=None, **kw):
    N = np.ascontiguousarray(N, dtype=np.int32)
    n = len(N)
    g = np.ascontiguousarray(g if g is not None else [100.0] * n, dtype=np.float64)
    amp = np.ascontiguousarray(amp if amp is not None else [1.0] * n, dtype=np.float64)
    seed = np.ascontiguousarray(seed if seed is not None else list(range(1, n + 1)), dtype=np.uint64)
    p = gb.EnsParams()
    p.struct_size = ctypes.sizeof(gb.EnsParams)
    p.nlat = n
    p.N = N.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
    p.g2_over_lambda = g.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    p.amplitude = amp.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    p.seed = seed.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))
    p.L, p.dt, p.lam, p.phi0, p.dphi0 = 20.0, 0.01, 9e-14, 0.342, 0.0
    p.gws_on, p.device, p.nlog, p.gw_spec_quirk = 1, -1, 64, 1
    for k, v in kw.items():
        setattr(p, k, v)
    return p, (N, g, amp, seed)


@pytest.mark.parametrize("case", ["N_not_16", "N_small", "neg_amp", "nan_g", "nlog0", "dt0", "nlat0", "size",
                                  "log_top", "cut_neg", "smooth0", "det_without_cut", "det_2"])
def test_ensemble_create_rejects_bad_params(case):
    lib = gb._ens_lib()
    N, g, amp, kw = [32, 48], None, None, {}
    if case == "N_not_16":
        N = [32, 40]
    elif case == "N_small":
        N = [8]
    elif case == "neg_amp":
        amp = [1.0, -0.5]
    elif case == "nan_g":
        g = [float("nan"), 1.0]
    elif case == "nlog0":
        kw = {"nlog": 0}
    elif case == "dt0":
        kw = {"dt": 0.0}
    elif case == "nlat0":
        kw = {"nlat": 0}
    elif case == "size":
        kw = {"struct_size": 8}
    elif case == "log_top":
        kw = {"log_top_bin": -1}
    elif case == "cut_neg":
        kw = {"spec_cut_off": -0.1}
    elif case == "smooth0":
        kw = {"spec_cut_off": 0.25, "spec_smooth": 0.0}
    elif case == "det_without_cut":
        kw = {"ic_deterministic": 1}
    elif case == "det_2":
        kw = {"spec_cut_off": 0.25, "spec_smooth": 0.5, "ic_deterministic": 2}
    p, keep = _params(N, g, amp, **kw)
    h = ctypes.c_void_p()
    assert lib.gabe_ensemble_create(ctypes.byref(p), ctypes.byref(h)) == 1
    assert not h.value
    assert lib.gabe_ensemble_last_error(None)


@pytest.mark.parametrize("N,shape", [(96, 0), (48, 1), (64, 3), (64, -1)])
def test_ensemble_create_rejects_tile_shapes_that_do_not_divide_N(N, shape):
    """Work-item shapes: 0 = 64x8 sites (N % 64 == 0), 1 = 32x16 (N % 32 == 0),
    2 = 16x16 (any N % 16 == 0)."""
    lib = gb._ens_lib()
    shapes = np.array([shape], dtype=np.int32)
    cis = np.array([16], dtype=np.int32)
    p, keep = _params([N], tile_shape=shapes.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                      tile_ci=cis.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))
    h = ctypes.c_void_p()
    assert lib.gabe_ensemble_create(ctypes.byref(p), ctypes.byref(h)) == 1
    assert not h.value
    assert b"tile shape" in lib.gabe_ensemble_last_error(None)


def test_ensemble_null_handles_are_errors():
    lib = gb._ens_lib()
    assert lib.gabe_ensemble_destroy(None) == 0
    assert lib.gabe_ensemble_step(None, 1) == 1
    assert lib.gabe_ensemble_sync(None) == 1
    assert lib.gabe_ensemble_native_bins(None) == 0
    assert lib.gabe_ensemble_launches_per_step(None) == 0
    assert lib.gabe_ensemble_stream(None) is None


def test_sweep_parameters_follow_the_stated_distributions():
    N, g, amp, seeds = ge.sample_parameters(4096, 7)
    assert set(np.unique(N)) == set(ge.SIZES)
    assert np.all((g >= 1.0) & (g <= 500.0)) and np.all((amp >= 0.5) & (amp <= 2.0))
    # log-uniform: log g is uniform, its mean is the midpoint
    lg = np.log(g)
    assert abs(lg.mean() - 0.5 * np.log(500.0)) < 0.1
    assert len(np.unique(seeds)) == 4096
    N2, g2, a2, s2 = ge.sample_parameters(4096, 7)
    assert np.array_equal(N, N2) and np.array_equal(g, g2) and np.array_equal(seeds, s2)


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_partition_is_complete_and_balanced(world):
    N, *_ = ge.sample_parameters(256, 11)
    parts = ge.partition(N, world)
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(256))
    loads = [sum(int(N[i]) ** 3 for i in p) for p in parts]
    # LPT: no rank is more than one largest lattice above the lightest
    assert max(loads) - min(loads) <= 128 ** 3


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _gather_worker(rank, world, port, nlat, N, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        parts = ge.partition(N, world)
        mine = parts[rank]
        # each rank "evolves" its lattices: rows that encode the lattice index
        rows = np.stack([np.full((3, 4), float(i)) + np.arange(4) for i in mine]) if mine else np.zeros((0, 3, 4))
        full = ge.gather_rows(mine, rows, nlat, dist)
        if rank == 0:
            want = np.stack([np.full((3, 4), float(i)) + np.arange(4) for i in range(nlat)])
            q.put(bool(np.array_equal(full, want)))
        else:
            q.put(full is None)
    finally:
        dist.destroy_process_group()


def test_gather_over_two_gloo_ranks():
    nlat = 37
    N, *_ = ge.sample_parameters(nlat, 3)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gather_worker, args=(r, 2, port, nlat, N, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs)
    res = [q.get(timeout=5) for _ in range(2)]
    assert all(res)


def test_gather_without_a_group_places_rows():
    rows = np.arange(6.0).reshape(3, 2)
    out = ge.gather_rows([2, 0, 1], rows, 3)
    assert np.array_equal(out, np.array([[2.0, 3.0], [4.0, 5.0], [0.0, 1.0]]))
