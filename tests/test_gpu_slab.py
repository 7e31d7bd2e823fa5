"""A lattice split into slabs along i (gabe_slab_* through gabe_b200.slab)
against the same lattice on one handle (gabe_create).

* One slab holds the whole lattice between two halo planes that are copies
  of its own end planes: same tiles, same plane chunks, the same block sums
  in the same order, so FP64 results are bit for bit those of the handle --
  through the in-process communicator and through a one-rank NCCL group.
* Several slabs in one process (the ranks' kernels never wait on each
  other: sums are added on the host, halos copied between steps) differ
  from the handle only in the order of the energy sums: FP64 to ~1e-12,
  FP32 (fluctuations about the FP64 mean) to its rounding.
* With GWs the slabs transform their source planes in 2-D, transpose the
  half spectra between them by ky columns and take the pass along i and
  the h/l update of their own k-points; h and l agree with the handle's
  3-D cuFFT path to transform rounding (FP32 or FP64).
"""
import os
import socket

import numpy as np
import pytest
import torch

import gabe_b200 as gb
from gabe_b200 import slab as gs
from gabe_b200.ic import random_state

pytestmark = pytest.mark.gpu

STEPS = 6


def _state(N, seed=5):
    f, d, a0, ad0 = random_state(N, seed=seed)
    return f.numpy(), d.numpy(), a0, ad0


def _whole(N, precision, st, steps, **kw):
    f, d, a0, ad0 = st
    with gb.Lattice(N, precision=precision, **kw) as lat:
        lat.upload_state(f, d, a0=a0, adot0=ad0)
        lat.step(steps)
        sc = lat.scalars()
        f1, d1, _, _ = lat.download_state()
    want = np.array([v for k in ("a", "adot", "edkin", "edpot", "edgrad", "edrho") for v in sc[k]])
    return f1, d1, want


def _slabs(N, precision, st, steps, comm, **kw):
    f, d, a0, ad0 = st
    with gs.SlabLattice(N, comm, precision=precision, **kw) as lat:
        fs = [f[:, p0:p0 + n] for p0, n in lat.planes]
        ds = [d[:, p0:p0 + n] for p0, n in lat.planes]
        lat.upload(fs if len(fs) > 1 else fs[0], ds if len(ds) > 1 else ds[0], a0, ad0)
        lat.step(steps)
        sc = lat.scalars()
        per = [s.scalars() for s in lat.slabs]
        out = lat.download()
    f1 = np.concatenate([o[0] for o in out], axis=1)
    d1 = np.concatenate([o[1] for o in out], axis=1)
    for p in per[1:]:
        np.testing.assert_array_equal(p, per[0])  # every slab holds the same scalars
    return f1, d1, sc


def test_one_slab_is_the_whole_lattice_bitwise():
    N = 32
    st = _state(N)
    f0, d0, s0 = _whole(N, gb.FP64, st, STEPS)
    f1, d1, s1 = _slabs(N, gb.FP64, st, STEPS, gs.LocalComm(1))
    np.testing.assert_array_equal(f1, f0)
    np.testing.assert_array_equal(d1, d0)
    np.testing.assert_array_equal(s1, s0)


@pytest.mark.parametrize("world", [2, 3, 4])
def test_slabs_match_the_whole_lattice_fp64(world):
    N = 32
    st = _state(N, seed=9)
    f0, d0, s0 = _whole(N, gb.FP64, st, STEPS)
    f1, d1, s1 = _slabs(N, gb.FP64, st, STEPS, gs.LocalComm(world))
    # the fields see the scalars only through a and adot, which differ in the last bits
    for x, y in ((f1, f0), (d1, d0)):
        for fld in range(2):
            fl = y[fld] - y[fld].mean()
            assert np.abs(x[fld] - y[fld]).max() <= 1e-10 * np.abs(fl).max()
    rho = s0[10]
    for q in range(12):
        tol = 1e-12 * (abs(rho) if q in (8, 9) else abs(s0[q]))
        assert abs(s1[q] - s0[q]) <= tol, (q, s1[q], s0[q])


@pytest.mark.parametrize("case", ["expansion0", "expansion2", "quadratic", "one_plane_slabs"])
def test_slab_variants_match_the_whole_lattice_fp64(case):
    """expansion_type 0 and 2, the shipped m^2 phi^2 + g^2 phi^2 chi^2 model,
    and slabs of a single plane (every halo plane is a neighbour's)."""
    N, world, kw = 32, 4, {}
    if case == "expansion0":
        kw = {"expansion": 0}
    elif case == "expansion2":
        kw = {"expansion": 2}
    elif case == "quadratic":
        kw = {"model": gb.MODEL_QUADRATIC, "model_c": (1e-6, 2.5e-7)}
    else:
        N, world = 16, 16
    if case == "quadratic":
        f, d, a0, ad0 = random_state(N, seed=17, model=gb.MODEL_QUADRATIC, model_c=(1e-6, 2.5e-7), f0=(1.0, 0.0))
        st = (f.numpy(), d.numpy(), a0, ad0)
    else:
        st = _state(N, seed=17)
    f0, d0, s0 = _whole(N, gb.FP64, st, STEPS, **kw)
    f1, d1, s1 = _slabs(N, gb.FP64, st, STEPS, gs.LocalComm(world), **kw)
    for x, y in ((f1, f0), (d1, d0)):
        for fld in range(2):
            fl = y[fld] - y[fld].mean()
            assert np.abs(x[fld] - y[fld]).max() <= 1e-10 * max(np.abs(fl).max(), 1e-300)
    rho = s0[10]
    for q in range(12):
        tol = 1e-12 * (abs(rho) if q in (8, 9) else abs(s0[q])) + 1e-300
        assert abs(s1[q] - s0[q]) <= tol, (case, q, s1[q], s0[q])


def test_slabs_match_the_whole_lattice_fp32():
    N = 64
    st = _state(N, seed=13)
    f0, d0, s0 = _whole(N, gb.FP32, st, STEPS)
    f1, d1, s1 = _slabs(N, gb.FP32, st, STEPS, gs.LocalComm(3))
    for x, y in ((f1, f0), (d1, d0)):
        for fld in range(2):
            fl = y[fld] - y[fld].mean()
            assert np.abs(x[fld] - y[fld]).max() <= 1e-5 * np.abs(fl).max()
    rho = s0[10]
    for q in range(12):
        tol = 1e-6 * (abs(rho) if q in (8, 9) else abs(s0[q]))
        assert abs(s1[q] - s0[q]) <= tol, (q, s1[q], s0[q])


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_one_rank_nccl_group_is_the_whole_lattice_bitwise():
    import datetime

    import torch.distributed as dist

    N = 32
    st = _state(N, seed=21)
    f0, d0, s0 = _whole(N, gb.FP64, st, STEPS)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(_free_port())
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60))
    try:
        f1, d1, s1 = _slabs(N, gb.FP64, st, STEPS, gs.DistComm())
    finally:
        dist.destroy_process_group()
    np.testing.assert_array_equal(f1, f0)
    np.testing.assert_array_equal(d1, d0)
    np.testing.assert_array_equal(s1, s0)


def test_slab_rejects_sweeps_before_upload():
    s = gs.Slab(32, 0, 32)
    try:
        with pytest.raises(gb.GabeError):
            s.sweep(0)
        with pytest.raises(gb.GabeError):
            s.sweep(7)
    finally:
        s.close()


FFT_TOL = 1e-5  # relative, FP32 transforms
FFT_TOL64 = 1e-11  # relative, FP64 transforms


def _norm_rel(got, want):
    return float(np.linalg.norm(got - want) / np.linalg.norm(want))


def _gw_slabs(N, st, steps, comm, precision=gb.FP32):
    f, d, a0, ad0 = st
    with gs.SlabLattice(N, comm, precision=precision, gws=True) as lat:
        fs = [f[:, p0:p0 + n] for p0, n in lat.planes]
        ds = [d[:, p0:p0 + n] for p0, n in lat.planes]
        lat.upload(fs if len(fs) > 1 else fs[0], ds if len(ds) > 1 else ds[0], a0, ad0)
        lat.step(steps)
        sc = lat.scalars()
        out = lat.download()
        gw = lat.download_gw()
    f1 = np.concatenate([o[0] for o in out], axis=1)
    h1 = np.concatenate([g[0] for g in gw], axis=2)
    l1 = np.concatenate([g[1] for g in gw], axis=2)
    return f1, h1, l1, sc


def _gw_whole(N, st, steps, precision=gb.FP32):
    f, d, a0, ad0 = st
    with gb.Lattice(N, gws=True, precision=precision) as lat:
        lat.upload_state(f, d, a0=a0, adot0=ad0)
        lat.step(steps)
        sc = lat.scalars()
        f1, _, h1, l1 = lat.download_state()
    want = np.array([v for k in ("a", "adot", "edkin", "edpot", "edgrad", "edrho") for v in sc[k]])
    return f1, h1, l1, want


def _gw_compare(a, b):
    (f1, h1, l1, s1), (f0, h0, l0, s0) = a, b
    for fld in range(2):
        fl = f0[fld] - f0[fld].mean()
        assert np.abs(f1[fld] - f0[fld]).max() <= 1e-5 * np.abs(fl).max()
    rho = s0[10]
    for q in range(12):
        tol = 1e-6 * (abs(rho) if q in (8, 9) else abs(s0[q]))
        assert abs(s1[q] - s0[q]) <= tol, (q, s1[q], s0[q])
    assert np.linalg.norm(l0) > 0
    assert _norm_rel(h1, h0) <= FFT_TOL
    assert _norm_rel(l1, l0) <= FFT_TOL


@pytest.mark.parametrize("world", [1, 2, 3])
def test_gw_slabs_match_the_whole_lattice(world):
    N = 64
    st = _state(N, seed=25)
    _gw_compare(_gw_slabs(N, st, STEPS, gs.LocalComm(world)), _gw_whole(N, st, STEPS))


def _gw_compare64(a, b, world):
    """FP64: one slab's fields are the handle's bit for bit (GWs do not act
    on the fields; sweep A only also stores the sources); several slabs add
    the energy sums in another order (~1e-12)."""
    (f1, h1, l1, s1), (f0, h0, l0, s0) = a, b
    if world == 1:
        np.testing.assert_array_equal(f1, f0)
        np.testing.assert_array_equal(s1, s0)
    else:
        assert np.abs(f1 - f0).max() <= 1e-11 * np.abs(f0).max()
        for q in range(12):  # edgrad (8, 9) is ~1e-11 of rho here: measured against rho
            tol = 1e-11 * (abs(s0[10]) if q in (8, 9) else abs(s0[q]))
            assert abs(s1[q] - s0[q]) <= tol, (q, s1[q], s0[q])
    assert np.linalg.norm(l0) > 0
    assert _norm_rel(h1, h0) <= FFT_TOL64
    assert _norm_rel(l1, l0) <= FFT_TOL64


@pytest.mark.parametrize("N,world", [(64, 1), (64, 2), (48, 3)])
def test_fp64_gw_slabs_match_the_whole_lattice(N, world):
    st = _state(N, seed=31)
    got = _gw_slabs(N, st, STEPS, gs.LocalComm(world), precision=gb.FP64)
    _gw_compare64(got, _gw_whole(N, st, STEPS, precision=gb.FP64), world)


def test_gw_slabs_through_a_one_rank_nccl_group():
    import datetime

    import torch.distributed as dist

    N = 64
    st = _state(N, seed=27)
    want = _gw_whole(N, st, STEPS)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(_free_port())
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60))
    try:
        got = _gw_slabs(N, st, STEPS, gs.DistComm())
    finally:
        dist.destroy_process_group()
    _gw_compare(got, want)


def _cols_close(got, want, cols):
    g, w = got[:, cols], want[:, cols]
    floor = 1e-9 * np.abs(w).max(axis=0, keepdims=True)
    return float(np.max((np.abs(g - w) - floor) / np.abs(w).clip(min=1e-300)))


@pytest.mark.parametrize("world,gws,precision", [(1, True, gb.FP32), (3, True, gb.FP32), (2, False, gb.FP32),
                                                 (2, True, gb.FP64), (3, False, gb.FP64)])
def test_slab_spectra_match_the_whole_lattice(world, gws, precision):
    """specOut's table of a split lattice: each slab bins its own k-points
    after the fields' transpose; the sums over the slabs, normalised, are
    the handle's spectra to transform rounding (FP32 or FP64)."""
    N = 64
    f, d, a0, ad0 = _state(N, seed=29)
    with gb.Lattice(N, gws=gws, precision=precision) as lat:
        lat.upload_state(f, d, a0=a0, adot0=ad0)
        lat.step(STEPS)
        want = lat.spec_out()
    with gs.SlabLattice(N, gs.LocalComm(world), precision=precision, gws=gws) as sl:
        fs = [f[:, p0:p0 + n] for p0, n in sl.planes]
        ds = [d[:, p0:p0 + n] for p0, n in sl.planes]
        sl.upload(fs if len(fs) > 1 else fs[0], ds if len(ds) > 1 else ds[0], a0, ad0)
        sl.step(STEPS)
        got = sl.spectra()
    assert got.shape == want.shape
    np.testing.assert_array_equal(got[:, 0], want[:, 0])
    tol = FFT_TOL if precision == gb.FP32 else FFT_TOL64
    assert _cols_close(got, want, [1, 2, 3, 4]) <= tol
    if gws:
        assert np.abs(want[:, 5]).max() > 0
        assert _cols_close(got, want, [5, 6]) <= tol
        np.testing.assert_array_equal(got[:, 7], want[:, 7])

