"""gabe_spectra_from_sums -- specOut's normalisation (g2spectra.cpp:27,
94-103,114-117,186-195), shared by gabe_spectra and the slab spectra --
against the oracle's spectra table, on the CPU: binned sums and counts of
an oracle state formed here with numpy (native bin (int)|n|, weight 2 for
0 < kz < N/2; sum_ij |l_ij|^2 with off-diagonal weight 2, the kz = 0 plane
read at kz = N/2 as the reference's loop leaves it) go through the C
function and must give the oracle's table."""
import ctypes

import numpy as np
import pytest

import gabe_b200 as gb
from oracle import pyoracle as po

_dp = ctypes.POINTER(ctypes.c_double)


def _lib():
    lib = gb.library()
    lib.gabe_spectra_from_sums.argtypes = [ctypes.POINTER(gb.Params), ctypes.c_double, _dp, _dp, ctypes.c_int, _dp,
                                           ctypes.c_int]
    return lib


def _raw(cfg, field0, l0):
    N = cfg.N
    nz = N // 2 + 1
    nb = po.numbins(N)
    i = np.arange(N)
    p = np.where(i <= N // 2, i, i - N)
    kz = np.arange(nz)
    n2 = p[:, None, None] ** 2 + p[None, :, None] ** 2 + kz[None, None, :] ** 2
    b = np.sqrt(n2.astype(np.float64)).astype(np.int64)
    w = np.where((kz == 0) | (kz == N // 2), 1.0, 2.0)[None, None, :] * np.ones((N, N, 1))
    ns = 2 + (1 if l0 is not None else 0)
    sums = np.zeros((ns, nb))
    for f in range(2):
        F = np.fft.rfftn(field0[f])
        sums[f] = np.bincount(b.ravel(), (w * np.abs(F) ** 2).ravel(), minlength=nb)[:nb]
    if l0 is not None:
        lq = l0.copy()
        lq[:, :, :, 0] = l0[:, :, :, N // 2]  # the reference's kz = 0 quirk
        cw = np.array([1, 2, 2, 1, 2, 1], dtype=np.float64)
        p2 = sum(cw[c] * (lq[2 * c] ** 2 + lq[2 * c + 1] ** 2) for c in range(6))
        sums[2] = np.bincount(b.ravel(), (w * p2).ravel(), minlength=nb)[:nb]
    cnt = np.bincount(b.ravel(), w.ravel(), minlength=nb)[:nb]
    return sums, cnt


@pytest.mark.parametrize("gws", [0, 1])
def test_spectra_from_sums_reproduces_the_oracle_table(gws):
    cfg = po.Config(N=16, model=po.MODEL_LPHI4, gws=gws)
    st = po.init_state(cfg, seed=3)
    po.step(st, 5)
    l0 = st.l[0] if gws else None
    want = po.spectra(cfg, st.field[0], l0, st.sc.edrho[0])
    sums, cnt = _raw(cfg, st.field[0], l0)
    lib = _lib()
    p = gb.Params()
    lib.gabe_default_params(ctypes.byref(p), cfg.N)
    p.L, p.gws_on = cfg.L, gws
    nb, ncol = want.shape
    out = np.zeros((nb, ncol))
    sums = np.ascontiguousarray(sums)
    rc = lib.gabe_spectra_from_sums(ctypes.byref(p), float(st.sc.edrho[0]), sums.ctypes.data_as(_dp),
                                    np.ascontiguousarray(cnt).ctypes.data_as(_dp), nb, out.ctypes.data_as(_dp), ncol)
    assert rc == 0
    np.testing.assert_array_equal(out[:, 0], want[:, 0])
    np.testing.assert_allclose(out, want, rtol=1e-9, atol=1e-300)


def test_spectra_from_sums_rejects_a_wrong_table_shape():
    lib = _lib()
    p = gb.Params()
    lib.gabe_default_params(ctypes.byref(p), 16)
    nb = po.numbins(16)
    buf = np.zeros(8 * nb)
    assert lib.gabe_spectra_from_sums(ctypes.byref(p), 1.0, buf.ctypes.data_as(_dp), buf.ctypes.data_as(_dp), nb,
                                      buf.ctypes.data_as(_dp), 8) != 0  # GWs off: 5 columns
