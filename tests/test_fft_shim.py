"""The FFTW-API stand-in (oracle/fftw_shim) against numpy's pocketfft, on the
FFTW conventions the reference relies on: unnormalised, forward
exp(-i...), r2c half layout, c2r ignoring the imaginary parts of the
self-conjugate entries."""
import ctypes

import numpy as np
import pytest

from oracle import pyoracle as po

P = ctypes.c_void_p


def _plan(kind, n, a, b):
    L = po.lib()
    f = L.fftw_plan_dft_r2c_3d if kind == "r2c" else L.fftw_plan_dft_c2r_3d
    f.restype = ctypes.c_void_p
    f.argtypes = [ctypes.c_int] * 3 + [P, P, ctypes.c_uint]
    return f(*n, a.ctypes.data_as(P), b.ctypes.data_as(P), 0)


def _exec(p):
    L = po.lib()
    L.fftw_execute.argtypes = [P]
    L.fftw_destroy_plan.argtypes = [P]
    L.fftw_execute(P(p))
    L.fftw_destroy_plan(P(p))


@pytest.mark.parametrize("n", [(8, 8, 8), (16, 12, 10), (6, 10, 9), (48, 32, 64), (7, 5, 3), (2, 4, 4)])
def test_r2c_and_c2r(n):
    rng = np.random.default_rng(1)
    x = rng.standard_normal(n)
    out = np.zeros((n[0], n[1], n[2] // 2 + 1), complex)
    _exec(_plan("r2c", n, x, out))
    ref = np.fft.rfftn(x)
    assert np.abs(out - ref).max() <= 1e-13 * np.abs(ref).max()
    z = rng.standard_normal(out.shape) + 1j * rng.standard_normal(out.shape)
    y = np.zeros(n)
    zz = z.copy()
    _exec(_plan("c2r", n, zz, y))
    r2 = np.fft.irfftn(z, s=n, axes=(0, 1, 2)) * np.prod(n)
    assert np.abs(y - r2).max() <= 1e-13 * np.abs(r2).max()


def test_threads_do_not_change_results():
    x = np.random.default_rng(2).standard_normal((32, 32, 32))
    outs = []
    for t in (1, 4):
        po.lib().fftw_plan_with_nthreads(t)
        o = np.zeros((32, 32, 17), complex)
        _exec(_plan("r2c", (32, 32, 32), x, o))
        outs.append(o)
    po.lib().fftw_plan_with_nthreads(1)
    np.testing.assert_array_equal(outs[0], outs[1])
