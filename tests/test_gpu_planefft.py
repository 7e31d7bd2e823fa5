"""FP32 GW-source transforms: the library's plane kernels against cuFFT.

With FP32 storage, N in {64, 128, 256, 512} and GABE_FLAG_PLANE_FFT the
library transforms the ten GW source arrays with its own 2-D r2c over every
(j, k) plane (one thread-block cluster per plane, rows then columns in shared
memory) followed by a 1-D pass along i; by default it uses cuFFT's 3-D r2c
plan, the form of the reference's fft_stresstensor (g2evolutionpert.cpp:
183-195).  Both evolve the same state through the C ABI; h, l and the GW
spectrum must agree to FP32 transform rounding (the two transforms order
their sums differently).  512^3 runs the 16-CTA cluster configuration and is
compared through the spectra only, so that no 512^3 GW state crosses to the
host.
"""
import numpy as np
import pytest

import gabe_b200 as gb

pytestmark = pytest.mark.gpu

FFT_TOL = 1e-5  # relative, FP32 transforms of ~1e5..1e8 terms


def _norm_rel(got, want):
    return float(np.linalg.norm(got - want) / np.linalg.norm(want))


def _state(N, seed=7):
    from gabe_b200.ic import random_state

    f, d, a0, ad0 = random_state(N, seed=seed, device="cuda")
    return f.cpu().numpy(), d.cpu().numpy(), a0, ad0


def _gw_cols_close(got, want, tol=FFT_TOL):
    g, w = got[:, 5:7], want[:, 5:7]
    floor = 1e-9 * np.abs(w).max(axis=0, keepdims=True)
    return float(np.max((np.abs(g - w) - floor) / np.abs(w).clip(min=1e-300)))


@pytest.mark.parametrize("N", [64, 128, 256])
def test_plane_fft_matches_cufft_3d(N):
    f, d, a0, ad0 = _state(N)
    out = []
    for flags in (gb.FLAG_PLANE_FFT, 0):
        with gb.Lattice(N, gws=True, precision=gb.FP32, flags=flags) as lat:
            assert lat.launches_per_step == (4 if flags else 3)
            lat.upload_state(f, d, a0=a0, adot0=ad0)
            lat.step(3)
            out.append((lat.download_state(), lat.spec_out()))
    ((f0, d0, h0, l0), s0), ((f1, d1, h1, l1), s1) = out
    # the fields do not depend on the GW chain (no backreaction)
    np.testing.assert_array_equal(f0, f1)
    np.testing.assert_array_equal(d0, d1)
    assert np.linalg.norm(l1) > 0
    assert _norm_rel(h0, h1) <= FFT_TOL
    assert _norm_rel(l0, l1) <= FFT_TOL
    # field spectra: same fields; the binning's FP64 shared-memory sums vary in the last bit
    np.testing.assert_allclose(s0[:, :5], s1[:, :5], rtol=1e-12, atol=0)
    assert _gw_cols_close(s0, s1) <= FFT_TOL


@pytest.mark.parametrize("flags", [0, gb.FLAG_NO_OVERLAP, gb.FLAG_NO_GRAPH])
def test_plane_fft_launch_forms_agree(flags):
    """Overlapped graph, in-line and direct launches run the same kernels on
    the same data: bit-identical results."""
    N = 64
    f, d, a0, ad0 = _state(N, seed=11)
    res = []
    for fl in (gb.FLAG_PLANE_FFT, gb.FLAG_PLANE_FFT | flags):
        with gb.Lattice(N, gws=True, precision=gb.FP32, flags=fl) as lat:
            lat.upload_state(f, d, a0=a0, adot0=ad0)
            lat.step(5)
            res.append(lat.download_state())
    for a, b in zip(res[0], res[1]):
        np.testing.assert_array_equal(a, b)


def test_plane_fft_512_cluster16_matches_cufft_3d():
    N = 512
    f, d, a0, ad0 = _state(N, seed=3)
    specs = []
    for flags in (gb.FLAG_PLANE_FFT, 0):
        with gb.Lattice(N, gws=True, precision=gb.FP32, flags=flags) as lat:
            lat.upload_state(f, d, a0=a0, adot0=ad0)
            lat.step(2)
            specs.append(lat.spec_out())
    assert np.all(np.isfinite(specs[0]))
    assert np.abs(specs[1][:, 5]).max() > 0
    assert _gw_cols_close(specs[0], specs[1]) <= FFT_TOL
