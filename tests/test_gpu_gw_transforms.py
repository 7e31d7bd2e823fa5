"""FP32 GW-source transforms and the fused k-space update against cuFFT's 3-D
plan with the separate k-space pass.

The reference form of the comparisons below keeps the reference's structure
-- one 3-D r2c per source array (fft_stresstensor, g2evolutionpert.cpp:183-
195, here cuFFT's 3-D plan: the default below N = 512, GABE_FLAG_CUFFT_3D at
512) and a separate k-space pass (TT projection + both RK2 stages of h, l).
With FP32 storage and N in {64, 128, 256, 512}: GABE_FLAG_OWN_FFT does the
3-D r2c with the library's own three-pass FFT; GABE_FLAG_TRANSPOSED_FFT runs
the transposed three passes (fftt.cuh), the last one fused with the k-space
update and the amplitudes kept transposed.  All forms evolve the same state
through the C ABI; h, l and the GW spectrum must agree to FP32 transform
rounding (the forms order their sums differently), the fields bit for bit
(they do not depend on the GW chain).  512^3 is compared through the spectra
only, so that no 512^3 GW state crosses to the host.
"""
import numpy as np
import pytest

import gabe_b200 as gb

pytestmark = pytest.mark.gpu

FFT_TOL = 1e-5  # relative, FP32 transforms of ~1e5..1e8 terms
FORMS = {"own": gb.FLAG_OWN_FFT, "trans": gb.FLAG_TRANSPOSED_FFT}
LAUNCHES = {gb.FLAG_OWN_FFT: 6, gb.FLAG_TRANSPOSED_FFT: 5, gb.FLAG_CUFFT_3D: 3, 0: 3}


def _norm_rel(got, want):
    return float(np.linalg.norm(got - want) / np.linalg.norm(want))


def _state(N, seed=7):
    from gabe_b200.ic import random_state

    f, d, a0, ad0 = random_state(N, seed=seed, device="cuda")
    return f.cpu().numpy(), d.cpu().numpy(), a0, ad0


def _gw_cols_close(got, want):
    g, w = got[:, 5:7], want[:, 5:7]
    floor = 1e-9 * np.abs(w).max(axis=0, keepdims=True)
    return float(np.max((np.abs(g - w) - floor) / np.abs(w).clip(min=1e-300)))


def _run(N, flags, state, steps):
    f, d, a0, ad0 = state
    with gb.Lattice(N, gws=True, precision=gb.FP32, flags=flags) as lat:
        assert lat.launches_per_step == LAUNCHES[flags & ~(gb.FLAG_NO_OVERLAP | gb.FLAG_NO_GRAPH)]
        lat.upload_state(f, d, a0=a0, adot0=ad0)
        lat.step(steps)
        return lat.download_state(), lat.spec_out()


@pytest.mark.parametrize("form", sorted(FORMS))
@pytest.mark.parametrize("N", [64, 128, 256])
def test_gw_transform_forms_match_cufft_3d(N, form):
    st = _state(N)
    (f0, d0, h0, l0), s0 = _run(N, FORMS[form], st, 3)
    (f1, d1, h1, l1), s1 = _run(N, gb.FLAG_CUFFT_3D, st, 3)
    np.testing.assert_array_equal(f0, f1)
    np.testing.assert_array_equal(d0, d1)
    spec_rtol = 1e-12  # same fields; the binning's FP64 shared-memory sums vary in the last bit
    assert np.linalg.norm(l1) > 0
    assert _norm_rel(h0, h1) <= FFT_TOL
    assert _norm_rel(l0, l1) <= FFT_TOL
    np.testing.assert_allclose(s0[:, :5], s1[:, :5], rtol=spec_rtol, atol=0)
    assert _gw_cols_close(s0, s1) <= FFT_TOL


@pytest.mark.parametrize("flags", [gb.FLAG_NO_OVERLAP, gb.FLAG_NO_GRAPH])
@pytest.mark.parametrize("form", sorted(FORMS))
def test_gw_transform_launch_forms_agree(form, flags):
    """Overlapped graph, in-line and direct launches run the same kernels on
    the same data: bit-identical results."""
    N = 64
    st = _state(N, seed=11)
    a = _run(N, FORMS[form], st, 5)[0]
    b = _run(N, FORMS[form] | flags, st, 5)[0]
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)


@pytest.mark.parametrize("N,form", [(64, 0), (128, gb.FLAG_TRANSPOSED_FFT), (256, gb.FLAG_TRANSPOSED_FFT),
                                    (512, gb.FLAG_TRANSPOSED_FFT)])
def test_default_gw_transform_form(N, form):
    """FP32 with GWs defaults to the transposed form at N >= 128 (measured
    fastest there) and to cuFFT's plan at 64; GABE_FLAG_CUFFT_3D forces
    cuFFT's plan."""
    with gb.Lattice(N, gws=True, precision=gb.FP32) as lat:
        assert lat.launches_per_step == LAUNCHES[form]
    with gb.Lattice(N, gws=True, precision=gb.FP32, flags=gb.FLAG_CUFFT_3D) as lat:
        assert lat.launches_per_step == LAUNCHES[gb.FLAG_CUFFT_3D]


def test_gw_transforms_512_match_cufft_3d():
    N = 512
    f, d, a0, ad0 = _state(N, seed=3)
    specs = {}
    for name, flags in [*FORMS.items(), ("3d", gb.FLAG_CUFFT_3D), ("default", 0)]:
        with gb.Lattice(N, gws=True, precision=gb.FP32, flags=flags) as lat:
            if name == "default":
                assert lat.launches_per_step == LAUNCHES[gb.FLAG_TRANSPOSED_FFT]  # the transposed form at 512
            lat.upload_state(f, d, a0=a0, adot0=ad0)
            lat.step(2)
            specs[name] = lat.spec_out()
    assert np.abs(specs["3d"][:, 5]).max() > 0
    # same kernels; the binning's FP64 shared-memory sums vary in the last bit
    np.testing.assert_allclose(specs["default"], specs["trans"], rtol=1e-12, atol=0)
    for name in FORMS:
        assert np.all(np.isfinite(specs[name]))
        assert _gw_cols_close(specs[name], specs["3d"]) <= FFT_TOL, name


def test_transposed_form_keeps_an_uploaded_gw_state():
    """The transposed form stores the amplitudes as [4][kz][ky][kx]: an
    uploaded TT state (the oracle's, after a few steps with GWs) must
    download unchanged, and stepping it must match cuFFT's form."""
    from oracle import pyoracle as po

    cfg = po.Config(N=64, model=po.MODEL_LPHI4, gws=1)
    st = po.init_state(cfg)
    po.step(st, 4)
    c0, c1, *_ = po.model_constants(cfg.model)
    out = {}
    for name, flags in (("trans", gb.FLAG_TRANSPOSED_FFT), ("3d", gb.FLAG_CUFFT_3D)):
        with gb.Lattice(cfg.N, L=cfg.L, dt=cfg.dt, gws=True, model=cfg.model, model_c=(c0, c1),
                        precision=gb.FP32, flags=flags) as lat:
            lat.upload_state(st.field[0], st.dfield[0], st.h[0], st.l[0], a0=st.sc.a[0], adot0=st.sc.adot[0])
            _, _, h, l = lat.download_state()
            assert _norm_rel(h, st.h[0]) <= 1e-6 and _norm_rel(l, st.l[0]) <= 1e-6
            lat.step(3)
            out[name] = (lat.download_state(), lat.spec_out())
    (f0, d0, h0, l0), s0 = out["trans"]
    (f1, d1, h1, l1), s1 = out["3d"]
    np.testing.assert_array_equal(f0, f1)
    assert _norm_rel(h0, h1) <= FFT_TOL and _norm_rel(l0, l1) <= FFT_TOL
    assert _gw_cols_close(s0, s1) <= FFT_TOL
