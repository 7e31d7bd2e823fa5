"""Parity of the CUDA path (through the C ABI) with the oracle.

The oracle (oracle/gabe_oracle.c) reproduces the reference build bit for
bit (tests/test_oracle_golden.py); here the GPU library evolves the same
initial states and is compared with it:

  FP64  fields and momenta pointwise to <= 1e-10 relative (the GPU keeps the
        reference's operation order; only the order of the energy sums
        differs), scalars to <= 1e-12.
        h and l: <= 1e-12 in norm after the first step, whose GW sources are
        bit-identical on both sides (cuFFT vs the oracle's FFT differ at
        rounding level); <= 1e-8 later.  The reference forms the source
        gradients from full field values (phi ~ 0.3 + 1e-7 fluctuations), so
        a last-bit difference in phi -- which the different summation order
        of adot eventually produces -- is a ~1e-9 relative change of the
        source; the reference carries the same noise.
        Spectra: <= 1e-8 per bin for the fields (their FFT includes the large
        k=0 mode, whose rounding sets the floor for weak bins), <= 1e-6 for
        the GW columns.
  FP32  energies, a(t) and spectra against the FP64 path (<= 1e-4 energy).
"""
import math
import os

import numpy as np
import pytest

import gabe_b200 as gb
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def _lattice(cfg: po.Config, precision=gb.FP64, **kw):
    c0, c1, *_ = po.model_constants(cfg.model)
    return gb.Lattice(cfg.N, L=cfg.L, dt=cfg.dt, gws=bool(cfg.gws), model=cfg.model, model_c=(c0, c1),
                      precision=precision, gw_spec_quirk=bool(cfg.gw_spec_quirk), **kw)


def _upload(lat: gb.Lattice, st: po.State):
    lat.upload_state(st.field[0], st.dfield[0], st.h[0] if st.cfg.gws else None,
                     st.l[0] if st.cfg.gws else None, a0=st.sc.a[0], adot0=st.sc.adot[0])


def _pointwise_rel(got, want):
    """max over points of |got-want| / (|want| + rms(want))."""
    scale = np.abs(want) + np.sqrt(np.mean(want * want))
    return float(np.max(np.abs(got - want) / scale))


def _norm_rel(got, want):
    n = np.linalg.norm(want)
    return float(np.linalg.norm(got - want) / n) if n > 0 else float(np.abs(got).max())


def _scalar_tol(name, want, rho):
    """1e-12 relative; the gradient energy is the reference's sum of
    -f lap f over N^3 sites whose terms cancel (the mean field has zero
    Laplacian but is ~0.3), so its summation-order noise is bounded
    relative to rho, the quantity adot is formed from."""
    if name in ("grad", "edgrad"):
        return 1e-12 * abs(rho)
    return 1e-12 * abs(want)


def _spectra_close(got, want):
    """Per bin rtol, plus a floor set by the largest value of each column
    (FFT rounding is relative to the largest mode, so nearly empty bins such
    as chi's k=0 bin carry absolute, not relative, noise)."""
    for cols, rtol, floor in ((slice(0, 5), 1e-8, 1e-12), (slice(5, None), 1e-6, 1e-10)):
        g, w = got[:, cols], want[:, cols]
        if w.size == 0:
            continue
        tol = rtol * np.abs(w) + floor * np.abs(w).max(axis=0, keepdims=True)
        assert np.all(np.abs(g - w) <= tol), np.max(np.abs(g - w) / np.maximum(tol, 1e-300))


CASES = [
    # model, N, gws, steps
    (po.MODEL_LPHI4, 16, 1, 50),
    (po.MODEL_QUADRATIC, 32, 1, 20),
    (po.MODEL_LPHI4, 32, 0, 200),
    (po.MODEL_LPHI4, 48, 1, 10),
    (po.MODEL_LPHI4, 8, 1, 30),
    (po.MODEL_LPHI4, 64, 0, 200),
]


@pytest.mark.parametrize("model,N,gws,steps", CASES)
def test_fp64_matches_oracle(model, N, gws, steps):
    cfg = po.Config(N=N, model=model, gws=gws)
    st = po.init_state(cfg)
    with _lattice(cfg) as lat:
        _upload(lat, st)
        e0 = lat.calc_energy()
        for k in ("kin", "pot", "grad", "rho"):
            want = {"kin": st.sc.edkin[0], "pot": st.sc.edpot[0], "grad": st.sc.edgrad[0], "rho": st.sc.edrho[0]}[k]
            assert abs(e0[k] - want) <= _scalar_tol(k, want, st.sc.edrho[0]), (k, e0[k], want)
        done = 0
        for chunk in (1, steps - 1):
            lat.step(chunk)
            po.step(st, chunk)
            done += chunk
            f, d, h, l = lat.download_state()
            assert _pointwise_rel(f, st.field[0]) <= 1e-10, done
            assert _pointwise_rel(d, st.dfield[0]) <= 1e-10, done
            if gws:
                tol = 1e-12 if done == 1 else 1e-8
                assert _norm_rel(h, st.h[0]) <= tol, done
                assert _norm_rel(l, st.l[0]) <= tol, done
            sc = lat.scalars()
            for k in ("a", "adot", "edkin", "edpot", "edgrad", "edrho"):
                for s in (0, 1):
                    want = getattr(st.sc, k)[s]
                    assert abs(sc[k][s] - want) <= _scalar_tol(k, want, st.sc.edrho[s]), (k, s, sc[k][s], want)


@pytest.mark.parametrize("expansion,gws", [(0, 0), (0, 1), (2, 1)])
def test_expansion_types_match_oracle(expansion, gws):
    """expansion_type 0 (a, adot fixed, no tensor modes, only calcEnergy(0)
    per step, g2functions.cpp:207-232) and 2 (type 1 without tensor modes,
    :272-302): FP64 pointwise against the oracle, which reproduces the
    reference builds of both types bit for bit (tests/test_oracle_golden.py);
    FP32 energies against FP64."""
    N, steps = 32, 100
    cfg = po.Config(N=N, model=po.MODEL_LPHI4, gws=gws, expansion=expansion)
    st = po.init_state(cfg)
    first = st.copy()
    with _lattice(cfg, expansion=expansion) as lat, _lattice(cfg, precision=gb.FP32, expansion=expansion) as l32:
        _upload(lat, st)
        _upload(l32, st)
        lat.step(steps)
        l32.step(steps)
        po.step(st, steps)
        f, d, h, l = lat.download_state()
        assert _pointwise_rel(f, st.field[0]) <= 1e-10
        assert _pointwise_rel(d, st.dfield[0]) <= 1e-10
        if gws:  # tensor modes are not evolved: they keep their initial (zero) values
            assert np.abs(h).max() == 0 and np.abs(l).max() == 0
        sc = lat.scalars()
        for k in ("a", "adot", "edkin", "edpot", "edgrad", "edrho"):
            for s in (0, 1):
                want = getattr(st.sc, k)[s]
                assert abs(sc[k][s] - want) <= _scalar_tol(k, want, st.sc.edrho[s]), (k, s, sc[k][s], want)
        if expansion == 0:
            assert sc["a"] == (first.sc.a[0], first.sc.a[0]) and sc["adot"] == (0.0, 0.0)
        e64, e32 = lat.calc_energy(), l32.calc_energy()
        for k in ("kin", "pot", "rho", "a", "adot"):
            assert abs(e32[k] - e64[k]) <= 1e-4 * abs(e64[k]) + (1e-300 if k == "adot" else 0), (k, e32[k], e64[k])


def test_fp64_from_reference_dump():
    """Start from the state the reference itself wrote after 10 steps."""
    d = np.load(os.path.join(HERE, "golden", "ref_m1_n16_g1_step10.npz"))
    cfg = po.Config(N=16, model=po.MODEL_LPHI4, gws=1)
    st = po.State.empty(cfg)
    st.field[0], st.dfield[0], st.h[0], st.l[0] = d["field"], d["dfield"], d["h"], d["l"]
    for q, k in enumerate(("a", "adot", "edkin", "edpot", "edgrad", "edrho")):
        getattr(st.sc, k)[0], getattr(st.sc, k)[1] = d["scalars"][q]
    with _lattice(cfg) as lat:
        _upload(lat, st)
        lat.step(40)
        po.step(st, 40)
        f, dd, h, l = lat.download_state()
        assert _pointwise_rel(f, st.field[0]) <= 1e-10
        assert _pointwise_rel(dd, st.dfield[0]) <= 1e-10
        assert _norm_rel(l, st.l[0]) <= 1e-8


@pytest.mark.parametrize("gws", [0, 1])
def test_fp64_spectra_match_oracle(gws):
    cfg = po.Config(N=32, model=po.MODEL_LPHI4, gws=gws)
    st = po.init_state(cfg)
    with _lattice(cfg) as lat:
        _upload(lat, st)
        lat.step(25)
        po.step(st, 25)
        got = lat.spec_out()
        want = po.spectra(cfg, st.field[0], st.l[0] if gws else None, st.sc.edrho[0])
        assert got.shape == want.shape
        _spectra_close(got, want)


def test_gw_spectrum_quirk_switch():
    cfg = po.Config(N=16, model=po.MODEL_LPHI4, gws=1, gw_spec_quirk=0)
    st = po.init_state(cfg)
    with _lattice(cfg) as lat:
        _upload(lat, st)
        lat.step(10)
        po.step(st, 10)
        got = lat.spec_out()
        want = po.spectra(cfg, st.field[0], st.l[0], st.sc.edrho[0])
        _spectra_close(got, want)


def test_config1_64cubed_1000_steps():
    """64^3, L=20, dt=0.01, GWs off, 1000 steps: pointwise to 200 steps, then
    a(t), energies and binned spectra within 1%."""
    cfg = po.Config(N=64, model=po.MODEL_LPHI4, gws=0)
    st = po.init_state(cfg)
    with _lattice(cfg) as lat:
        _upload(lat, st)
        lat.step(200)
        po.step(st, 200)
        f, d, _, _ = lat.download_state()
        assert _pointwise_rel(f, st.field[0]) <= 1e-10
        lat.step(800)
        po.step(st, 800)
        sc = lat.scalars()
        for k in ("a", "adot", "edkin", "edpot", "edgrad", "edrho"):
            assert abs(sc[k][0] - getattr(st.sc, k)[0]) <= 1e-2 * abs(getattr(st.sc, k)[0]), k
        got = lat.spec_out()
        want = po.spectra(cfg, st.field[0], None, st.sc.edrho[0])
        nz = want[:, 1:] != 0
        assert np.max(np.abs(got[:, 1:][nz] - want[:, 1:][nz]) / np.abs(want[:, 1:][nz])) <= 1e-2


def test_graph_and_direct_launches_agree():
    cfg = po.Config(N=32, model=po.MODEL_LPHI4, gws=1)
    st = po.init_state(cfg)
    out = []
    for flags in (0, gb.FLAG_NO_GRAPH):
        with _lattice(cfg, flags=flags) as lat:
            _upload(lat, st)
            lat.step(7)
            out.append(lat.download_state())
    for a, b in zip(out[0], out[1]):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("precision", [gb.FP64, gb.FP32])
def test_tile_shapes_and_chunks_agree(precision):
    cfg = po.Config(N=32, model=po.MODEL_LPHI4, gws=1)
    st = po.init_state(cfg)
    res = []
    for shape, ci in ((-1, 0), (2, 3), (3, 32), (1, 5)):
        with _lattice(cfg, precision=precision, tile_shape=shape, tile_ci=ci) as lat:
            _upload(lat, st)
            lat.step(5)
            res.append(lat.download_state())
    tol = 1e-14 if precision == gb.FP64 else 1e-6
    for r in res[1:]:
        for a, b in zip(res[0], r):
            assert _norm_rel(b, a) <= tol


def test_runs_are_deterministic():
    cfg = po.Config(N=32, model=po.MODEL_LPHI4, gws=1)
    st = po.init_state(cfg)
    out = []
    for _ in range(2):
        with _lattice(cfg) as lat:
            _upload(lat, st)
            lat.step(6)
            out.append((lat.download_state(), lat.scalars()))
    for a, b in zip(out[0][0], out[1][0]):
        np.testing.assert_array_equal(a, b)
    assert out[0][1] == out[1][1]


@pytest.mark.parametrize("N,gws,flags", [(32, 0, 0), (32, 1, 0), (64, 1, 0), (64, 1, gb.FLAG_OWN_FFT),
                                         (64, 1, gb.FLAG_TRANSPOSED_FFT)])
def test_fp32_against_fp64(N, gws, flags):
    """FP32 storage of fluctuations vs the FP64 path: energies <= 1e-4.  The
    FP32 GW sources go through cuFFT's 3-D plan, or the library's three-pass
    3-D FFT (GABE_FLAG_OWN_FFT), and the separate k-space pass, or through the
    transposed passes with the pass along i fused into the k-space update
    (GABE_FLAG_TRANSPOSED_FFT)."""
    steps = 200
    cfg = po.Config(N=N, model=po.MODEL_LPHI4, gws=gws)
    st = po.init_state(cfg)
    with _lattice(cfg, precision=gb.FP64) as l64, _lattice(cfg, precision=gb.FP32, flags=flags) as l32:
        _upload(l64, st)
        _upload(l32, st)
        e64, e32 = l64.calc_energy(), l32.calc_energy()
        for k in ("kin", "pot", "rho"):
            assert abs(e32[k] - e64[k]) <= 1e-6 * abs(e64[k]), (k, e32[k], e64[k])
        # the FP64 (reference) form of the gradient energy sums f lap f with
        # f ~ 0.34 + 1e-7: ~1e-5 relative rounding noise at the initial state
        assert abs(e32["grad"] - e64["grad"]) <= 1e-4 * abs(e64["grad"])
        l64.step(steps)
        l32.step(steps)
        e64, e32 = l64.calc_energy(), l32.calc_energy()
        for k in ("kin", "pot", "rho", "a", "adot"):
            assert abs(e32[k] - e64[k]) <= 1e-4 * abs(e64[k]), (k, e32[k], e64[k])
        assert abs(e32["grad"] - e64["grad"]) <= 1e-4 * abs(e64["grad"]) + 1e-6 * e64["rho"]
        f64, d64, h64, ll64 = l64.download_state()
        f32, d32, h32, ll32 = l32.download_state()
        for q in range(2):
            fl = f64[q] - f64[q].mean()
            assert np.abs((f32[q] - f32[q].mean()) - fl).max() <= 1e-3 * np.abs(fl).max()
        s64, s32 = l64.spec_out(), l32.spec_out()
        # per-bin spectrum error <= 1e-4 relative, above the FFT noise floor
        # of each column (chi's k=0 bin holds only rounding noise)
        w, g = s64[:, 1:5], s32[:, 1:5]
        floor = 1e-9 * np.abs(w).max(axis=0, keepdims=True)
        assert np.all(np.abs(g - w) <= 1e-4 * np.abs(w) + floor)
        if gws:
            assert _norm_rel(ll32, ll64) <= 1e-3


def test_upload_download_roundtrip():
    """h and l are kept as two TT polarization amplitudes; TT data (any state
    the evolution produced) round-trips, non-TT data is refused."""
    cfg = po.Config(N=16, model=po.MODEL_LPHI4, gws=1)
    st = po.init_state(cfg)
    po.step(st, 6)
    for prec, tol in ((gb.FP64, 1e-14), (gb.FP32, 1e-6)):
        with _lattice(cfg, precision=prec) as lat:
            _upload(lat, st)
            f, d, h, l = lat.download_state()
            if prec == gb.FP64:
                np.testing.assert_array_equal(f, st.field[0])
                np.testing.assert_array_equal(d, st.dfield[0])
            else:
                for q in range(2):
                    fl = st.field[0, q] - st.field[0, q].mean()
                    assert np.abs(f[q] - st.field[0, q]).max() <= 1e-6 * np.abs(fl).max() + 1e-15
            assert _norm_rel(h, st.h[0]) <= tol and _norm_rel(l, st.l[0]) <= tol
    bad = st.copy()
    bad.l[0] = np.random.default_rng(0).standard_normal(bad.l[0].shape) * 1e-9
    with _lattice(cfg) as lat:
        with pytest.raises(gb.GabeError) as ei:
            _upload(lat, bad)
        assert ei.value.code == 1


def test_refused_upload_leaves_the_handle_without_a_state():
    """A re-upload that is refused after it began to overwrite the device
    state (non-TT l: the fields are already in place when the amplitudes are
    checked) must not leave a half-new state to step on: steps report
    GABE_ERR_STATE until an upload succeeds, and the handle then runs as a
    fresh one does."""
    cfg = po.Config(N=16, model=po.MODEL_LPHI4, gws=1)
    st = po.init_state(cfg)
    po.step(st, 6)
    bad = st.copy()
    bad.l[0] = np.random.default_rng(1).standard_normal(bad.l[0].shape) * 1e-9
    with _lattice(cfg) as lat, _lattice(cfg) as ref:
        _upload(lat, st)
        lat.step(2)
        with pytest.raises(gb.GabeError) as ei:
            _upload(lat, bad)
        assert ei.value.code == 1
        with pytest.raises(gb.GabeError) as ei:
            lat.step(1)
        assert ei.value.code == 7
        _upload(lat, st)
        _upload(ref, st)
        lat.step(3)
        ref.step(3)
        for got, want in zip(lat.download_state(), ref.download_state()):
            np.testing.assert_array_equal(got, want)


def test_nonfinite_state_is_reported():
    cfg = po.Config(N=16, model=po.MODEL_LPHI4, gws=0)
    st = po.init_state(cfg)
    st.field[0, 1, 3, 4, 5] = np.nan
    with _lattice(cfg) as lat:
        with pytest.raises(gb.GabeError) as ei:
            _upload(lat, st)
        assert ei.value.code == 5


def test_blowup_during_steps_is_reported():
    # an absurd time step makes the stencil diverge within a few steps
    cfg = po.Config(N=16, model=po.MODEL_LPHI4, gws=0, dt=5.0)
    st = po.init_state(cfg)
    with _lattice(cfg) as lat:
        _upload(lat, st)
        lat.step(400)
        with pytest.raises(gb.GabeError) as ei:
            lat.sync()
        assert ei.value.code == 5


def test_step_before_upload_is_an_error():
    cfg = po.Config(N=16)
    with _lattice(cfg) as lat:
        with pytest.raises(gb.GabeError) as ei:
            lat.step(1)
        assert ei.value.code == 7


def _variance_tol(var, av, N):
    """Variance sum(f^2 - mean^2)/N^3 of a field with mean ~0.34 and ~1e-7
    fluctuations: absolute rounding noise ~ eps mean^2 sqrt(N^3) (both sides
    form it this way, with different summation orders)."""
    return 1e-6 * abs(var) + 16 * np.finfo(float).eps * av * av * N ** 1.5


@pytest.mark.parametrize("precision", [gb.FP64, gb.FP32])
def test_meansvars_and_field_slice_match_oracle(precision):
    """gabe_meansvars and gabe_field_slice (meansvars and the outputfield rows
    with calcrho, g2output.cpp:25-121, g2functions.cpp:70-122,176-186)
    against the oracle's restatements, which tests/test_oracle_output.py pins
    to the reference program's own files."""
    cfg = po.Config(N=32, model=po.MODEL_LPHI4, gws=1)
    st = po.init_state(cfg)
    po.step(st, 20)
    with _lattice(cfg, precision=precision) as lat:
        _upload(lat, st)
        mv = lat.meansvars()
        slices = {(d, sk): lat.field_slice(d, sk) for d, sk in ((1, 1), (2, 2), (3, 3))}
    want_mv = po.meansvars(st.field[0])
    for q in range(2):
        av, var = want_mv[q]
        rms = float(np.sqrt(np.mean(st.field[0, q] ** 2)))
        tol = 1e-13 * abs(av) + 16 * np.finfo(float).eps * rms
        if precision == gb.FP32:  # fluctuations stored in FP32: ~eps32 rms(fluctuation) in the mean
            tol += np.finfo(np.float32).eps * float(np.std(st.field[0, q]))
        assert abs(mv[q, 0] - av) <= tol, (q, mv[q, 0], av)
        assert abs(mv[q, 1] - var) <= _variance_tol(var, av, cfg.N), (q, mv[q, 1], var)
    for (d, sk), got in slices.items():
        want = po.field_slice(cfg, st.field[0], st.dfield[0], st.sc.a[0], d, sk)
        assert got.shape == want.shape == (((cfg.N + sk - 1) // sk) ** d, 3)
        if precision == gb.FP64:
            np.testing.assert_array_equal(got[:, :2], want[:, :2])
            assert np.all(np.abs(got[:, 2] - want[:, 2]) <= 1e-13 * np.abs(want[:, 2]))
        else:  # FP32 fluctuations about the FP64 homogeneous values
            assert np.all(np.abs(got[:, :2] - want[:, :2]) <= 1e-12 * np.abs(want[:, :2]).max())
            assert np.all(np.abs(got[:, 2] - want[:, 2]) <= 1e-6 * np.abs(want[:, 2]))


def test_field_slice_rejects_bad_arguments():
    import ctypes

    cfg = po.Config(N=16, model=po.MODEL_LPHI4, gws=0)
    st = po.init_state(cfg)
    lib = gb.library()
    with _lattice(cfg) as lat:
        _upload(lat, st)
        buf = np.zeros(3 * 64)
        ptr = buf.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        assert lib.gabe_field_slice(lat.handle, 0, 1, ptr, buf.size) == 1
        assert lib.gabe_field_slice(lat.handle, 2, 0, ptr, buf.size) == 1
        assert lib.gabe_field_slice(lat.handle, 2, 1, ptr, buf.size) == 1  # 256 rows do not fit
        assert lib.gabe_field_slice(lat.handle, 2, 2, ptr, buf.size) == 0
