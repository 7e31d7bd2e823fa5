"""Checkpoint / restart through the C ABI (gabe_save_state, gabe_load_state).

A run of K steps is saved, the file is loaded into a new handle with the
same parameters, and both continue for M steps: the restarted run must equal
the uninterrupted one bit for bit -- fields, momenta, h, l and all twelve
scalars; the spectra to the last-bit noise of their binning -- in FP64 and
in FP32 storage (cuFFT's plan, the
library's three-pass FFT and the transposed form, whose amplitudes are kept
in another order).  The file's portable part holds the FP64 state at step K
in the reference's layout.  A dump without a restart block (as the
reference harness writes) is uploaded as an initial state instead."""
import numpy as np
import pytest

import gabe_b200 as gb
from gabe_b200 import checkpoint as ck
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


def _lat(cfg, precision, flags):
    c0, c1, *_ = po.model_constants(cfg.model)
    return gb.Lattice(cfg.N, L=cfg.L, dt=cfg.dt, gws=bool(cfg.gws), model=cfg.model, model_c=(c0, c1),
                      precision=precision, flags=flags)


def _snapshot(lat):
    f, d, h, l = lat.download_state()
    sc = lat.scalars()
    return [f, d, h, l, np.array([sc[k] for k in sorted(sc)]), lat.spec_out()]


@pytest.mark.parametrize("precision,flags,N", [(gb.FP64, 0, 32), (gb.FP32, 0, 64), (gb.FP32, gb.FLAG_OWN_FFT, 64),
                                               (gb.FP32, gb.FLAG_TRANSPOSED_FFT, 64)])
def test_restart_continues_bit_for_bit(tmp_path, precision, flags, N):
    cfg = po.Config(N=N, model=po.MODEL_LPHI4, gws=1)
    st = po.init_state(cfg)
    path = str(tmp_path / "ckpt.bin")
    K, M = 7, 6
    with _lat(cfg, precision, flags) as a:
        a.upload_state(st.field[0], st.dfield[0], st.h[0], st.l[0], a0=st.sc.a[0], adot0=st.sc.adot[0])
        a.step(K)
        a.save(path)
        f, d, h, l = a.download_state()
        a.step(M)
        want = _snapshot(a)
    port = ck.read_state(path)
    assert port["step"] == K and ck.read_restart_header(path)["precision"] == precision
    np.testing.assert_array_equal(port["field"], f)
    np.testing.assert_array_equal(port["dfield"], d)
    np.testing.assert_array_equal(port["l"], l)
    with _lat(cfg, precision, flags) as b:
        assert b.load(path) is True
        b.step(M)
        got = _snapshot(b)
    _same(got, want)


def _same(got, want):
    """State and scalars bit for bit; the spectra to 1e-12, because the
    binning adds FP64 histogram entries with shared-memory atomics whose
    order (and so the last bit of a bin) varies from run to run."""
    for x, y in zip(got[:5], want[:5]):
        np.testing.assert_array_equal(x, y)
    np.testing.assert_allclose(got[5], want[5], rtol=1e-12, atol=0)


def test_a_dump_without_restart_block_is_an_initial_state(tmp_path):
    cfg = po.Config(N=32, model=po.MODEL_LPHI4, gws=1)
    st = po.init_state(cfg)
    po.step(st, 3)
    path = str(tmp_path / "ref.bin")
    po.write_dump(path, st)
    with _lat(cfg, gb.FP64, 0) as a, _lat(cfg, gb.FP64, 0) as b:
        assert a.load(path) is False
        b.upload_state(st.field[0], st.dfield[0], st.h[0], st.l[0], a0=st.sc.a[0], adot0=st.sc.adot[0])
        a.step(4)
        b.step(4)
        _same(_snapshot(a), _snapshot(b))


def test_load_refuses_a_dump_of_another_lattice(tmp_path):
    cfg = po.Config(N=16, model=po.MODEL_LPHI4, gws=1)
    st = po.init_state(cfg)
    path = str(tmp_path / "n16.bin")
    po.write_dump(path, st)
    with _lat(po.Config(N=32, model=po.MODEL_LPHI4, gws=1), gb.FP64, 0) as a:
        with pytest.raises(gb.GabeError) as ei:
            a.load(path)
        assert ei.value.code == 1
