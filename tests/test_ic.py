"""gabe_b200.ic.random_state with the reference's initial-spectrum knobs
(g2parameters.h:72-74, randInit g2init.cpp:117-165).

field_full_rand 0 is deterministic, so the generator must reproduce the
oracle's initial state -- which tests/test_oracle_golden.py pins bit for bit
to the reference built with those knobs -- to FFT rounding.  spec_cut_off
multiplies every mode of the random draws by the window
(1 - tanh(spec_smooth (|n| - N spec_cut_off)))/2: with the same seed, phi's
spectrum with the cut-off is the spectrum without it times the window."""
import math

import numpy as np
import pytest
import torch

from gabe_b200.ic import random_state
from oracle import pyoracle as po

CUT, SMOOTH = math.sqrt(3.0) / 8.0, 0.5


def test_deterministic_spectrum_matches_oracle():
    N = 32
    cfg = po.Config(N=N, model=po.MODEL_LPHI4, gws=0, ic_variant=2)
    st = po.init_state(cfg)
    c0, c1, B, f0, df0 = po.model_constants(cfg.model)
    f, d, a0, adot0 = random_state(N, model_c=(c0, c1), rescale_B=B, f0=f0, df0=df0, spec_cut_off=CUT,
                                   spec_smooth=SMOOTH, full_rand=False)
    f, d = f.numpy(), d.numpy()
    for got, want in ((f, st.field[0]), (d, st.dfield[0])):
        for q in range(2):
            fl = want[q] - want[q].mean()
            assert np.abs(got[q] - want[q]).max() <= 1e-10 * np.abs(fl).max() + 1e-300, q
    # adot0 from the homogeneous energy in closed form; the reference sums it over N^3 sites
    assert a0 == st.sc.a[0] and abs(adot0 - st.sc.adot[0]) <= 1e-12 * st.sc.adot[0]


def test_spectral_cut_off_scales_every_mode():
    N = 32
    kw = dict(seed=5)
    f1, d1, _, _ = random_state(N, **kw)
    f2, d2, _, _ = random_state(N, spec_cut_off=CUT, spec_smooth=SMOOTH, **kw)
    i = np.arange(N)
    i2 = np.where(i < N // 2 + 1, i * i, (N - i) ** 2).astype(float)
    k2 = np.arange(N // 2 + 1, dtype=float) ** 2
    n = np.sqrt(i2[:, None, None] + i2[None, :, None] + k2[None, None, :])
    window = (1.0 - np.tanh(SMOOTH * (n - N * CUT))) / 2.0
    for a, b in ((f1[0], f2[0]), (d1[0], d2[0])):  # phi: its omega_k does not depend on the draws
        A = np.fft.rfftn((a - a.mean()).numpy())
        Bk = np.fft.rfftn((b - b.mean()).numpy())
        ok = np.abs(A) > 1e-8 * np.abs(A).max()
        assert np.all(np.abs(Bk[ok] - window[ok] * A[ok]) <= 1e-9 * np.abs(A).max())
        assert window[ok].min() < 1e-3  # the cut-off bites inside the lattice


def test_deterministic_spectrum_needs_the_cut_off():
    with pytest.raises(ValueError):
        random_state(8, full_rand=False)
