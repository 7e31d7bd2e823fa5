"""The oracle's restatements of meansvars (g2output.cpp:70-121) and of the
outputfield rows with calcrho and its fourth-order gradients
(g2output.cpp:25-68, g2functions.cpp:70-122,176-186), pinned against the
files the reference program itself writes: the whole reference program
(g2main.cpp and g2output.cpp included, built by `make -C oracle full`) runs
20 steps of a 32^3 lattice with field_outdim 2, field_sliceskip 2 and
var_output 1, and every slices_fields_<n>.dat and meansvariances.dat row must
match the oracle's state at the same step to the precision the reference
prints (%e: 7 significant digits; the variance column, a sum of f^2 - mean^2
with f ~ 0.34, to its cancellation noise, see variance_tol)."""
import os
import tempfile

import numpy as np
import pytest

from oracle import pyoracle as po


def test_field_slices_and_meansvars_match_reference_program():
    binary = os.path.join(po.REF_DIR, "reffull_m1_n32_g0_p0")
    if not os.path.exists(binary):
        pytest.skip("built by `make -C oracle full` where the reference is mounted")
    cfg = po.Config(N=32, model=po.MODEL_LPHI4, gws=0)
    with tempfile.TemporaryDirectory() as d:
        po.run_ref(binary, [], d, threads=1)
        mv_ref = np.loadtxt(os.path.join(d, "slices", "meansvariances.dat"), ndmin=2)
        slices = [np.loadtxt(os.path.join(d, "slices", f"slices_fields_{n}.dat")) for n in range(5)]
    st = po.init_state(cfg)
    for n in range(5):
        if n:
            po.step(st, 5)
        got = po.field_slice(cfg, st.field[0], st.dfield[0], st.sc.a[0], 2, 2)
        assert got.shape == slices[n].shape == (256, 3)
        assert np.all(np.abs(got - slices[n]) <= 6e-7 * np.abs(slices[n]) + 1e-300), n
        mv = po.meansvars(st.field[0])
        for q in range(2):
            av, var = mv_ref[n, 1 + 2 * q], mv_ref[n, 2 + 2 * q]
            rms = float(np.sqrt(np.mean(st.field[0, q] ** 2)))
            assert abs(mv[q, 0] - av) <= mean_tol(av, rms), (n, q)
            assert abs(mv[q, 1] - var) <= variance_tol(var, av, cfg.N), (n, q)


def mean_tol(av, rms):
    """%e precision, plus the rounding noise of a serial mean (~eps rms): chi
    has zero mean in exact arithmetic and prints noise of order 1e-26."""
    return 6e-7 * abs(av) + 16 * np.finfo(float).eps * rms


def variance_tol(var, av, N):
    """meansvars forms the variance as sum(f^2 - mean^2)/N^3 after a serial
    sum for the mean: the mean's rounding error (~sqrt(N^3) eps |mean|)
    enters every term through mean^2, so the printed variance of a field with
    a large mean and tiny fluctuations (phi ~ 0.34 +- 1e-7) carries absolute
    noise ~ eps mean^2 sqrt(N^3); 16 times that plus 1e-3 relative."""
    return 1e-3 * abs(var) + 16 * np.finfo(float).eps * av * av * N ** 1.5
