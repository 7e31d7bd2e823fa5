"""Known-answer tests of the oracle (derived from the mathematics)."""
import math

import numpy as np
import pytest

from oracle import pyoracle as po
from tests.kspace_ref import pol_tensors, sym, tt_project


def test_laplacian_plane_wave_eigenvalue():
    N, L, A = 16, 20.0, 1e-3
    cfg = po.Config(N=N, L=L, model=po.MODEL_LPHI4)
    dx = L / N
    x = np.arange(N)
    n = (1, 2, 3)
    th = [2 * math.pi * q / N for q in n]
    f = np.zeros((2, N, N, N))
    f[0] = A * np.cos(th[0] * x[:, None, None] + th[1] * x[None, :, None] + th[2] * x[None, None, :])
    df = np.zeros_like(f)
    e = po.calc_energy(cfg, f, df, 1.3)
    lam = 4 / dx ** 2 * sum(math.sin(t / 2) ** 2 for t in th)
    assert e[0] == 0.0
    assert abs(e[2] - lam * A * A / 4 / 1.3 ** 2) <= 1e-12 * abs(e[2])


def test_potential_derivatives_consistent():
    for model in (po.MODEL_QUADRATIC, po.MODEL_LPHI4):
        cfg = po.Config(N=8, model=model)
        p = cfg.params()
        L = po.lib()
        for (P, C) in [(0.3, 0.01), (0.1, -0.2), (-0.25, 0.05)]:
            for fld in (0, 1):
                h = 1e-6
                if fld == 0:
                    fd = (L.ora_potential(p, P + h, C) - L.ora_potential(p, P - h, C)) / (2 * h)
                else:
                    fd = (L.ora_potential(p, P, C + h) - L.ora_potential(p, P, C - h)) / (2 * h)
                an = L.ora_dvdf(p, fld, P, C)
                assert abs(fd - an) <= 1e-6 * max(1.0, abs(an)), (model, fld, fd, an)


@pytest.mark.parametrize("seed", range(5))
def test_tt_projection_formulas_agree(seed):
    rng = np.random.default_rng(seed)
    n = rng.integers(-8, 9, size=3)
    if not n.any():
        n[0] = 1
    S = rng.standard_normal(6) + 1j * rng.standard_normal(6)
    # make S traceless, as the real-space source is
    tr = (S[0] + S[3] + S[5]) / 3
    S[0] -= tr; S[3] -= tr; S[5] -= tr
    nm = 0.37
    Sri = np.zeros(12)
    Sri[0::2], Sri[1::2] = S.real, S.imag
    Tref = po.tt_point(n, nm, Sri)
    k = n / np.linalg.norm(n)
    T = nm * tt_project(k, S)
    np.testing.assert_allclose(T.real, Tref[0::2], atol=1e-14 * np.abs(Tref).max())
    np.testing.assert_allclose(T.imag, Tref[1::2], atol=1e-14 * np.abs(Tref).max())
    # transverse, traceless, idempotent
    M = sym(T)
    assert np.abs(M @ k).max() <= 1e-13 * np.abs(M).max()
    assert abs(np.trace(M)) <= 1e-13 * np.abs(M).max()
    np.testing.assert_allclose(nm * tt_project(k, T / nm), T, atol=1e-13 * np.abs(T).max())


def test_homogeneous_state_follows_zero_mode_ode():
    N = 8
    cfg = po.Config(N=N, model=po.MODEL_LPHI4, gws=1)
    st = po.State.empty(cfg)
    phi0 = 0.342
    st.field[0, 0] = phi0
    lam, g, *_ = po.model_constants(po.MODEL_LPHI4)
    st.sc.a[0] = 1.0
    e = po.calc_energy(cfg, st.field[0], st.dfield[0], 1.0)
    st.sc.adot[0] = po.adf(e[3], 1.0)
    po.step(st, 20)
    # spatially homogeneous, and GWs are never sourced
    assert np.ptp(st.field[0, 0]) == 0.0 and np.ptp(st.dfield[0, 0]) == 0.0
    assert not st.h[0].any() and not st.l[0].any()
    # scalar RK2 of the same discrete scheme
    f, d, a, ad = phi0, 0.0, 1.0, st.sc.adot[0]
    ad = po.adf(lam / 4 * phi0 ** 4 + 0 * e[2], 1.0)
    dt = cfg.dt
    for _ in range(20):
        f1 = f + 0.5 * dt * d
        d1 = d + 0.5 * dt * (-lam * f ** 3 - 3 * ad / a * d)
        a1 = a + 0.5 * dt * ad
        ad1 = math.sqrt(8 * math.pi / 3 * (0.5 * d1 * d1 + lam / 4 * f1 ** 4)) * a1
        f, d = f + dt * d1, d + dt * (-lam * f1 ** 3 - 3 * ad1 / a1 * d1)
        a = a + dt * ad1
        ad = math.sqrt(8 * math.pi / 3 * (0.5 * d * d + lam / 4 * f ** 4)) * a
    assert abs(st.field[0, 0, 0, 0, 0] - f) <= 1e-9 * abs(f)
    assert abs(st.sc.a[0] - a) <= 1e-9 * a


def test_spectra_parseval_and_bins():
    N = 16
    cfg = po.Config(N=N, model=po.MODEL_LPHI4)
    st = po.init_state(cfg)
    sp = po.spectra(cfg, st.field[0], None, st.sc.edrho[0])
    nb = po.numbins(N)
    assert nb == int(math.sqrt(3) * N / 2 + 1) and sp.shape == (nb, 5)
    # counts from the geometry of the half spectrum
    cnt = np.zeros(nb)
    for i in range(N):
        px = i if i <= N // 2 else i - N
        for j in range(N):
            py = j if j <= N // 2 else j - N
            for kz in range(N // 2 + 1):
                w = 1 if kz in (0, N // 2) else 2
                cnt[int(math.sqrt(px * px + py * py + kz * kz))] += w
    assert cnt.sum() == N ** 3
    L = cfg.L
    spec_norm = (L / N) ** 6 * (2 * math.pi / L) ** 3
    for f in range(2):
        tot = (sp[:, 1 + 2 * f] * cnt / spec_norm).sum()
        want = N ** 3 * (st.field[0, f] ** 2).sum()
        assert abs(tot - want) <= 1e-10 * want


@pytest.mark.parametrize("n", [(1, 0, 0), (0, 0, 3), (0, 2, 0), (1, 1, 0), (3, -2, 5), (-4, 4, 4), (2, -7, 1)])
def test_polarization_basis_spans_the_tt_projector(n):
    """sum_p eps^p (x) eps^p / 2 equals Lambda, so evolving the two
    amplitudes X_p = eps^p:X/2 reproduces the six-component TT evolution;
    and with S33 = -S11 - S22 the traceless source gives the same eps^p:S."""
    ep, ex = pol_tensors(n)
    k = np.asarray(n, float) / np.linalg.norm(n)
    P = np.eye(3) - np.outer(k, k)
    lam = np.einsum("il,jm->ijlm", P, P) - 0.5 * np.einsum("ij,lm->ijlm", P, P)
    got = 0.5 * (np.einsum("ij,lm->ijlm", ep, ep) + np.einsum("ij,lm->ijlm", ex, ex))
    # Lambda acting on symmetric tensors: symmetrise over (l, m)
    lam_s = 0.5 * (lam + lam.transpose(0, 1, 3, 2))
    np.testing.assert_allclose(got, lam_s, atol=1e-14)
    for e in (ep, ex):
        assert abs(np.trace(e)) < 1e-14 and np.abs(e @ k).max() < 1e-14
        assert abs(np.sum(e * e) - 2.0) < 1e-14
    rng = np.random.default_rng(3)
    S = rng.standard_normal((3, 3)); S = S + S.T; S -= np.trace(S) / 3 * np.eye(3)
    T = np.einsum("ijlm,lm->ij", lam, S)
    recon = 0.5 * (np.sum(ep * S) * ep + np.sum(ex * S) * ex)
    np.testing.assert_allclose(recon, T, atol=1e-13)
