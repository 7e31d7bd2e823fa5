"""Parity and accuracy at the lattice sizes of the headline configurations.

* 256^3, FP64, GWs on (L = 20, dt = 0.01, lambda phi^4 with g^2/lambda =
  100): the reference program, built from its own sources (oracle/_ref,
  step() of g2functions.cpp:234-271 with evolve_perts of
  g2evolutionpert.cpp:343-455 and its initial conditions of g2init.cpp:
  68-189), writes its initial state and its states after 1, 10 and 20
  steps.  The library starts from the reference's initial dump and must
  match every later dump: fields and momenta pointwise to 1e-10 relative,
  a and adot to 1e-12, h and l in norm to 1e-12 after the first step (its
  sources are bit-identical; the two FFTs differ at rounding level) and to
  1e-8 later (the energy sums are added in another order, so a last-bit
  difference of phi ~ 0.34 enters the source gradients).
* FP32 storage against the FP64 path at 256^3 with GWs, 500 steps at
  dt = dx/40 (theta = dt sqrt(12)/dx = 0.087, inside RK2's stability
  region): a, adot, kin, pot, grad, rho, the continuity residual and every
  spectrum column per bin within 1e-4 (gabe_b200.accuracy).
"""
import os

import numpy as np
import pytest

import gabe_b200 as gb
from gabe_b200.accuracy import compare_precisions
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


def _pointwise_rel(got, want):
    """max over points of |got-want| / (|want| + rms(want))."""
    scale = np.abs(want) + np.sqrt(np.mean(want * want))
    return float(np.max(np.abs(got - want) / scale))


def _norm_rel(got, want):
    n = np.linalg.norm(want)
    return float(np.linalg.norm(got - want) / n) if n > 0 else float(np.abs(got).max())


REF256 = po.ref_binary(po.MODEL_LPHI4, 256, 1, 1)


@pytest.mark.skipif(not os.path.exists(REF256), reason="reference build oracle/_ref/ref_m1_n256_g1_p1 missing "
                                                       "(make -C oracle ref)")
def test_fp64_256cubed_gws_matches_the_reference_build(tmp_path):
    dumps = (0, 1, 10, 20)
    po.run_ref(REF256, ["--steps", str(dumps[-1]), "--dump-at", ",".join(map(str, dumps)),
                        "--dump-prefix", str(tmp_path / "state_")], str(tmp_path), threads=os.cpu_count(),
               timeout=1800)
    cfg = po.Config(N=256, model=po.MODEL_LPHI4, gws=1)
    st = po.read_dump(str(tmp_path / "state_0.bin"), cfg)
    c0, c1, *_ = po.model_constants(cfg.model)
    with gb.Lattice(cfg.N, L=cfg.L, dt=cfg.dt, gws=True, model=cfg.model, model_c=(c0, c1)) as lat:
        lat.upload_state(st.field[0], st.dfield[0], st.h[0], st.l[0], a0=st.sc.a[0], adot0=st.sc.adot[0])
        del st
        done = 0
        for n in dumps[1:]:
            lat.step(n - done)
            done = n
            ref = po.read_dump(str(tmp_path / f"state_{n}.bin"), cfg)
            f, d, h, l = lat.download_state()
            sc = lat.scalars()
            assert _pointwise_rel(f, ref.field[0]) <= 1e-10, n
            assert _pointwise_rel(d, ref.dfield[0]) <= 1e-10, n
            for k in ("a", "adot"):
                assert abs(sc[k][0] - getattr(ref.sc, k)[0]) <= 1e-12 * abs(getattr(ref.sc, k)[0]), (n, k)
            tol = 1e-12 if n == 1 else 1e-8
            assert np.linalg.norm(ref.l[0]) > 0
            assert _norm_rel(h, ref.h[0]) <= tol, n
            assert _norm_rel(l, ref.l[0]) <= tol, n
            del ref, f, d, h, l
            os.remove(tmp_path / f"state_{n}.bin")


@pytest.mark.parametrize("flags32", [0, gb.FLAG_TRANSPOSED_FFT])
def test_fp32_matches_fp64_at_256cubed_over_500_stable_steps(flags32):
    from gabe_b200.ic import random_state

    N, L = 256, 20.0
    f, d, a0, ad0 = random_state(N, seed=9, device="cuda")
    f, d = f.cpu().numpy(), d.cpu().numpy()
    rep = compare_precisions(f, d, a0, ad0, N=N, steps=500, dt=L / N / 40, L=L, gws=True, spectra_every=100,
                             flags32=flags32)
    assert rep["finite"] and rep["theta"] < 0.1
    assert rep["max_rel_err"] <= 1e-4, rep
    assert rep["eps_max_abs_diff"] <= 1e-6, rep
