"""Energy-conservation error on the GPU (gabe_b200.energy, the continuity
residual eps(t) of the per-step scalars): the FP64 path's eps(t) is the
oracle's (the reference's step() restated) to 1e-9, and the FP32-storage
path's is the FP64 path's to 1e-5, well inside the 1e-4 the FP32 form is
held to."""
import numpy as np
import pytest

import gabe_b200 as gb
from gabe_b200 import energy
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


def test_continuity_residual_fp64_is_the_oracles_and_fp32_follows():
    N, steps = 32, 200
    cfg = po.Config(N=N, model=po.MODEL_LPHI4, gws=1)
    st = po.init_state(cfg)
    c0, c1, *_ = po.model_constants(cfg.model)
    f0, d0, h0, l0 = st.field[0].copy(), st.dfield[0].copy(), st.h[0].copy(), st.l[0].copy()
    a0, ad0 = st.sc.a[0], st.sc.adot[0]
    rows_o = [(0.0, a0, ad0, st.sc.edkin[0], st.sc.edpot[0], st.sc.edgrad[0], st.sc.edrho[0])]
    for n in range(steps):
        po.step(st, 1)
        s = st.sc
        rows_o.append(((n + 1) * cfg.dt, s.a[0], s.adot[0], s.edkin[0], s.edpot[0], s.edgrad[0], s.edrho[0]))
    eps = {"oracle": energy.continuity_residual(*np.array(rows_o).T)}
    for name, prec in (("fp64", gb.FP64), ("fp32", gb.FP32)):
        with gb.Lattice(N, L=cfg.L, dt=cfg.dt, gws=True, model=cfg.model, model_c=(c0, c1), precision=prec) as lat:
            lat.upload_state(f0, d0, h0, l0, a0=a0, adot0=ad0)
            rows = []
            for n in range(steps + 1):
                if n:
                    lat.step(1)
                e = lat.calc_energy()
                rows.append((n * cfg.dt, e["a"], e["adot"], e["kin"], e["pot"], e["grad"], e["rho"]))
        eps[name] = energy.continuity_residual(*np.array(rows).T)
    assert eps["oracle"][-1] > 0
    assert np.abs(eps["fp64"] - eps["oracle"]).max() <= 1e-9
    assert np.abs(eps["fp32"] - eps["fp64"]).max() <= 1e-5
