"""gabe_b200.energy: the continuity residual eps(t) of a run's scalars, on
the CPU.  An exact FRW background gives eps ~ 0 (trapezoid error only); on
oracle runs (the reference's step() restated) eps falls as dt^2, as RK2
with a fixed step must."""
import numpy as np
import pytest

from gabe_b200 import energy
from oracle import pyoracle as po


def _oracle_rows(N, dt, steps):
    cfg = po.Config(N=N, model=po.MODEL_LPHI4, gws=0, dt=dt)
    st = po.init_state(cfg)

    def row(t):
        s = st.sc
        return (t, s.a[0], s.adot[0], s.adot[0] / s.a[0], s.edkin[0], s.edpot[0], s.edgrad[0], s.edrho[0])

    rows = [row(0.0)]
    for n in range(steps):
        po.step(st, 1)
        rows.append(row((n + 1) * dt))
    return np.array(rows)


def test_exact_background_has_no_residual():
    # stiff matter (kin only, p = rho): a = t^(1/3), H = 1/(3t), rho = 3H^2/(8 pi)
    t = np.linspace(1.0, 2.0, 4001)
    a, H = t ** (1.0 / 3.0), 1.0 / (3.0 * t)
    rho = 3.0 * H ** 2 / (8.0 * np.pi)
    z = np.zeros_like(t)
    eps = energy.continuity_residual(t, a, a * H, rho, z, z, rho)
    assert eps[0] == 0.0 and eps.max() < 1e-6
    # the same background with a missing 10 % of kinetic pressure is caught
    bad = energy.continuity_residual(t, a, a * H, 0.9 * rho, z, z, rho)
    assert bad.max() > 1e-2


def test_oracle_residual_falls_as_dt_squared():
    eps = [energy.residual_from_rows(_oracle_rows(32, dt, steps))[-1]
           for dt, steps in ((0.02, 100), (0.01, 200), (0.005, 400))]
    assert 0 < eps[2] < eps[1] < eps[0] < 1e-2
    for coarse, fine in zip(eps, eps[1:]):
        assert 3.8 < coarse / fine < 4.2, eps


def test_bad_series_are_rejected():
    with pytest.raises(ValueError):
        energy.continuity_residual([0.0, 1.0], [1.0], [0.0, 0.0], [1.0, 1.0], [0.0, 0.0], [0.0, 0.0], [1.0, 1.0])
    with pytest.raises(ValueError):
        energy.continuity_residual([1.0, 0.0], [1.0, 1.0], [0.0, 0.0], [1.0, 1.0], [0.0, 0.0], [0.0, 0.0],
                                   [1.0, 1.0])
    with pytest.raises(ValueError):
        energy.residual_from_rows(np.zeros((3, 7)))


def test_command_line_check_on_the_reference_programs_own_file(tmp_path, capsys):
    """`python -m gabe_b200.energy slices_time.dat` on the file the whole
    reference program writes (g2main.cpp and g2output.cpp, built by
    `make -C oracle full`): one row per output slice, eps(t0) = 0, and the
    same eps as the library function on the same rows."""
    import json
    import os

    binary = os.path.join(po.REF_DIR, "reffull_m1_n32_g0_p0")
    if not os.path.exists(binary):
        pytest.skip("built by `make -C oracle full` where the reference is mounted")
    po.run_ref(binary, [], str(tmp_path), threads=1)
    path = str(tmp_path / "slices" / "slices_time.dat")
    out = energy.main([path])
    assert json.loads(capsys.readouterr().out.strip().splitlines()[-1]) == out
    rows = np.loadtxt(path, ndmin=2)
    eps = energy.residual_from_rows(rows)
    assert out["rows"] == rows.shape[0] >= 2 and eps[0] == 0.0
    assert out["eps_end"] == eps[-1] and out["eps_max"] == eps.max()
    assert 0.0 < out["eps_max"] < 1e-2
