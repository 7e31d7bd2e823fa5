"""Host helpers of the FP32-vs-FP64 error report (gabe_b200.accuracy): the
RK2 stability number and the per-bin spectrum difference with its noise
floor, on hand-made tables."""
import numpy as np
import pytest

from gabe_b200 import accuracy as acc


def test_stability_theta_of_the_reference_default_and_the_headline_runs():
    # the reference's default dt = dx / 80 (g2parameters.h:61)
    assert acc.stability_theta(512, 20.0, 20.0 / 512 / 80) == pytest.approx(np.sqrt(12) / 80)
    # dt = dx / 40, the accuracy runs
    assert acc.stability_theta(256, 20.0, 20.0 / 256 / 40) == pytest.approx(0.0866, abs=1e-4)
    # dt = 0.01 at 512^3: outside the stable range for the top modes
    assert acc.stability_theta(512, 20.0, 0.01) == pytest.approx(0.887, abs=1e-3)


def _table(nb=20, seed=0):
    rng = np.random.default_rng(seed)
    t = np.zeros((nb, 8))
    t[:, 0] = np.arange(nb)
    t[:, 1:7] = 10.0 ** rng.uniform(-6, 2, size=(nb, 6))
    return t


def test_relative_difference_per_bin_above_the_floor():
    want = _table()
    got = want.copy()
    b = int(np.argmax(want[:, 3]))
    got[b, 3] *= 1 + 3e-5  # the largest bin of the chi column off by 3e-5
    got[0, 3] += 0.5e-9 * want[b, 3]  # and a small bin by half the floor: not reported
    d = acc.spectra_rel_diff(got, want, acc.FIELD_COLS)
    assert d == pytest.approx(3e-5 - 1e-9, rel=1e-6)
    assert acc.spectra_rel_diff(got, want, acc.GW_COLS) == 0.0  # other columns untouched


def test_differences_below_the_noise_floor_and_empty_bins_count_as_zero():
    want = _table()
    want[0, 1:7] = 0.0  # the k = 0 bin of a mean-free field
    got = want.copy()
    got[:, 1] += 1e-10 * np.abs(want[:, 1]).max()  # below 1e-9 of the column's largest value
    assert acc.spectra_rel_diff(got, want, acc.FIELD_COLS) == 0.0
    # a bin that should be empty but is not, above the floor, is reported
    got[0, 5] = 1e-3 * np.abs(want[:, 5]).max()
    assert acc.spectra_rel_diff(got, want, acc.GW_COLS) > 1e100
