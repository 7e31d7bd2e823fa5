"""What the trained emulator gains over the sweep without it, on a small
sweep (uniform 32^3 lattices so that the held-out check runs at the training size):

* accuracy: on held-out parameter points evolved on the lattice, the
  emulator's phi, chi and GW log spectra are closer to the lattice than the
  best the sweep has without it -- the spectra of the nearest training
  lattice of the same size;
* cost: one emulator query (one parameter point at one time) costs a
  tiny fraction of the lattice run it replaces;
* screening: points flagged for a lattice re-run are those whose member
  spread exceeds the threshold calibrated on validation lattices.
"""
import numpy as np
import pytest

from gabe_b200 import emulator as em

pytestmark = pytest.mark.gpu


def test_emulator_beats_nearest_neighbour_and_is_cheaper_than_the_lattice():
    rep = em.run_sweep(nlat=160, ensembles=1, steps=600, every=50, holdout=16, holdout_N=32, members=2, epochs=300,
                       batch=256, master_seed=4242, sizes=(32,), log=lambda *a: None)
    mae = rep["mae_dex"]
    for f in ("phi", "chi", "gw"):
        assert mae["emulator"][f] < mae["nearest_neighbour"][f], (f, mae)
        assert mae["emulator"][f] < 0.2
    # one lattice run yields len(tau) spectra; the emulator answers that many
    # queries far faster than the lattice runs
    assert rep["spectra_per_s_emulator_over_lattice"] > 1e4
    assert rep["n_flagged"] == len(rep["flagged_points"]) <= 16
    assert np.isfinite(rep["flag_threshold_dex"])


def test_emulator_trained_on_uneven_sizes_beats_nearest_neighbour_at_the_checked_size():
    """Training lattices of two sizes, checked at the larger: the lattice size is
    an input, so the GW spectra -- which differ strongly between sizes -- are
    emulated for the size asked for, and every column beats the lookup of the
    nearest training lattice of that size."""
    rep = em.run_sweep(nlat=160, ensembles=1, steps=600, every=50, holdout=16, holdout_N=64, members=2, epochs=300,
                       batch=256, master_seed=4242, sizes=(32, 64), log=lambda *a: None)
    mae = rep["mae_dex"]
    for f in ("phi", "chi", "gw"):
        assert mae["emulator"][f] < mae["nearest_neighbour"][f], (f, mae)
