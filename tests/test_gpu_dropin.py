"""The drop-in: GABE's own driver (g2main.cpp) with step(), specOut() and
outputslice() taken by gabe_b200/host/gabe_dropin.cpp -- the field slices,
means/variances and spectra computed on the GPU, no state download -- against
the same program built entirely from the reference sources.  Every file under
slices/ must match to the precision the reference prints (%e, 7 significant
digits), apart from quantities the reference computes with cancellation: the
mean and variance columns of meansvariances.dat (a serial mean of f ~ 0.34,
then sum of f^2 - mean^2: noise ~ eps mean^2 sqrt(N^3), and chi's mean, zero
in exact arithmetic) and the gradient-energy column of slices_time.dat (sum
of -f lap f).

Both programs are compiled by `make -C oracle full dropin` where the
reference tree is mounted; the binaries travel with the repository."""
import glob
import os
import subprocess

import numpy as np
import pytest

from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


def _run(binary, cwd):
    os.makedirs(os.path.join(cwd, "slices"), exist_ok=True)
    r = subprocess.run([binary], cwd=cwd, capture_output=True, text=True, timeout=600,
                       env=dict(os.environ, GABE_REF_THREADS="1"))
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]


def _close(got, want, rtol, floor_frac=0.0):
    floor = floor_frac * np.abs(want).max(axis=0, keepdims=True) if want.ndim == 2 else 0.0
    return np.all(np.abs(got - want) <= rtol * np.abs(want) + floor + 1e-300)


@pytest.mark.parametrize("cfg", ["m1_n32_g1_p0", "m1_n32_g0_p0"])
def test_dropin_program_matches_reference_program(cfg, tmp_path):
    ref_bin = os.path.join(po.REF_DIR, f"reffull_{cfg}")
    gpu_bin = os.path.join(po.REF_DIR, f"dropin_{cfg}")
    if not (os.path.exists(ref_bin) and os.path.exists(gpu_bin)):
        pytest.skip("drop-in programs are built by `make -C oracle full dropin` where the reference is mounted")
    a, b = tmp_path / "ref", tmp_path / "gpu"
    _run(ref_bin, str(a))
    _run(gpu_bin, str(b))
    names = sorted(os.path.basename(p) for p in glob.glob(str(a / "slices" / "*.dat")))
    assert names == sorted(os.path.basename(p) for p in glob.glob(str(b / "slices" / "*.dat")))
    assert any(n.startswith("slices_spectra_") for n in names) and "slices_time.dat" in names
    for n in names:
        want = np.loadtxt(a / "slices" / n, ndmin=2)
        got = np.loadtxt(b / "slices" / n, ndmin=2)
        assert got.shape == want.shape, n
        if n == "slices_time.dat":
            cols = [c for c in range(want.shape[1]) if c != 6]
            assert _close(got[:, cols], want[:, cols], 2e-6), n
            assert _close(got[:, 6], want[:, 6], 1e-4), n
        elif n == "meansvariances.dat":
            # columns: t, then (mean, variance) per field
            assert _close(got[:, [0, 1]], want[:, [0, 1]], 2e-6), n
            assert np.all(np.abs(got[:, 3] - want[:, 3]) <= 1e-20), n  # chi: rounding noise of a zero mean
            N = 32
            for c in (2, 4):
                av = want[:, c - 1]
                tol = 1e-3 * np.abs(want[:, c]) + 16 * np.finfo(float).eps * av * av * N ** 1.5
                assert np.all(np.abs(got[:, c] - want[:, c]) <= tol), n
        elif n.startswith("slices_spectra_"):
            assert _close(got, want, 1e-5, floor_frac=1e-10), n
        else:
            assert _close(got, want, 2e-6), n


def test_dropin_checkpoint_and_restart_continue_the_run(tmp_path):
    """GABE_B200_CHECKPOINT(_EVERY) writes checkpoints from the drop-in
    program; GABE_B200_RESTART starts a new run from one, at the saved
    step's time.  The restarted run's slices_time.dat rows must equal the
    uninterrupted run's rows at the same times, to every printed digit (the
    restart block holds the device state bit for bit)."""
    gpu_bin = os.path.join(po.REF_DIR, "dropin_m1_n32_g1_p0")
    if not os.path.exists(gpu_bin):
        pytest.skip("drop-in programs are built by `make -C oracle full dropin` where the reference is mounted")
    a, b = tmp_path / "full", tmp_path / "restart"
    for d in (a, b):
        os.makedirs(d / "slices")
    ck = str(tmp_path / "ck_%d.bin")
    env = dict(os.environ, GABE_REF_THREADS="1", GABE_B200_CHECKPOINT=ck, GABE_B200_CHECKPOINT_EVERY="10")
    r = subprocess.run([gpu_bin], cwd=str(a), capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    assert os.path.exists(str(tmp_path / "ck_10.bin"))
    env = dict(os.environ, GABE_REF_THREADS="1", GABE_B200_RESTART=str(tmp_path / "ck_10.bin"))
    r = subprocess.run([gpu_bin], cwd=str(b), capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "restarted from" in r.stdout
    full = {row[0]: row for row in np.loadtxt(a / "slices" / "slices_time.dat", ndmin=2)}
    rest = np.loadtxt(b / "slices" / "slices_time.dat", ndmin=2)
    assert rest[0, 0] == pytest.approx(0.1) and len(rest) >= 2
    common = [row for row in rest if row[0] in full]
    assert len(common) >= 2
    for row in common:
        np.testing.assert_array_equal(row, full[row[0]])
