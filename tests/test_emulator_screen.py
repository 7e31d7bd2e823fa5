"""Host logic of the emulator's screen-and-fallback sweep
(gabe_b200.emulator.screened_sweep): the emulator answers every
(point, output time), the points whose member spread exceeds the threshold
are evolved on the lattice and answered by it.  The emulator and the
lattice runner are stand-ins here, so the row order, the flagging and the
merge are checked without a GPU."""
import numpy as np

from gabe_b200 import emulator as em

NLOG = 4


class FakeEmulator:
    """mean = 10 * log10 g + tau in every output; spread = amplitude / 10 on
    every output but the last, which holds a large spread that only counts
    when the valid mask lets it."""

    def predict(self, feats):
        f = np.asarray(feats)
        mean = np.repeat((10 * f[:, 0] + f[:, 2])[:, None], 3 * NLOG, axis=1)
        spread = np.repeat((f[:, 1] / 10)[:, None], 3 * NLOG, axis=1)
        spread[:, -1] = 5.0
        return mean, spread


class FakeLattice:
    def __init__(self):
        self.calls = []

    def __call__(self, N, g, amp, seeds, steps, every, nlog, dt=0.01):
        self.calls.append((np.array(N), np.array(g), np.array(amp), np.array(seeds)))
        taus = em.output_times(steps, every, dt)
        T, P = len(taus), len(g)
        # time-major, point-minor, as ensemble_samples: -(seed) - 100 tau in every bin
        y = -(np.tile(seeds, T)[:, None] + 100 * np.repeat(taus, P)[:, None]) * np.ones((1, 3 * nlog))
        return None, y, np.tile(np.arange(P), T), 1.0


def _sweep():
    N = np.array([32, 64, 48, 32, 128])
    g = np.array([1.0, 10.0, 100.0, 3.0, 300.0])
    amp = np.array([0.5, 1.5, 0.7, 1.9, 1.0])
    seeds = np.array([11, 12, 13, 14, 15])
    return N, g, amp, seeds


def test_flagged_points_come_from_the_lattice_and_the_rest_from_the_emulator():
    N, g, amp, seeds = _sweep()
    lat = FakeLattice()
    valid = np.ones(3 * NLOG, dtype=bool)
    valid[-1] = False  # the bin with the large fake spread does not count
    ans, flagged, spread = em.screened_sweep(FakeEmulator(), 0.12, N, g, amp, seeds, steps=100, every=50,
                                             nlog=NLOG, valid_mask=valid, runner=lat)
    np.testing.assert_allclose(spread, amp / 10)
    assert flagged.tolist() == [False, True, False, True, False]
    assert len(lat.calls) == 1  # one batched run of the flagged points, in their order
    cN, cg, camp, cseeds = lat.calls[0]
    assert cN.tolist() == [64, 32] and cg.tolist() == [10.0, 3.0] and camp.tolist() == [1.5, 1.9]
    assert cseeds.tolist() == [12, 14]
    taus = em.output_times(100, 50)
    assert ans.shape == (len(taus) * 5, 3 * NLOG)
    rows = ans.reshape(len(taus), 5, 3 * NLOG)
    for t, tau in enumerate(taus):
        for p in range(5):
            want = -(seeds[p] + 100 * tau) if flagged[p] else 10 * np.log10(g[p]) + tau
            np.testing.assert_allclose(rows[t, p], want)


def test_no_lattice_run_when_nothing_is_flagged_and_the_mask_decides():
    N, g, amp, seeds = _sweep()
    lat = FakeLattice()
    ans, flagged, _ = em.screened_sweep(FakeEmulator(), 0.5, N, g, amp, seeds, steps=50, every=50, nlog=NLOG,
                                        valid_mask=np.arange(3 * NLOG) < 3 * NLOG - 1, runner=lat)
    assert not flagged.any() and lat.calls == []
    # without a mask the large spread of the last output flags every point
    ans2, flagged2, spread2 = em.screened_sweep(FakeEmulator(), 0.5, N, g, amp, seeds, steps=50, every=50,
                                                nlog=NLOG, runner=lat)
    assert flagged2.all() and np.all(spread2 == 5.0)
    assert len(lat.calls) == 1 and lat.calls[0][3].tolist() == seeds.tolist()
    # a per-point mask: only point 2 counts its last output
    vm = np.ones((5, 3 * NLOG), dtype=bool)
    vm[:, -1] = False
    vm[2, -1] = True
    _, flagged3, _ = em.screened_sweep(FakeEmulator(), 0.5, N, g, amp, seeds, steps=50, every=50, nlog=NLOG,
                                       valid_mask=vm, runner=lat)
    assert flagged3.tolist() == [False, False, True, False, False]


def test_output_times_match_the_recording_loop():
    np.testing.assert_allclose(em.output_times(2000, 50), np.arange(41) * 0.5)
    np.testing.assert_allclose(em.output_times(120, 50, dt=0.02), [0.0, 1.0, 2.0])
