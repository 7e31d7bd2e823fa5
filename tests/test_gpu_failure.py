"""Failure detection on the GPU without a fault: every wait of the library's
kernels on an mbarrier (bulk copies of the transform passes, the TMA loads
and MMAs of the emulator's tcgen05 forward) is bounded by GPU time and
reports ST_TIMEOUT through a status word.  gabe_wait_probe runs that wait on
a barrier that nothing arrives at (the failure made on purpose); the wait
must give up after its limit, the status must reach the host, and the
context must stay usable for the next lattice."""
import time

import numpy as np
import pytest

import gabe_b200 as gb

pytestmark = pytest.mark.gpu


def test_bounded_wait_gives_up_and_reports_the_timeout():
    limit = 200_000_000  # 0.2 s of GPU time
    t0 = time.perf_counter()
    rc, status, waited = gb.wait_probe(limit)
    elapsed = time.perf_counter() - t0
    assert rc == 6, gb.STATUS.get(rc, rc)  # GABE_ERR_TIMEOUT
    assert status & 2  # ST_TIMEOUT
    assert limit <= waited < 5 * limit
    assert elapsed < 30


def test_context_stays_usable_after_a_timeout():
    assert gb.wait_probe(50_000_000)[0] == 6
    N = 32
    rng = np.random.default_rng(3)
    f = 0.3 + 1e-3 * rng.standard_normal((2, N, N, N))
    d = 1e-4 * rng.standard_normal((2, N, N, N))
    with gb.Lattice(N, gws=True, precision=gb.FP32) as lat:
        lat.upload_state(f, d, adot0=0.1)
        lat.step(3)
        e = lat.calc_energy()
    assert all(np.isfinite(v) for v in e.values())
