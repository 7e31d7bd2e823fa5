"""Index arithmetic of the library's row pass along k (fft3d.cuh
row_r2c_kernel), restated on the CPU for N in {64, 128, 256, 512} with the
four-step splits N = L1 L2 of fftreg.cuh FourStep:

* RowGeom::phys, the position of real e of a row in shared memory, permutes
  the row, keeps each pair of reals (2m, 2m+1) together and 8-byte aligned
  (the row lands with 8-byte copies), and puts the L2 reals read by one
  four-step column (n1 + L1 k2, k2 < L2) on distinct banks;
* the four-step order (L2-point FFTs over n2 at stride L1, twiddles
  W_N^(n1 k2), L1-point FFTs over n1, output k = k2 + L2 k1) is the DFT;
* two real rows travel as z = x_a + i x_b and separate into their half
  spectra as X_a[k] = (Z[k] + conj Z[N-k]) / 2, X_b[k] = (Z[k] - conj Z[N-k]) / 2i."""
import numpy as np
import pytest

SPLITS = {64: (8, 8), 128: (16, 8), 256: (16, 16), 512: (32, 16)}  # N: (L1, L2)


def phys(e, L1):
    cpr, h = 32 // L1, L1 // 2  # chunks per 32-bank row, pairs per chunk
    c, q = e // L1, (e % L1) >> 1
    return c * L1 + 2 * (q ^ ((c // cpr) % h)) + (e & 1)


@pytest.mark.parametrize("N", sorted(SPLITS))
def test_shared_layout_is_a_pair_preserving_permutation_with_distinct_banks(N):
    L1, L2 = SPLITS[N]
    pos = np.array([phys(e, L1) for e in range(N)])
    assert sorted(pos) == list(range(N))
    assert np.all(pos[0::2] % 2 == 0) and np.all(pos[1::2] == pos[0::2] + 1)
    for n1 in range(L1):
        banks = [phys(n1 + L1 * k2, L1) % 32 for k2 in range(L2)]
        assert len(set(banks)) == L2, (N, n1, banks)


@pytest.mark.parametrize("N", sorted(SPLITS))
def test_four_step_order_and_pair_separation_give_the_real_fft(N):
    L1, L2 = SPLITS[N]
    rng = np.random.default_rng(N)
    xa, xb = rng.standard_normal(N), rng.standard_normal(N)
    z = (xa + 1j * xb).astype(np.complex128)
    buf = z.copy()
    n1 = np.arange(L1)
    for a in range(L1):  # pass 1: L2-point FFTs over n2, twiddle W_N^(n1 k2), in place at n1 + L1 k2
        col = np.fft.fft(buf[a + L1 * np.arange(L2)])
        buf[a + L1 * np.arange(L2)] = col * np.exp(-2j * np.pi * a * np.arange(L2) / N)
    Z = np.empty(N, dtype=np.complex128)
    for k2 in range(L2):  # pass 2: L1-point FFTs over n1, output k = k2 + L2 k1
        Z[k2 + L2 * n1] = np.fft.fft(buf[n1 + L1 * k2])
    np.testing.assert_allclose(Z, np.fft.fft(z), rtol=0, atol=1e-9 * np.abs(Z).max())
    k = np.arange(N // 2 + 1)
    Zm = np.conj(Z[(N - k) % N])
    np.testing.assert_allclose((Z[k] + Zm) / 2, np.fft.rfft(xa), rtol=0, atol=1e-9 * N)
    np.testing.assert_allclose((Z[k] - Zm) / 2j, np.fft.rfft(xb), rtol=0, atol=1e-9 * N)
