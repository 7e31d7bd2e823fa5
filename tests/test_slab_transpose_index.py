"""Index arithmetic of the slab transpose (gabe_b200/csrc/slabgw.cuh and the
slab forms of fft3d.cuh col_fft_kernel), restated on the CPU for every rank
of 1-5 ranks on small lattices.

* pack (slab_gw_pack_kernel): row (q, il, ky) of a rank's 2-D transforms goes
  to the block of the rank that owns ky, at
  ncomp nloc nz p0(r') + ((q nloc + il) n(r') + ky - p0(r')) nz;
* the all-to-all moves block r' of every sender to r', placed at the
  sender's offset ncomp m nz p0(r);
* unpack (slab_gw_unpack_kernel) reads row (q, i, y) of T at
  ncomp m nz p0(r) + ((q n(r) + i - p0(r)) m + y) nz, r the owner of plane i;
* the FP32 pass along j writes output index ky of line b = q nloc + il at
  (b1 p0(r') + ky - p0(r') + b n(r')) nz  (scatter, b1 = ncomp nloc), and the
  pass along i reads value i of line (q, y) at
  (ncomp p0(r) + i - p0(r) + q n(r)) m nz + y nz  (gather).

pack -> all-to-all -> unpack must rebuild the global T[q][i][ky][kz] columns
of every rank, the scatter and gather offsets must equal the pack and unpack
ones, and every access must stay inside its buffer."""
import numpy as np
import pytest

from gabe_b200.slab import split_planes


def _owner(parts, x):
    for r, (p0, n) in enumerate(parts):
        if p0 <= x < p0 + n:
            return r
    raise AssertionError(x)


@pytest.mark.parametrize("N", [16, 32, 48, 64])
@pytest.mark.parametrize("W", [1, 2, 3, 4, 5])
@pytest.mark.parametrize("ncomp", [2, 10])
def test_pack_alltoall_unpack_and_the_fused_passes(N, W, ncomp):
    nz = N // 2 + 1
    parts = split_planes(N, W)
    rng = np.random.default_rng(N * 100 + W * 10 + ncomp)
    full = rng.standard_normal((ncomp, N, N, nz))  # [q][i][ky][kz] after the 2-D transforms
    sends = []
    for r, (p0, nloc) in enumerate(parts):
        rows = full[:, p0:p0 + nloc].reshape(-1, nz)  # row index (q nloc + il) N + ky
        send = np.full(ncomp * nloc * N * nz, np.nan)
        b1 = ncomp * nloc
        for row in range(ncomp * nloc * N):
            ky, b = row % N, row // N
            rr = _owner(parts, ky)
            q0, m = parts[rr]
            dst = ncomp * nloc * nz * q0 + (b * m + ky - q0) * nz
            scatter = (b1 * q0 + ky - q0 + b * m) * nz  # the pass along j, output index ky of line b
            assert dst == scatter
            assert 0 <= dst and dst + nz <= send.size
            send[dst:dst + nz] = rows[row]
        assert not np.isnan(send).any()  # every place written once
        sends.append(send)
    for rd, (y0, m) in enumerate(parts):
        recv = np.full(ncomp * N * m * nz, np.nan)
        for r, (p0, nloc) in enumerate(parts):
            so, ro, cnt = ncomp * nloc * nz * y0, ncomp * m * nz * p0, ncomp * nloc * m * nz
            recv[ro:ro + cnt] = sends[r][so:so + cnt]
        assert not np.isnan(recv).any()
        T = np.empty((ncomp, N, m, nz))
        for q in range(ncomp):
            for i in range(N):
                r = _owner(parts, i)
                p0, nr = parts[r]
                for y in range(m):
                    src = ncomp * m * nz * p0 + ((q * nr + i - p0) * m + y) * nz
                    gather = (ncomp * p0 + i - p0 + q * nr) * m * nz + y * nz  # the pass along i, value i of (q, y)
                    assert src == gather
                    assert 0 <= src and src + nz <= recv.size
                    T[q, i, y] = recv[src:src + nz]
        np.testing.assert_array_equal(T, full[:, :, y0:y0 + m])
