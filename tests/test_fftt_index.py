"""Index arithmetic of the transposed three-pass transform
(gabe_b200/csrc/fftt.cuh), restated on the CPU with numpy's FFTs in place of
the in-kernel ones.

* pass 1 (rowt_kernel): tile t of 16 rows (q N + i = t / (N/16), rows
  j0 = 16 (t % (N/16)) ..) of S[q][i][j][N+2]; task (p = t % 8, kz = t / 8)
  writes rows j0 + 2p, j0 + 2p + 1 at kz to T1 at ((q N + i) NH + kz) N +
  j0 + 2p as one 16-byte pair;
* pass 2 (colt_kernel): tile t = (q NH + kz) (N/16) + ib reads the 16 lines
  (q, i = 16 ib + w, kz) at ((q N + i) NH + kz) N, N values each, and writes
  output ky of line w to T2 at (q NH + kz) N N + ky N + 16 ib + w;
* pass 3 (ikspace_kernel): task = kz N + ky reads the ten lines
  q M + task N (M = NH N N) and the amplitudes p M + task N, and its FFT of
  line q along i is the 3-D r2c of source q at (kx, ky, kz);
* the amplitudes live at g_index(i, j, kz) = (kz N + j) N + i.

Every access stays inside its buffer, every output element is written
exactly once, and the chain equals numpy's rfftn of every source array."""
import numpy as np
import pytest


def _chain(N, ncomp, S):
    NH, RP, R, W = N // 2 + 1, N + 2, 16, 16
    M = NH * N * N
    T1 = np.full(ncomp * M, np.nan + 0j, dtype=np.complex128)
    written = np.zeros(ncomp * M, dtype=np.int32)
    flat = S.reshape(-1)
    # pass 1
    ntiles = ncomp * N * N // R
    assert ntiles * R * RP == flat.size
    for tile in range(ntiles):
        rows = flat[tile * R * RP:(tile + 1) * R * RP].reshape(R, RP)[:, :N]
        X = np.fft.rfft(rows, axis=1)  # [16][NH]
        qi, j0 = tile // (N // R), (tile % (N // R)) * R
        for t in range(8 * NH):  # the kernel's task order: p = t % 8, kz = t // 8
            p, kz = t % 8, t // 8
            off = qi * NH * N + kz * N + j0 + 2 * p
            assert off % 2 == 0 and 0 <= off and off + 1 < ncomp * M  # 16-byte aligned pair
            T1[off:off + 2] = X[2 * p:2 * p + 2, kz]
            written[off:off + 2] += 1
    assert np.all(written == 1)
    # pass 2
    T2 = np.full(ncomp * M, np.nan + 0j, dtype=np.complex128)
    written[:] = 0
    ntiles = ncomp * NH * (N // W)
    for tile in range(ntiles):
        ib, qk = tile % (N // W), tile // (N // W)
        kz, q = qk % NH, qk // NH
        lines = []
        for w in range(W):
            src = ((q * N + ib * W + w) * NH + kz) * N
            assert src >= 0 and src + N <= ncomp * M and src % N == 0
            lines.append(T1[src:src + N])
        Y = np.fft.fft(np.array(lines), axis=1)  # [w][ky]
        ky = np.arange(N)[None, :]
        w = np.arange(W)[:, None]
        off = qk * N * N + ib * W + ky * N + w
        assert off.min() >= 0 and off.max() < ncomp * M
        T2[off] = Y
        written[off] += 1
    assert np.all(written == 1)
    # pass 3: the FFT along i of each task's lines
    out = np.zeros((ncomp, N, N, NH), dtype=np.complex128)  # [q][kx][ky][kz]
    for task in range(NH * N):
        kz, ky = task // N, task % N
        for q in range(ncomp):
            src = q * M + task * N
            assert src + N <= ncomp * M
            out[q, :, ky, kz] = np.fft.fft(T2[src:src + N])
        for p in range(4):
            assert p * M + task * N + N <= 4 * M
    return out


@pytest.mark.parametrize("N", [64, 128])
def test_transposed_chain_is_the_3d_r2c(N):
    ncomp = 10 if N == 64 else 2
    rng = np.random.default_rng(N)
    S = np.zeros((ncomp, N, N, N + 2))
    S[..., :N] = rng.standard_normal((ncomp, N, N, N))
    out = _chain(N, ncomp, S)
    want = np.fft.rfftn(S[..., :N], axes=(1, 2, 3))
    assert np.abs(out - want).max() <= 1e-9 * np.abs(want).max()


def test_amplitude_index_is_a_bijection():
    N = 32
    NH = N // 2 + 1
    i, j, kz = np.meshgrid(np.arange(N), np.arange(N), np.arange(NH), indexing="ij")
    gi = (kz * N + j) * N + i
    assert sorted(gi.reshape(-1).tolist()) == list(range(N * N * NH))
