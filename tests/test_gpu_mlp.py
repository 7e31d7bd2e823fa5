"""The emulator's MLP kernels (gabe_mlp_*) against the CPU oracle
(oracle/mlp_oracle.py): initialisation, forward, gradient, the AdamW step
and training, in FP32- and BF16-activation modes."""
import numpy as np
import pytest
import torch

from gabe_b200 import emulator as em
from oracle import mlp_oracle as mo

pytestmark = pytest.mark.gpu

SHAPE = (3, 256, 4, 192)


def _batch(n, seed=0, nan_frac=0.3):
    rng = np.random.default_rng(seed)
    x = rng.normal(size=(n, 3)).astype(np.float32)
    t = rng.normal(size=(n, 192)).astype(np.float32)
    t[rng.uniform(size=t.shape) < nan_frac] = np.nan
    return x, t


def _dev(a):
    return torch.tensor(a, device="cuda")


def _perturbed_params(seed):
    p = mo.init_params(seed)
    rng = np.random.default_rng(seed)
    lay, _ = mo.layout()
    for K, N, oW, ob in lay:
        p[ob:ob + N] = (0.1 * rng.normal(size=N)).astype(np.float32)
    return p


def test_device_initialisation_equals_oracle():
    with em.MLP(seed=1234) as net:
        assert net.num_params == 247744
        np.testing.assert_array_equal(net.get_params(), mo.init_params(1234))


@pytest.mark.parametrize("fp32_act", [True, False])
def test_forward_matches_oracle(fp32_act):
    p = _perturbed_params(5)
    x, _ = _batch(1000, seed=1)
    with em.MLP(fp32_act=fp32_act, max_rows=384) as net:  # several chunks
        net.set_params(p)
        y = net.forward(_dev(x)).cpu().numpy()
    y64, _, _ = mo.forward(p, x, mode="fp64")
    if fp32_act:
        assert np.linalg.norm(y - y64) / np.linalg.norm(y64) <= 1e-5
    else:
        ybf, _, _ = mo.forward(p, x, mode="bf16")
        # same roundings as the oracle's emulation up to rare one-ulp flips
        assert np.linalg.norm(y - ybf) / np.linalg.norm(ybf) <= 2e-3
        assert np.linalg.norm(y - y64) / np.linalg.norm(y64) <= 2e-2


@pytest.mark.parametrize("fp32_act", [True, False])
def test_gradient_matches_oracle(fp32_act):
    p = _perturbed_params(7)
    x, t = _batch(512, seed=2)
    with em.MLP(fp32_act=fp32_act) as net:
        net.set_params(p)
        loss, g = net.loss_grad(_dev(x), _dev(t))
    mode = "fp64" if fp32_act else "bf16"
    lref, gref = mo.loss_grad(p, x, t, mode=mode)
    assert abs(loss - lref) <= (1e-6 if fp32_act else 2e-3) * lref
    lay, _ = mo.layout()
    tol = 1e-4 if fp32_act else 2e-2
    for K, N, oW, ob in lay:
        for a, b in ((oW, oW + K * N), (ob, ob + N)):
            rel = np.linalg.norm(g[a:b] - gref[a:b]) / np.linalg.norm(gref[a:b])
            assert rel <= tol, (K, N, a, rel)


def test_adam_step_matches_oracle():
    p = _perturbed_params(11)
    x, t = _batch(256, seed=3)
    perm = torch.arange(256, dtype=torch.int32, device="cuda")
    with em.MLP(fp32_act=True, lr=3e-3, weight_decay=0.01) as net:
        net.set_params(p)
        _, g = net.loss_grad(_dev(x), _dev(t))
        xd, td = _dev(x), _dev(t)
        net.train_batches(xd, td, perm, 256, 1)
        net.sync()
        p1 = net.get_params()
        loss, steps = net.train_loss()
    assert steps == 1
    z = np.zeros_like(p)
    want, _, _ = mo.adamw_step(p, g, z, z.copy(), 1, lr=3e-3, wd=0.01)
    np.testing.assert_allclose(p1, want, rtol=1e-6, atol=1e-7)


def test_graph_and_direct_training_agree_bitwise():
    x, t = _batch(4096, seed=4, nan_frac=0.1)
    out = []
    for graph in (True, False):
        with em.MLP(graph=graph, seed=3) as net:
            net.fit(_dev(x), _dev(t), epochs=2, batch=512, seed=9)
            out.append(net.get_params())
    np.testing.assert_array_equal(out[0], out[1])


def test_training_fits_a_smooth_map():
    rng = np.random.default_rng(5)
    x = rng.uniform(-1, 1, size=(8192, 3)).astype(np.float32)
    k = np.linspace(0, 3, 192)
    t = (np.sin(np.outer(x[:, 0], k) + x[:, 1:2]) * (1 + 0.5 * x[:, 2:3])).astype(np.float32)
    t[:, 150:][x[:, 0] > 0.5] = np.nan  # ragged valid region
    with em.MLP(lr=2e-3, seed=2) as net:
        l0, _ = net.loss_grad(_dev(x[:2048]), _dev(t[:2048]), want_grad=False)
        hist = net.fit(_dev(x), _dev(t), epochs=60, batch=256, seed=1, log_every=10)
        l1, _ = net.loss_grad(_dev(x[:2048]), _dev(t[:2048]), want_grad=False)
    assert hist[-1][1] < hist[0][1]
    assert l1 < 0.02 * l0, (l0, l1)


def test_cosine_schedule_matches_oracle():
    p = _perturbed_params(13)
    x, t = _batch(128, seed=6)
    perm = torch.arange(128, dtype=torch.int32, device="cuda")
    lr0, lr1 = 4e-3, 1e-4
    with em.MLP(fp32_act=True, lr=lr0) as net:
        net.set_params(p)
        net.set_schedule(lr0, lr1, 2)
        xd, td = _dev(x), _dev(t)
        ref, m, v = p.copy(), np.zeros_like(p), np.zeros_like(p)
        for s in range(1, 4):
            net.set_params(ref)
            _, g = net.loss_grad(xd, td)
            net.reset_batches()
            net.train_batches(xd, td, perm, 128, 1)
            net.sync()
            got = net.get_params()
            f = min(s - 1, 2) / 2
            lr = lr1 + 0.5 * (lr0 - lr1) * (1 + np.cos(np.pi * f))
            ref, m, v = mo.adamw_step(ref, g, m, v, s, lr=lr)
            np.testing.assert_allclose(got, ref, rtol=1e-6, atol=1e-7)


def test_forward_forms():
    """BF16 layers 1 .. depth take the tcgen05 kernel (their BF16 weights fit
    in shared memory), or mma.sync on request; FP32 activations and the
    first layer stay on FP32 FMA."""
    with em.MLP(seed=1) as a, em.MLP(seed=1, mma_sync=True) as b, em.MLP(seed=1, fp32_act=True) as c:
        assert [a.forward_form(l) for l in range(5)] == ["fma"] + ["tcgen05"] * 4
        assert [b.forward_form(l) for l in range(5)] == ["fma"] + ["mma.sync"] * 4
        assert [c.forward_form(l) for l in range(5)] == ["fma"] * 5
        with pytest.raises(IndexError):
            a.forward_form(5)


@pytest.mark.parametrize("rows", [1, 127, 128, 129, 300, 4096 + 17])
def test_tcgen05_forward_matches_mma_sync(rows):
    """The tcgen05 forward (TMEM accumulators, 128-row tiles, rows beyond
    the last full tile read as zeros) against the mma.sync forward of the
    same BF16 network: the same BF16 roundings of every operand, FP32 sums
    in another order, so outputs agree to a few BF16 flips of the hidden
    activations."""
    p = _perturbed_params(17)
    rng = np.random.default_rng(rows)
    x = rng.normal(size=(rows, 3)).astype(np.float32)
    ys = []
    for mma_sync in (False, True):
        with em.MLP(seed=1, mma_sync=mma_sync, max_rows=4096) as net:
            net.set_params(p)
            ys.append(net.forward(_dev(x)).cpu().numpy())
            net.sync()
    assert np.all(np.isfinite(ys[0]))
    assert np.linalg.norm(ys[0] - ys[1]) / np.linalg.norm(ys[1]) <= 2e-3
    ybf, _, _ = mo.forward(p, x, mode="bf16")
    assert np.linalg.norm(ys[0] - ybf) / np.linalg.norm(ybf) <= 2e-3


@pytest.mark.parametrize("shape", [(4, 128, 2, 64), (2, 64, 3, 64), (5, 512, 2, 128)])
def test_forward_forms_agree_on_other_shapes(shape):
    """Other widths and depths: layers whose BF16 weights fit in shared
    memory (K, N <= 256) take tcgen05 (K = 64 and 128, N = 64 .. 128 here),
    wider ones the mma.sync kernel; both forms of the same network agree."""
    n_in, width, depth, n_out = shape
    rng = np.random.default_rng(n_in)
    x = rng.normal(size=(1000, n_in)).astype(np.float32)
    ys, forms = [], []
    for mma_sync in (False, True):
        with em.MLP(n_in=n_in, width=width, depth=depth, n_out=n_out, seed=2, mma_sync=mma_sync,
                    max_rows=512) as net:
            forms.append([net.forward_form(l) for l in range(depth + 1)])
            ys.append(net.forward(_dev(x)).cpu().numpy())
            net.sync()
    want = "tcgen05" if width <= 256 else "mma.sync"
    assert forms[0] == ["fma"] + [want] * depth
    assert forms[1] == ["fma"] + ["mma.sync"] * depth
    assert np.all(np.isfinite(ys[0]))
    assert np.linalg.norm(ys[0] - ys[1]) / np.linalg.norm(ys[1]) <= 2e-3


def test_tcgen05_training_matches_mma_sync_training():
    """Training steps (forward with pre-activations kept for the backward)
    through either forward kernel reach nearly the same parameters."""
    x, t = _batch(2048, seed=8, nan_frac=0.1)
    out = []
    for mma_sync in (False, True):
        with em.MLP(seed=3, mma_sync=mma_sync) as net:
            net.fit(_dev(x), _dev(t), epochs=2, batch=256, seed=4)
            net.sync()
            out.append(net.get_params())
    rel = np.linalg.norm(out[0] - out[1]) / np.linalg.norm(out[1])
    assert rel <= 1e-2, rel


def test_tensor_core_forward_outruns_the_fp32_path():
    """With BF16 activations the layers after the first run on tensor cores
    (tcgen05 BF16 x BF16 -> FP32 in TMEM); on a million queries that forward
    must be several times faster than the FP32-activation path, which keeps
    every product on the CUDA-core kernel, and faster than the mma.sync
    form of the same network."""
    with em.MLP(seed=1, max_rows=1 << 20) as tcn, em.MLP(seed=1, fp32_act=True, max_rows=1 << 20) as simt, \
            em.MLP(seed=1, max_rows=1 << 20, mma_sync=True) as legacy:
        q_tc, info_tc = em.queries_per_second(tcn, n=1 << 20, reps=3)
        q_s, info_s = em.queries_per_second(simt, n=1 << 20, reps=3)
        q_l, info_l = em.queries_per_second(legacy, n=1 << 20, reps=3)
    assert q_tc > 3 * q_s, (info_tc, info_s)
    assert q_tc > q_l, (info_tc, info_l)
