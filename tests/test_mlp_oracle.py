"""The MLP oracle on the CPU, pinned three ways: its FP64 gradient against
central finite differences and against torch.autograd, its bfloat16
rounding against torch's, and its AdamW step against torch.optim.AdamW."""
import numpy as np
import torch

from oracle import mlp_oracle as mo

SMALL = (3, 64, 2, 64)


def _data(n, shape, seed=0, nan_frac=0.2):
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1, 1, size=(n, shape[0]))
    t = rng.normal(size=(n, shape[3]))
    t[rng.uniform(size=t.shape) < nan_frac] = np.nan
    return x, t


def test_default_layout_has_247744_parameters():
    _, P = mo.layout()
    assert P == 247744


def test_fp64_gradient_matches_finite_differences():
    p = mo.init_params(5, *SMALL).astype(np.float64)
    p += 0.05 * np.random.default_rng(1).normal(size=p.shape)  # non-zero biases
    x, t = _data(16, SMALL)
    loss, g = mo.loss_grad(p, x, t, SMALL, "fp64")
    rng = np.random.default_rng(2)
    idx = rng.choice(len(p), size=60, replace=False)
    h = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (mo.loss_grad(pp, x, t, SMALL, "fp64")[0] - mo.loss_grad(pm, x, t, SMALL, "fp64")[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-7 + 1e-5 * abs(g[i]), (i, fd, g[i])


def test_fp64_gradient_matches_autograd():
    p = mo.init_params(9, *SMALL).astype(np.float64)
    p += 0.05 * np.random.default_rng(3).normal(size=p.shape)
    x, t = _data(32, SMALL, seed=4)
    loss, g = mo.loss_grad(p, x, t, SMALL, "fp64")
    lay, _ = mo.layout(*SMALL)
    pt = torch.tensor(p, requires_grad=True)
    h = torch.tensor(x)
    for l, (K, N, oW, ob) in enumerate(lay):
        z = h @ pt[oW:oW + K * N].view(K, N) + pt[ob:ob + N]
        h = z if l + 1 == len(lay) else torch.nn.functional.silu(z)
    tt = torch.tensor(t)
    mask = torch.isfinite(tt)
    lt = ((h - torch.nan_to_num(tt))[mask] ** 2).mean()
    lt.backward()
    assert abs(lt.item() - loss) <= 1e-12 * abs(loss)
    np.testing.assert_allclose(g, pt.grad.numpy(), rtol=1e-9, atol=1e-14)


def test_bf16_rounding_matches_torch():
    rng = np.random.default_rng(6)
    x = np.concatenate([rng.normal(size=10000).astype(np.float32) * 10.0 ** rng.integers(-20, 20, size=10000),
                        np.array([0.0, -0.0, 1.0, 1.00390625, 1.01171875, 65504.0], dtype=np.float32)])
    want = torch.tensor(x).to(torch.bfloat16).to(torch.float32).numpy()
    np.testing.assert_array_equal(mo.bf16_round(x), want)


def test_adamw_step_matches_torch():
    rng = np.random.default_rng(7)
    p0 = rng.normal(size=500).astype(np.float32)
    grads = [rng.normal(size=500).astype(np.float32) for _ in range(3)]
    pt = torch.tensor(p0.copy(), requires_grad=True)
    opt = torch.optim.AdamW([pt], lr=1e-2, betas=(0.9, 0.999), eps=1e-8, weight_decay=0.01)
    p, m, v = p0.copy(), np.zeros(500, np.float32), np.zeros(500, np.float32)
    for s, g in enumerate(grads, 1):
        pt.grad = torch.tensor(g)
        opt.step()
        p, m, v = mo.adamw_step(p, g, m, v, s, lr=1e-2, wd=0.01)
    np.testing.assert_allclose(p, pt.detach().numpy(), rtol=2e-6, atol=2e-7)


def test_bf16_forward_stays_close_to_fp64():
    p = mo.init_params(3)
    x, _ = _data(64, (3, 256, 4, 192), seed=8)
    y64, _, _ = mo.forward(p, x, mode="fp64")
    y16, _, _ = mo.forward(p, x, mode="bf16")
    assert np.linalg.norm(y16 - y64) / np.linalg.norm(y64) < 2e-2
