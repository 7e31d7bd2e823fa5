"""CPU oracle of the spectra emulator's MLP (test infrastructure only: the
product path is gabe_b200/csrc/mlp.cu and never calls this module).

The emulator has no counterpart in the reference, so this restates the
network's own definition (include/gabe_mlp.h): layers n_in -> width x depth
(SiLU) -> n_out (linear), flat FP32 parameters W_l [K][N] then b_l [N], loss
= mean of (y - t)^2 over finite targets, AdamW with bias correction.

Three arithmetic modes:
  "fp64"  everything in float64: the analytic reference for gradient checks
          (itself pinned by finite differences and by torch.autograd).
  "fp32"  float32 products and activations (GABE_MLP_FP32_ACT).
  "bf16"  float32 products; pre-activations Z and activations H rounded to
          bfloat16 (round to nearest even) where the device stores them; the
          SiLU is taken of the unrounded FP32 pre-activation, its derivative
          of the stored (rounded) one.  The forward products of every layer
          after the first take the weights rounded to bfloat16 (the device
          runs them on tensor cores from BF16 weight copies); the first layer
          and the backward products use the FP32 weights.
"""
from __future__ import annotations

import math

import numpy as np


def layout(n_in=3, width=256, depth=4, n_out=192):
    """[(K, N, offW, offb)] per layer and the parameter count."""
    out, P = [], 0
    for l in range(depth + 1):
        K = n_in if l == 0 else width
        N = n_out if l == depth else width
        offW = P
        P += K * N
        offb = P
        P += N
        out.append((K, N, offW, offb))
    return out, P


def _splitmix(state):
    M = (1 << 64) - 1
    state = (state + 0x9E3779B97F4A7C15) & M
    z = state
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M
    return state, z ^ (z >> 31)


def init_params(seed=1, n_in=3, width=256, depth=4, n_out=192):
    """Glorot-uniform weights U(-a, a), a = sqrt(6/(K+N)), from a splitmix64
    stream (53-bit uniforms), zero biases -- the device's initialisation."""
    lay, P = layout(n_in, width, depth, n_out)
    p = np.zeros(P, dtype=np.float32)
    s = seed & ((1 << 64) - 1)
    for K, N, offW, _ in lay:
        a = math.sqrt(6.0 / (K + N))
        vals = np.empty(K * N, dtype=np.float64)
        for i in range(K * N):
            s, z = _splitmix(s)
            vals[i] = (2.0 * ((z >> 11) * (1.0 / 9007199254740992.0)) - 1.0) * a
        p[offW:offW + K * N] = vals.astype(np.float32)
    return p


def bf16_round(x):
    """float32 -> nearest bfloat16 (ties to even) -> float32."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32)


def _sig(z):
    return 1.0 / (1.0 + np.exp(-z))


def _silu(z):
    return z * _sig(z)


def _dsilu(z):
    s = _sig(z)
    return s * (1.0 + z * (1.0 - s))


def _unpack(params, lay, dt):
    Ws, bs = [], []
    for K, N, offW, offb in lay:
        Ws.append(params[offW:offW + K * N].astype(dt).reshape(K, N))
        bs.append(params[offb:offb + N].astype(dt))
    return Ws, bs


def forward(params, x, shape=(3, 256, 4, 192), mode="fp64"):
    """y and the stored (Z, H) per hidden layer."""
    lay, _ = layout(*shape)
    dt = np.float64 if mode == "fp64" else np.float32
    Ws, bs = _unpack(np.asarray(params), lay, dt)
    with np.errstate(over="ignore"):
        h = np.asarray(x, dtype=dt)
        Zs, Hs = [], []
        for l in range(len(lay)):
            W = bf16_round(Ws[l]) if (mode == "bf16" and l > 0) else Ws[l]
            z = (h @ W + bs[l]).astype(dt)
            if l + 1 == len(lay):
                return z, Zs, Hs
            a = _silu(z).astype(dt)
            if mode == "bf16":
                zs, a = bf16_round(z), bf16_round(a)
            else:
                zs = z
            Zs.append(zs)
            Hs.append(a)
            h = a


def loss_grad(params, x, t, shape=(3, 256, 4, 192), mode="fp64"):
    """(loss, flat gradient) of the masked mean squared error."""
    lay, P = layout(*shape)
    dt = np.float64 if mode == "fp64" else np.float32
    Ws, _ = _unpack(np.asarray(params), lay, dt)
    x = np.asarray(x, dtype=dt)
    t = np.asarray(t, dtype=np.float64)
    y, Zs, Hs = forward(params, x, shape, mode)
    mask = np.isfinite(t)
    cnt = mask.sum()
    d = np.where(mask, y.astype(np.float64) - np.where(mask, t, 0.0), 0.0)
    loss = float((d * d).sum() / cnt) if cnt else 0.0
    delta = (2.0 * d).astype(dt)
    g = np.zeros(P, dtype=np.float64)
    with np.errstate(over="ignore"):
        for l in range(len(lay) - 1, -1, -1):
            K, N, offW, offb = lay[l]
            inp = x if l == 0 else Hs[l - 1]
            g[offW:offW + K * N] = (inp.T @ delta).reshape(-1)
            g[offb:offb + N] = delta.sum(axis=0)
            if l:
                delta = ((delta @ Ws[l].T) * _dsilu(Zs[l - 1])).astype(dt)
    if cnt:
        g /= cnt
    return loss, g


def adamw_step(params, grad, m, v, step, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8, wd=0.0):
    """One AdamW step in float32 (step counts from 1), returns new
    (params, m, v)."""
    f = np.float32
    p = np.asarray(params, dtype=f).copy()
    g = np.asarray(grad, dtype=f)
    bc1 = f(1.0 - b1 ** step)
    bc2 = f(1.0 - b2 ** step)
    p = p - f(lr) * f(wd) * p
    m = f(b1) * m + (f(1) - f(b1)) * g
    v = f(b2) * v + (f(1) - f(b2)) * g * g
    p = p - f(lr) * (m / bc1) / (np.sqrt(v / bc2) + f(eps))
    return p.astype(f), m.astype(f), v.astype(f)
