"""Initial conditions with the reference's convention (g2init.cpp:68-189,
g2model.cpp:113-144), vectorised.

The reference draws its Gaussian random field with libc rand() inside an
OpenMP loop, so its realisation depends on thread scheduling; this module
draws the same distribution from a seeded torch generator instead:

  * homogeneous values f0, df0; a0 = 1, adot0 = adf of the homogeneous energy
    (initexpansion, g2init.cpp:26-29 -- adot0 is not recomputed after the
    fluctuations are added, exactly as in the reference);
  * per field, in order phi then chi: m_eff^2 from the current fields
    (effMass), omega_k = sqrt(k^2 + m_eff^2), two independent
    (Rayleigh amplitude B sqrt(-ln u / (2 omega L^3)), uniform phase)
    draws R1, R2 per half-spectrum mode; f_k = (R1 + R2)/sqrt 2,
    fdot_k = i-rotated (R2 - R1) omega/sqrt 2 - H0 f_k; zero mode 0;
  * unnormalised c2r added to the homogeneous values.

For bit-exact reproduction of a reference run use the reference's own dump
(or the oracle's restatement of rand()); this generator is for workloads
that need the same statistics at sizes where a serial rand() loop is slow.
"""
from __future__ import annotations

import math

import torch

from . import MODEL_LPHI4, MODEL_QUADRATIC


def _dv_m2(model: int, mc, f_phi: torch.Tensor, f_chi: torch.Tensor, fld: int) -> float:
    if model == MODEL_QUADRATIC:
        coup = mc[1] / mc[0] / mc[0]  # gsq/mphi/mphi
        return float((1.0 + coup * f_chi * f_chi).mean()) if fld == 0 else float((coup * f_phi * f_phi).mean())
    lam, g = mc
    return float((3.0 * lam * f_phi * f_phi + g * f_chi * f_chi).mean()) if fld == 0 else float((g * f_phi * f_phi).mean())


def _potential(model: int, mc, p: float, c: float) -> float:
    if model == MODEL_QUADRATIC:
        coup = mc[1] / mc[0] / mc[0]
        return 0.5 * p * p + 0.5 * coup * p * p * c * c
    lam, g = mc
    return 0.25 * lam * p ** 4 + 0.5 * g * p * p * c * c


def random_state(N: int, *, L: float = 20.0, seed: int = 44463132, model: int = MODEL_LPHI4, model_c=None,
                 f0=(0.342, 0.0), df0=(0.0, 0.0), rescale_B: float | None = None, amplitude: float = 1.0,
                 spec_cut_off: float | None = None, spec_smooth: float = 0.5, full_rand: bool = True,
                 device: str | torch.device = "cpu"):
    """Returns (field0, dfield0, a0, adot0): float64 tensors [2][N][N][N] on
    `device` and the two scalars.  `amplitude` multiplies every fluctuation
    amplitude (the ensemble's amplitude multiplier).  The reference's
    initial-spectrum knobs (g2parameters.h:72-74, g2init.cpp:117-165):
    `spec_cut_off` (with `spec_smooth`) multiplies every mode's amplitude by
    (1 - tanh(spec_smooth (|n| - N spec_cut_off)))/2; `full_rand=False`
    (field_full_rand 0, which the reference only defines with the cut-off)
    replaces the random draws by the deterministic real amplitude
    sqrt(1/(2 omega_k L^3)) and fdot_k = -H0 f_k."""
    if not full_rand and spec_cut_off is None:
        raise ValueError("full_rand=False needs spec_cut_off (the reference's field_full_rand 0 uses it)")
    if model_c is None:
        model_c = (1.0 / 0.342 ** 2, 100.0 / 0.342 ** 2) if model == MODEL_LPHI4 else (1e-6, 2.5e-7)
    if rescale_B is None:
        rescale_B = math.sqrt(9e-14) * 0.342 if model == MODEL_LPHI4 else model_c[0]
    dev = torch.device(device)
    gen = torch.Generator(device=dev)
    gen.manual_seed(int(seed))
    nz = N // 2 + 1
    f = torch.empty((2, N, N, N), dtype=torch.float64, device=dev)
    d = torch.empty((2, N, N, N), dtype=torch.float64, device=dev)
    for q in range(2):
        f[q].fill_(f0[q])
        d[q].fill_(df0[q])
    # homogeneous energy -> H0 and adot0 (kinetic + potential; gradient is 0)
    rho_h = 0.5 * (df0[0] ** 2 + df0[1] ** 2) + _potential(model, model_c, f0[0], f0[1])
    H0 = math.sqrt(8.0 * math.pi / 3.0 * rho_h)
    a0, adot0 = 1.0, H0 * 1.0
    i = torch.arange(N, device=dev, dtype=torch.float64)
    i2 = torch.where(i < N // 2 + 1, i * i, (N - i) * (N - i))
    k2 = torch.arange(nz, device=dev, dtype=torch.float64) ** 2
    dk2 = 4.0 * math.pi * math.pi / L / L
    n2 = i2[:, None, None] + i2[None, :, None] + k2[None, None, :]
    L3 = L * L * L
    cut = None
    if spec_cut_off is not None:
        cut = (1.0 - torch.tanh(spec_smooth * (torch.sqrt(n2) - N * spec_cut_off))) / 2.0
    for q in range(2):
        m2 = _dv_m2(model, model_c, f[0], f[1], q)
        wk = torch.sqrt(dk2 * n2 + m2)
        if not full_rand:
            amp = amplitude * rescale_B * torch.sqrt(1.0 / (2.0 * wk * L3)) * cut
            fk = torch.complex(amp, torch.zeros_like(amp))
            fd = torch.complex(-H0 * amp, torch.zeros_like(amp))
            fk[0, 0, 0] = 0
            fd[0, 0, 0] = 0
            scale = float(N) ** 3  # FFTW's c2r is unnormalised
            f[q] += torch.fft.irfftn(fk, s=(N, N, N)) * scale
            d[q] += torch.fft.irfftn(fd, s=(N, N, N)) * scale
            del fk, fd, amp, wk
            continue
        draws = []
        for _ in range(2):
            u = 1.0 - torch.rand((N, N, nz), generator=gen, device=dev, dtype=torch.float64)
            th = 2.0 * math.pi * torch.rand((N, N, nz), generator=gen, device=dev, dtype=torch.float64)
            r = amplitude * rescale_B * torch.sqrt(-torch.log(u) / (2.0 * wk * L3))
            if cut is not None:
                r = r * cut
            draws.append((r * torch.cos(th), r * torch.sin(th)))
            del u, th, r
        (r1, i1), (r2, i2_) = draws
        s2 = math.sqrt(2.0)
        fk = torch.complex((r1 + r2) / s2, (i1 + i2_) / s2)
        fd = torch.complex((i2_ - i1) * wk / s2 - H0 * fk.real, (r1 - r2) * wk / s2 - H0 * fk.imag)
        fk[0, 0, 0] = 0
        fd[0, 0, 0] = 0
        del draws, r1, i1, r2, i2_, wk
        scale = float(N) ** 3  # FFTW's c2r is unnormalised
        f[q] += torch.fft.irfftn(fk, s=(N, N, N)) * scale
        d[q] += torch.fft.irfftn(fd, s=(N, N, N)) * scale
        del fk, fd
    return f, d, a0, adot0
