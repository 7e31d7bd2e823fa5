"""FP32 storage against the FP64 path on one lattice: the error report of
the FP32 form.

Both precisions evolve the same initial state side by side on the device
(the reference's step(), g2functions.cpp:234-271, with GWs).  After every
step both handles' stage-0 scalars -- the columns of the reference's
slices_time.dat, t, a, adot, edkin, edpot, edgrad, edrho (g2output.cpp:
174-179) -- are read; every `spectra_every` steps both handles' specOut
tables (g2spectra.cpp:23-234) are taken.  The report holds

* the largest relative difference FP32 - FP64 of a, adot, kin, pot, grad and
  rho over the run (grad, a sum of terms that cancel, relative to rho as
  well as to itself);
* the energy-conservation error of each run (gabe_b200.energy: the
  continuity residual eps(t)) and their largest difference;
* the largest per-bin relative difference of the spectrum columns above
  each column's FFT noise floor (1e-9 of the column's largest value), over
  every output time: P_phi, D2_phi, P_chi, D2_chi and, with GWs, P_gw,
  Omega_gw.

dt must lie inside RK2's stability region for the lattice's top modes
(theta = dt sqrt(12) / dx well below 1; the reference's default dt = dx/80
gives 0.043): the midpoint scheme amplifies a mode of frequency omega by
sqrt(1 + (omega dt)^4 / 4) per step, so a run with theta near 1 measures
the growth of its UV modes, not the storage precision."""
from __future__ import annotations

import numpy as np

from . import FP32, FP64, Lattice
from .energy import continuity_residual

SCALARS = ("a", "adot", "kin", "pot", "grad", "rho")
FIELD_COLS = (1, 2, 3, 4)  # P_phi, D2_phi, P_chi, D2_chi of the specOut table
GW_COLS = (5, 6)            # P_gw, Omega_gw


def stability_theta(N: int, L: float, dt: float) -> float:
    """dt sqrt(12) / dx: omega_max dt of the 7-point Laplacian's top mode at a = 1."""
    return dt * np.sqrt(12.0) / (L / N)


def spectra_rel_diff(got: np.ndarray, want: np.ndarray, cols) -> float:
    """Largest |got - want| / |want| per bin of the given columns, with each
    column's FFT noise floor (1e-9 of its largest value) subtracted."""
    w, g = want[:, cols], got[:, cols]
    floor = 1e-9 * np.abs(w).max(axis=0, keepdims=True)
    return float(((np.abs(g - w) - floor).clip(min=0) / np.abs(w).clip(min=1e-300)).max())


def compare_precisions(field0, dfield0, a0: float, adot0: float, *, N: int, steps: int, dt: float,
                       L: float = 20.0, gws: bool = True, spectra_every: int = 0, device: int = 0,
                       flags32: int = 0, flags64: int = 0) -> dict:
    """Evolves field0/dfield0 ([2][N][N][N], FP64) in FP64 and in FP32
    storage for `steps` steps and returns the report described above."""
    lat64 = Lattice(N, L=L, dt=dt, gws=gws, precision=FP64, device=device, flags=flags64)
    lat32 = None
    try:
        lat32 = Lattice(N, L=L, dt=dt, gws=gws, precision=FP32, device=device, flags=flags32)
        for lat in (lat64, lat32):
            lat.upload_state(field0, dfield0, a0=a0, adot0=adot0)
        rows = {64: [], 32: []}
        spec = {64: [], 32: []}
        every = spectra_every if spectra_every > 0 else steps
        for n in range(steps + 1):
            if n:
                lat64.step(1)
                lat32.step(1)
            for key, lat in ((64, lat64), (32, lat32)):
                e = lat.calc_energy()
                rows[key].append((n * dt, e["a"], e["adot"], e["kin"], e["pot"], e["grad"], e["rho"]))
            if n and (n % every == 0 or n == steps):
                spec[64].append(lat64.spec_out())
                spec[32].append(lat32.spec_out())
    finally:
        lat64.close()
        if lat32 is not None:
            lat32.close()
    r64, r32 = np.array(rows[64]), np.array(rows[32])
    rel = {}
    for c, name in enumerate(SCALARS, start=1):
        rel[name] = float(np.max(np.abs(r32[:, c] - r64[:, c]) / np.abs(r64[:, c])))
    rel["grad_over_rho"] = float(np.max(np.abs(r32[:, 5] - r64[:, 5]) / np.abs(r64[:, 6])))
    eps64 = continuity_residual(*(r64[:, c] for c in range(7)))
    eps32 = continuity_residual(*(r32[:, c] for c in range(7)))
    spectra = {"fields": max(spectra_rel_diff(s32, s64, FIELD_COLS) for s32, s64 in zip(spec[32], spec[64]))}
    if gws:
        spectra["gw"] = max(spectra_rel_diff(s32, s64, GW_COLS) for s32, s64 in zip(spec[32], spec[64]))
    finite = bool(np.all(np.isfinite(r32)) and np.all(np.isfinite(r64)))
    return {
        "N": N, "steps": steps, "dt": dt, "L": L, "gws": gws, "t_end": steps * dt,
        "theta": stability_theta(N, L, dt),
        "spectra_times": len(spec[64]),
        "scalars_max_rel_diff": rel,
        "eps_fp64": float(eps64[-1]), "eps_fp32": float(eps32[-1]),
        "eps_max_abs_diff": float(np.max(np.abs(eps32 - eps64))),
        "spectra_max_rel_diff": spectra,
        "finite": finite,
        "max_rel_err": max(*rel.values(), *spectra.values()),
    }
