"""Energy-conservation error of a run, from its time series of scalars.

The reference writes one row per output time to slices_time.dat:
t, a, adot, adot/a, edkin, edpot, edgrad, edrho (g2output.cpp:174-179).  Its
step() sets adot from the Friedmann constraint at every stage
(g2functions.cpp:250-252, 268-270), so that constraint holds by construction
and measures nothing.  The continuity equation of the homogeneous background,
d rho / dt = -3 H (rho + p), with H = adot/a and the pressure of the
reference's energy components (avgKin, avgPot, avgGrad, g2functions.cpp:
124-174) p = kin - grad/3 - pot, does:

    eps(t) = | rho(t) - rho(t0) + int_{t0}^{t} 3 H (rho + p) dt' | / rho(t),

the integral taken by the trapezoid rule over the recorded times.  For RK2
with a fixed step eps falls as dt^2 (checked against the oracle)."""
import numpy as np

# columns of slices_time.dat, in order
TIME_COLUMNS = ("t", "a", "adot", "hubble", "kin", "pot", "grad", "rho")


def pressure(kin, pot, grad):
    """p = kin - grad/3 - pot of the volume-averaged energy components."""
    return np.asarray(kin) - np.asarray(grad) / 3.0 - np.asarray(pot)


def continuity_residual(t, a, adot, kin, pot, grad, rho) -> np.ndarray:
    """eps(t) at every recorded time (eps(t0) = 0); arrays of equal length,
    times increasing."""
    t, a, adot, rho = (np.asarray(x, dtype=np.float64) for x in (t, a, adot, rho))
    if t.ndim != 1 or t.size < 1 or any(np.shape(x) != t.shape for x in (a, adot, kin, pot, grad, rho)):
        raise ValueError("continuity_residual needs 1-D series of equal length")
    if t.size > 1 and not np.all(np.diff(t) > 0):
        raise ValueError("times must increase")
    f = 3.0 * (adot / a) * (rho + pressure(kin, pot, grad))
    integral = np.concatenate([[0.0], np.cumsum(0.5 * (f[1:] + f[:-1]) * np.diff(t))])
    return np.abs(rho - rho[0] + integral) / rho


def residual_from_rows(rows) -> np.ndarray:
    """eps(t) from rows in slices_time.dat's column order."""
    r = np.asarray(rows, dtype=np.float64)
    if r.ndim != 2 or r.shape[1] != len(TIME_COLUMNS):
        raise ValueError(f"rows need the {len(TIME_COLUMNS)} columns {TIME_COLUMNS}")
    t, a, adot, _, kin, pot, grad, rho = r.T
    return continuity_residual(t, a, adot, kin, pot, grad, rho)


def main(argv=None) -> dict:
    """python -m gabe_b200.energy <slices_time.dat>: prints, as one JSON
    line, the number of rows, the last time, eps at the last time and the
    largest eps of the run."""
    import argparse
    import json

    ap = argparse.ArgumentParser(description="energy-conservation error of a run from its slices_time.dat")
    ap.add_argument("path", help="slices_time.dat written by the reference or by the drop-in")
    args = ap.parse_args(argv)
    rows = np.loadtxt(args.path, ndmin=2)
    eps = residual_from_rows(rows)
    out = {"rows": int(rows.shape[0]), "t_end": float(rows[-1, 0]), "eps_end": float(eps[-1]),
           "eps_max": float(eps.max())}
    print(json.dumps(out))
    return out


if __name__ == "__main__":
    main()
