"""numpy restatement of the CUDA k-space update (gabe_b200/csrc/kspace.cuh),
used by the CPU tests to check its projection formula against the
reference's explicit one (g2evolutionpert.cpp:203-310)."""
import numpy as np


def tt_project(k, S):
    """k: unit vector (3,), S: 6 components 11,12,13,22,23,33 (real or
    complex).  Returns Lambda(k) S = P S P - 1/2 P tr(P S)."""
    kx, ky, kz = k
    S11, S12, S13, S22, S23, S33 = S
    u1 = S11 * kx + S12 * ky + S13 * kz
    u2 = S12 * kx + S22 * ky + S23 * kz
    u3 = S13 * kx + S23 * ky + S33 * kz
    s = kx * u1 + ky * u2 + kz * u3
    g = 0.5 * ((S11 + S22 + S33) - s)
    return np.array([
        S11 - 2 * kx * u1 + s * kx * kx - g * (1 - kx * kx),
        S12 - kx * u2 - u1 * ky + (s + g) * kx * ky,
        S13 - kx * u3 - u1 * kz + (s + g) * kx * kz,
        S22 - 2 * ky * u2 + s * ky * ky - g * (1 - ky * ky),
        S23 - ky * u3 - u2 * kz + (s + g) * ky * kz,
        S33 - 2 * kz * u3 + s * kz * kz - g * (1 - kz * kz),
    ])


def sym(S):
    S11, S12, S13, S22, S23, S33 = S
    return np.array([[S11, S12, S13], [S12, S22, S23], [S13, S23, S33]])


def pol_tensors(n):
    """numpy restatement of pol_tensors() in gabe_b200/csrc/kspace.cuh."""
    k = np.asarray(n, dtype=float) / np.linalg.norm(n)
    r = int(np.argmin(np.abs(k))) if len(set(np.abs(k))) == 3 else (
        0 if abs(k[0]) <= abs(k[1]) and abs(k[0]) <= abs(k[2]) else (1 if abs(k[1]) <= abs(k[2]) else 2))
    a = np.zeros(3)
    a[r] = 1.0
    e1 = a - k[r] * k
    e1 /= np.linalg.norm(e1)
    e2 = np.cross(k, e1)
    ep = np.outer(e1, e1) - np.outer(e2, e2)
    ex = np.outer(e1, e2) + np.outer(e2, e1)
    return ep, ex
