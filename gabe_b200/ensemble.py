"""Parameter sweeps on the batched ensemble (gabe_ensemble_*).

* `sample_parameters` draws the uneven ensemble the sweep runs: sizes
  uniform on {32, 48, 64, 96, 128}, g^2/lambda log-uniform on [1, 500],
  amplitude multiplier uniform on [0.5, 2] (it scales the randInit mode
  amplitudes, g2init.cpp:136-143), one seed per lattice -- all from one
  recorded master seed.
* `partition` splits the lattices over ranks balanced by sum N^3 (the work
  per step); `gather_rows` collects per-lattice rows on rank 0 in the
  original order.  Lattices are independent, so this gather is the only
  collective.
* `evolve_and_record` steps an ensemble and reads its log-binned spectra
  every `every` steps: the (parameters, time, log spectra) samples the
  emulator trains on.
"""
from __future__ import annotations

import numpy as np

SIZES = (32, 48, 64, 96, 128)


def sample_parameters(nlat: int, master_seed: int, sizes=SIZES, g_range=(1.0, 500.0), amp_range=(0.5, 2.0)):
    rng = np.random.default_rng(master_seed)
    N = rng.choice(np.asarray(sizes), size=nlat).astype(np.int32)
    g = np.exp(rng.uniform(np.log(g_range[0]), np.log(g_range[1]), size=nlat))
    amp = rng.uniform(amp_range[0], amp_range[1], size=nlat)
    seeds = rng.integers(1, 2 ** 63 - 1, size=nlat, dtype=np.int64).astype(np.uint64)
    return N, g, amp, seeds


def partition(N, world: int) -> list[list[int]]:
    """Longest-processing-time split of lattice indices over `world` ranks,
    weight N^3; each rank's list keeps ascending index order."""
    N = np.asarray(N, dtype=np.int64)
    if world < 1:
        raise ValueError("world must be >= 1")
    load = np.zeros(world)
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(N)), key=lambda q: (-int(N[q]) ** 3, q)):
        r = int(np.argmin(load))
        parts[r].append(i)
        load[r] += float(N[i]) ** 3
    return [sorted(p) for p in parts]


def gather_rows(local_idx, rows: np.ndarray, nlat: int, dist=None, dst: int = 0):
    """Assemble per-lattice rows (rows[q] belongs to lattice local_idx[q])
    into one [nlat, ...] array on rank `dst` (None elsewhere).  Without a
    process group the local rows are the whole ensemble."""
    rows = np.asarray(rows)
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        out = np.empty((nlat,) + rows.shape[1:], dtype=rows.dtype)
        out[np.asarray(local_idx, dtype=np.int64)] = rows
        return out
    payload = (list(map(int, local_idx)), rows)
    objs = [None] * dist.get_world_size() if dist.get_rank() == dst else None
    dist.gather_object(payload, objs, dst=dst)
    if dist.get_rank() != dst:
        return None
    out = np.empty((nlat,) + rows.shape[1:], dtype=rows.dtype)
    seen = np.zeros(nlat, dtype=bool)
    for idx, r in objs:
        if seen[idx].any():
            raise RuntimeError("lattice gathered twice")
        out[idx] = r
        seen[idx] = True
    if not seen.all():
        raise RuntimeError(f"{int((~seen).sum())} lattices missing from the gather")
    return out


def evolve_and_record(ens, steps: int, every: int, dt: float = 0.01):
    """Step `ens` for `steps` steps, reading the log spectra after every
    `every` steps (and at step 0).  Returns (tau [T], logs [T, nlat, 3,
    nlog], scalars [T, nlat, 12])."""
    taus, logs, scs = [], [], []
    for s in range(0, steps + 1, every):
        if s:
            ens.step(every)
        lg, _, _ = ens.log_spectra()
        taus.append(s * dt)
        logs.append(lg)
        scs.append(ens.scalars())
    return np.asarray(taus), np.asarray(logs), np.asarray(scs)
