#!/usr/bin/env python
"""Throughput of GABE's RK2 lattice step on B200: site-updates/s at 512^3
with GWs on, FP32 storage (headline) next to the FP64 path.

One JSON line on rank 0.  A step is one RK2 step of the full path (field
stencil sweeps, GW sources, 12 R2C transforms, TT projection + h/l update,
Friedmann scalars).  Each rank evolves its own lattice (independent
replicas of the workload, weak scaling); no collective touches the data
path, only the timing max over ranks.

  value   device-resident: state uploaded before the timed region, K steps
          bracketed by CUDA events on the library's stream.
  e2e     the drop-in driver's use of the C ABI: upload the FP64 initial
          state from pinned host memory, then per step gabe_step +
          gabe_energies (the scalars slices_time.dat records), then one
          specOut and a download of field[0]/dfield[0] -- all inside the
          timed region.
  --impl reference  times the reference's own CPU step() (compiled from the
          reference sources under oracle/_ref) on the host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "site-updates/s FP32-storage vs FP64 RK2 at 512³+GW, ≤1e-4 energy err; HBM %"
UNIT = "site-updates/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--N", type=int, default=512)
    ap.add_argument("--gws", type=int, default=1)
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-N", type=int, default=0,
                    help="lattice of the CPU reference sample (0 = the headline lattice, --N)")
    ap.add_argument("--cpu-baseline-steps", type=int, default=3, help="timed steps of the in-line CPU baseline")
    ap.add_argument("--profile-steps", type=int, default=3)
    ap.add_argument("--lattice-flags", type=int, default=0,
                    help="gabe_params.flags of the lattices (e.g. 16: GABE_FLAG_OWN_FFT, 128: GABE_FLAG_TRANSPOSED_FFT)")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the batched-ensemble leg")
    ap.add_argument("--no-slab", action="store_true", help="skip the slab leg (one lattice split over the ranks)")
    ap.add_argument("--no-energy", action="store_true", help="skip the energy-conservation block (64^3, rank 0)")
    ap.add_argument("--no-e2e", action="store_true",
                    help="skip the end-to-end leg and its pinned output buffers (for lattices whose FP64 host "
                         "copies would not fit pinned memory, e.g. 1024^3)")
    ap.add_argument("--no-accuracy", action="store_true",
                    help="skip the FP32-vs-FP64 accuracy block on the headline lattice (rank 0)")
    ap.add_argument("--acc-steps", type=int, default=1000, help="steps of the accuracy block")
    ap.add_argument("--acc-dt-div", type=float, default=40.0, help="accuracy block's dt = dx / this (stable RK2)")
    ap.add_argument("--slab-N", type=int, default=512, help="lattice of the slab leg")
    ap.add_argument("--slab-steps", type=int, default=20)
    ap.add_argument("--ens-lattices", type=int, default=256)
    ap.add_argument("--ens-steps", type=int, default=200, help="timed ensemble steps (multiple of --ens-every)")
    ap.add_argument("--ens-every", type=int, default=50, help="steps between log-spectra outputs")
    ap.add_argument("--ens-seed", type=int, default=20261203, help="master seed of the ensemble's parameters")
    return ap.parse_args()


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 200 ms."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.lines: list[str] = []
        self.t = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.idx)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def algorithmic_bytes(N: int, w: int, gws: bool) -> dict:
    """Bytes each phase must move per step (one launch each), w = bytes per
    stored real:
      stage1  sweep A: read f0, fdot0 (2 fields); write 2 x 5 traceless GW
              source components (11,12,13,22,23 of both RK2 stages)
      fft     10 real-to-complex transforms: read N^3, write N^2(N/2+1) complex each
      kspace  read 10 transformed source components and the 4 TT amplitudes
              (h+, hx, l+, lx), write the 4 amplitudes: 36 reals per k-point
      stage2  sweep B: read f0, fdot0; write f0', fdot0'
    and, for the library's 3-D FFT, each of its passes (one launch each):
      fft_rows  read the N^3 reals, write N^2(N/2+1) complex per array
      fft_j, fft_i  read and write N^2(N/2+1) complex per array
      fft_i_kspace  the transposed form's pass along i fused with the
              k-space update: the k-space bytes (its transformed sources are
              read once and never written)"""
    n3 = N ** 3
    M = N * N * (N // 2 + 1)
    b = {"stage1": (4 + (10 if gws else 0)) * n3 * w, "stage2": 8 * n3 * w}
    if gws:
        b["fft"] = 10 * (n3 + 2 * M) * w
        b["kspace"] = 36 * M * w
        b["fft_rows"] = 10 * (n3 + 2 * M) * w
        b["fft_j"] = b["fft_i"] = 10 * 4 * M * w
        b["fft_i_kspace"] = b["kspace"]
    return b


def ensemble_step_bytes(N: int) -> int:
    """Algorithmic bytes of one FP32 ensemble step of an N^3 lattice with
    GWs: sweep A, the ten transforms counted once as one pass (cuFFT's
    batched plan transforms the ensemble's sources; its internal passes are
    not counted), the k-space update and sweep B."""
    b = algorithmic_bytes(N, 4, True)
    return b["stage1"] + b["fft"] + b["kspace"] + b["stage2"]


def reference_formulation_bytes(w: int, gws: bool) -> int:
    """Bytes per site-update the reference's own formulation needs at the
    minimum (two state sweeps + one write of 2 fields: 12 words; with GWs
    12 source words, 24 FFT words, 36 k-space words for 6 components of h
    and l): 96/672 B in FP64, 48/336 B in FP32."""
    return (12 + (72 if gws else 0)) * w


def traffic_scaled(kernel: str, precision: str, N: int):
    """ncu-measured DRAM bytes per launch from profiles/traffic.json, scaled
    from the captured lattice to N by the sites processed."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as fh:
        d = json.load(fh)
    e = d.get(precision, {}).get(kernel)
    if not e:
        return None
    # DRAM bytes grow with the sites (sweeps, row pass) or k-points (k-space, column passes) processed
    kpts = kernel in ("kspace", "fft_j", "fft_i", "fft_i_kspace")
    scale = (N / e["N"]) ** 3 if not kpts else (N * N * (N // 2 + 1)) / (e["N"] ** 2 * (e["N"] // 2 + 1))
    return e["bytes"] * scale


def cpu_reference_sample(N: int, steps: int, warm: int = 1):
    """Time the reference's own step() (oracle/_ref binary) with all host
    threads on an N^3 GW-on lattice; returns (site-updates/s, info)."""
    from oracle import pyoracle as po

    threads = os.cpu_count() or 1
    binary = po.ref_binary(1, N, 1, 1)
    import tempfile

    if os.path.exists(binary):
        with tempfile.TemporaryDirectory() as d:
            out = po.run_ref(binary, ["--steps", str(warm + steps), "--cheap-ic", "--time"], d, threads=threads,
                             timeout=3600)
        rec = json.loads(out.strip().splitlines()[-1])
        st = rec["step_s"][warm:]
        return N ** 3 * len(st) / sum(st), {"kind": "reference", "cores": threads, "step_s": st,
                                            "sample": f"reference step() on a {N}^3 lattice, GWs on, L=20, dt=0.01, "
                                                      f"lambda phi^4 g^2/lambda=100, {len(st)} timed steps after "
                                                      f"{warm} warm-up, {threads} OpenMP threads, FFT via the "
                                                      f"project's FFTW-API shim"}
    # the oracle restatement (serial) if the reference binary was not built
    Np = 32
    cfg = po.Config(N=Np, gws=1)
    stt = po.init_state(cfg)
    po.step(stt, 1)
    t0 = time.perf_counter()
    po.step(stt, steps)
    dt = time.perf_counter() - t0
    return Np ** 3 * steps / dt, {"kind": "port", "cores": 1, "sample": f"oracle port, {Np}^3 GW on, {steps} steps"}


def slab_leg(args, rank: int, world: int, local: int, dist, barrier, max_over_ranks):
    """One lattice split into slabs of planes along i over the ranks (FP32
    storage, GWs on): per step sweep A, an all-reduce of the 8 stage sums,
    the finish, 2-D transforms of the own source planes, an all-to-all
    transpose by ky columns, the pass along i and the h/l update of the
    rank's k-points, sweep B and the exchange of boundary planes (strong
    scaling: the lattice is fixed).  Timed with CUDA events on the slab's stream,
    which record the whole step including the waits for the exchanges; max
    over ranks."""
    import numpy as np
    import torch

    import gabe_b200 as gb
    from gabe_b200 import slab as gs
    from gabe_b200.ic import random_state

    N, K, W = args.slab_N, args.slab_steps, max(3, args.warmup)
    lat = None
    ok = 1.0
    try:
        comm = gs.DistComm() if dist else gs.LocalComm(1)
        lat = gs.SlabLattice(N, comm, precision=gb.FP32, device=local, gws=True)
        (p0, n), = lat.planes
        f, d, a0, ad0 = random_state(N, seed=11, device="cuda")
        fl, dl = f[:, p0:p0 + n].cpu().numpy(), d[:, p0:p0 + n].cpu().numpy()
        mean = np.array([float(f[0].mean()), float(f[1].mean()), float(d[0].mean()), float(d[1].mean())])
        del f, d
        torch.cuda.empty_cache()
    except Exception as e:  # noqa: BLE001 -- reported in the line, and every rank skips together
        ok, err = 0.0, f"{type(e).__name__}: {e}"
    if max_over_ranks(-ok) > -1.0:  # some rank failed its setup
        if lat:
            lat.close()
        return {"skipped": err if ok == 0.0 else "setup failed on another rank"}
    lat.upload(fl, dl, a0, ad0, mean=mean)
    lat.step(W)
    (s,) = lat.slabs
    stream = torch.cuda.ExternalStream(s.stream_ptr)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    barrier()
    ev[0].record(stream)
    lat.step(K)
    ev[1].record(stream)
    ev[1].synchronize()
    ms = max_over_ranks(ev[0].elapsed_time(ev[1]))
    sc = lat.scalars()
    lat.close()
    sites = float(N) ** 3
    return {"workload": f"{N}^3 lattice split into {world} slab(s) of planes along i, GWs on, FP32 storage; "
                        f"per step: sweep A, all-reduce of 8 FP64 sums, finish, 2-D transforms of the source "
                        f"planes, all-to-all transpose, pass along i + h/l update, sweep B, boundary-plane exchange",
            "planes": [list(pp) for pp in gs.split_planes(N, world)], "scaling": "strong", "n_gpus": world,
            "steps": K, "warmup": W, "ms_per_step": ms / K, "site_updates_per_s": sites * K / (ms / 1e3),
            "halo_bytes_per_rank_per_step": 2 * s.halo_bytes,
            "transpose_bytes_per_rank_per_step": int(sum(s.gw_send_bytes)), "finite": bool(np.all(np.isfinite(sc)))}


def ensemble_leg(args, rank: int, world: int, local: int, dist, barrier, max_over_ranks):
    """The uneven batched ensemble: lattices of N in {32,48,64,96,128},
    g^2/lambda log-uniform [1,500], amplitude U[0.5,2], FP32 storage, GWs
    on, 64-bin log spectra of phi, chi and GWs every `ens_every` steps.
    Lattices are split over ranks by sum N^3 (strong scaling: the ensemble
    is fixed); the spectra are gathered on rank 0 at the end."""
    import numpy as np
    import torch

    import gabe_b200 as gb
    from gabe_b200 import ensemble as ge

    Ns, g, amp, seeds = ge.sample_parameters(args.ens_lattices, args.ens_seed)
    mine = ge.partition(Ns, world)[rank]
    every = args.ens_every
    K = max(every, args.ens_steps // every * every)
    ens = gb.Ensemble(Ns[mine], g[mine], amp[mine], seeds[mine], nlog=64, device=local, tiles="auto",
                      log_top_bin=gb.numbins(max(ge.SIZES)))
    stream = torch.cuda.ExternalStream(ens.stream_ptr)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    ev[0].record(stream)
    ens.init()
    ev[1].record(stream)
    ev[1].synchronize()
    ms_init = max_over_ranks(ev[0].elapsed_time(ev[1]))
    ens.step(max(3, args.warmup))
    ens.log_spectra()
    barrier()
    # steps with the log-spectra output cadence (each output reads the
    # spectra back to the host)
    ev[0].record(stream)
    for _ in range(K // every):
        ens.step(every)
        logs, _, _ = ens.log_spectra()
    ev[1].record(stream)
    ev[1].synchronize()
    ms = max_over_ranks(ev[0].elapsed_time(ev[1]))
    # the same steps without outputs
    barrier()
    ev[2].record(stream)
    ens.step(K)
    ev[3].record(stream)
    ev[3].synchronize()
    ms_steps = max_over_ranks(ev[2].elapsed_time(ev[3]))
    sc = ens.scalars()
    logs, cnt, _ = ens.log_spectra()
    local_rows = np.concatenate([logs.reshape(len(mine), -1), sc], axis=1)
    launches = ens.launches_per_step
    graph_active = ens.graph_active
    dev_bytes = ens.device_bytes
    ens.close()
    torch.cuda.empty_cache()
    full = ge.gather_rows(mine, local_rows, args.ens_lattices, dist if world > 1 else None)
    sites = float(np.sum(np.asarray(Ns, dtype=np.float64) ** 3))
    nspec = args.ens_lattices * (K // every)
    algo = sum(ensemble_step_bytes(int(n)) for n in Ns)
    out = {
        "workload": f"{args.ens_lattices} lattices, N uniform on {{32,48,64,96,128}}, g^2/lambda log-uniform "
                    f"[1,500], amplitude U[0.5,2], master seed {args.ens_seed}, FP32 storage, GWs on, "
                    f"64-bin log spectra every {every} steps",
        "sites": sites, "steps": K, "scaling": "strong", "n_gpus": world,
        "site_updates_per_s": sites * K / (ms / 1e3),
        "spectra_per_s": nspec / (ms / 1e3),
        "ms_per_step_with_outputs": ms / K,
        "site_updates_per_s_steps_only": sites * K / (ms_steps / 1e3),
        "ms_per_step_steps_only": ms_steps / K,
        "step_algorithmic_bytes": algo,
        "step_achieved_gbs": algo / (ms_steps / K / 1e3) / 1e9,
        "ms_init": ms_init,
        "gpu_launches_per_step": launches,
        "graph_active": graph_active,
        "device_bytes_rank0": dev_bytes,
    }
    if full is not None:
        nl = 3 * 64
        out["finite_lattices"] = int(np.sum(np.all(np.isfinite(full[:, nl:]), axis=1)))
        out["nonempty_log_bins_mean"] = float(np.mean(np.sum(np.isfinite(full[:, :64]), axis=1)))
    return out


def run_reference_arm(args, rank: int):
    if rank != 0:
        return
    args.ref_N = args.ref_N or args.N
    v, info = cpu_reference_sample(args.ref_N, args.steps, warm=args.warmup)
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * sum(info.get("step_s", [0])) / max(1, len(info.get("step_s", [1]))),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"GABE RK2 step, {args.ref_N}^3 lattice, GWs on"
                               + ("" if args.ref_N == args.N else f" (a sample of the {args.N}^3 workload)"),
                   "N": args.ref_N, "gws": 1, "L": 20.0, "dt": 0.01, "model": "lambda phi^4, g^2/lambda=100"},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": info["cores"], "kind": info["kind"],
                         "sample": info["sample"]},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def energy_conservation(N: int = 64, steps: int = 500, dt: float = 0.01, device: int = 0) -> dict:
    """Energy-conservation error (gabe_b200.energy: the continuity residual
    eps(t) of the per-step scalars) of an FP64 and an FP32 run of one lattice
    from the same initial state, GWs on, at a size where dt = 0.01 is inside
    RK2's stability region (64^3: dt sqrt(12)/dx = 0.11)."""
    import numpy as np

    import gabe_b200 as gb
    from gabe_b200 import energy
    from gabe_b200.ic import random_state

    f, d, a0, ad0 = random_state(N, seed=5, device="cuda")
    f, d = f.cpu().numpy(), d.cpu().numpy()
    eps, spec = {}, {}
    for name, prec in (("fp64", gb.FP64), ("fp32", gb.FP32)):
        with gb.Lattice(N, gws=True, precision=prec, device=device, dt=dt) as lat:
            lat.upload_state(f, d, a0=a0, adot0=ad0)
            rows = []
            for n in range(steps + 1):
                if n:
                    lat.step(1)
                e = lat.calc_energy()
                rows.append((n * dt, e["a"], e["adot"], e["kin"], e["pot"], e["grad"], e["rho"]))
            spec[name] = lat.spec_out()
        r = np.array(rows)
        eps[name] = energy.continuity_residual(*(r[:, c] for c in range(7)))

    def max_rel(cols):  # per-bin relative difference above each column's FFT noise floor
        w, g = spec["fp64"][:, cols], spec["fp32"][:, cols]
        floor = 1e-9 * np.abs(w).max(axis=0, keepdims=True)
        return float(((np.abs(g - w) - floor).clip(min=0) / np.abs(w).clip(min=1e-300)).max())

    return {"workload": f"{N}^3 lattice, GWs on, dt={dt}, {steps} steps, one initial state for both precisions",
            "measure": "eps(t) = |rho(t) - rho(0) + int 3H(rho + p) dt| / rho(t), p = kin - grad/3 - pot",
            "eps_fp64": float(eps["fp64"][-1]), "eps_fp32": float(eps["fp32"][-1]),
            "max_abs_diff_fp32_vs_fp64": float(np.abs(eps["fp32"] - eps["fp64"]).max()),
            "spectra_max_rel_diff_fp32_vs_fp64": {"fields": max_rel([1, 2, 3, 4]), "gw": max_rel([5, 6])}}


def accuracy_block(args, device: int) -> dict:
    """FP32 storage against the FP64 path on the headline lattice with GWs,
    from one initial state, at a dt inside RK2's stability region
    (gabe_b200.accuracy): the largest relative differences of a, adot, kin,
    pot, grad, rho over every step, the continuity residual eps(t) of both
    runs, and the per-bin differences of every spectrum column at four
    output times.  Outside the timed regions."""
    import torch

    from gabe_b200.accuracy import compare_precisions
    from gabe_b200.ic import random_state

    N, L = args.N, 20.0
    f, d, a0, ad0 = random_state(N, seed=20261204, device="cuda")
    f, d = f.cpu().numpy(), d.cpu().numpy()
    torch.cuda.empty_cache()
    K = args.acc_steps
    rep = compare_precisions(f, d, a0, ad0, N=N, steps=K, dt=L / N / args.acc_dt_div, L=L, gws=True,
                             spectra_every=max(1, K // 4), device=device, flags32=args.lattice_flags)
    rep["workload"] = (f"{N}^3 lattice, GWs on, dt = dx/{args.acc_dt_div:g}, {K} steps, FP32 storage and FP64 "
                       f"from one initial state, scalars compared every step, spectra every {max(1, K // 4)} steps")
    return rep


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference_arm(args, rank)
        return

    import torch

    import gabe_b200 as gb
    from gabe_b200.ic import random_state

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as tdist

        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
        dist = tdist

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x: float) -> float:
        if not dist:
            return x
        t = torch.tensor([x], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    N, K, W, gws = args.N, args.steps, args.warmup, bool(args.gws)
    hbm_peak, peak_kind = peaks()
    f, d, a0, adot0 = random_state(N, seed=44463132 + 1000 * rank, device="cuda")
    hf = torch.empty(f.shape, dtype=torch.float64, pin_memory=True)
    hd = torch.empty(d.shape, dtype=torch.float64, pin_memory=True)
    hf.copy_(f)
    hd.copy_(d)
    of = None if args.no_e2e else torch.empty_like(hf, pin_memory=True)
    od = None if args.no_e2e else torch.empty_like(hd, pin_memory=True)
    del f, d
    torch.cuda.empty_cache()

    legs = {}
    precisions = [("fp32", gb.FP32)] + ([] if args.no_fp64 else [("fp64", gb.FP64)])
    clocks = None
    for name, prec in precisions:
        lat = gb.Lattice(N, gws=gws, precision=prec, device=local, tile_shape="auto", flags=args.lattice_flags)
        stream = torch.cuda.ExternalStream(lat.stream_ptr)
        # ---- device-resident leg
        lat.upload_ptrs(hf.data_ptr(), hd.data_ptr(), None, None, a0, adot0)
        lat.step(W)
        lat.sync()
        barrier()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        sampler = ClockSampler(local)
        with sampler:
            time.sleep(0.3)
            ev0.record(stream)
            lat.step(K)
            ev1.record(stream)
            ev1.synchronize()
        torch.cuda.synchronize()
        ms = max_over_ranks(ev0.elapsed_time(ev1))
        if name == "fp32":
            clocks = sampler.summary()
        try:
            en = lat.calc_energy()
            finite = True
        except gb.GabeError:
            en, finite = None, False
        phases = lat.profile_steps(args.profile_steps)
        try:  # the library's own transforms: time their passes one by one
            phases.update(lat.profile_fft_passes(args.profile_steps))
        except gb.GabeError:  # cuFFT's plan: one phase
            pass
        # ---- end-to-end leg through the C ABI with host buffers
        ms_e2e, nonfinite_e2e = None, False
        if not args.no_e2e:
            barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            lat.upload_ptrs(hf.data_ptr(), hd.data_ptr(), None, None, a0, adot0)
            for _ in range(K):
                lat.step(1)
                try:
                    lat.calc_energy()
                except gb.GabeError:
                    nonfinite_e2e = True
            try:
                lat.spec_out()
            except gb.GabeError:
                nonfinite_e2e = True
            lat.download_ptrs(of.data_ptr(), od.data_ptr())
            e1.record(stream)
            e1.synchronize()
            ms_e2e = max_over_ranks(e0.elapsed_time(e1))
        legs[name] = {"ms": ms, "ms_e2e": ms_e2e, "phases": phases, "energies": en, "finite": finite,
                      "graph_active": lat.graph_active,
                      "nonfinite_e2e": nonfinite_e2e, "device_bytes": lat.device_bytes,
                      "launches_per_step": lat.launches_per_step,
                      "tile": [lat.params.tile_shape, lat.params.tile_ci]}
        lat.close()
        torch.cuda.empty_cache()

    sites = N ** 3
    L32 = legs["fp32"]
    value = world * sites * K / (L32["ms"] / 1e3)
    e2e = world * sites * K / (L32["ms_e2e"] / 1e3) if L32["ms_e2e"] else None
    w = 4
    algo = algorithmic_bytes(N, w, gws)
    kern = {}
    for ph, b in algo.items():
        if ph not in L32["phases"]:  # passes of the library's FFT when cuFFT's plan ran instead
            continue
        t = L32["phases"][ph] / 1e3
        kern[ph] = {"ms": L32["phases"][ph], "algorithmic_bytes": b, "achieved_gbs": b / t / 1e9 if t > 0 else None}
    # the dominant launch among the library's own kernels: the FFT phase is three launches (its passes
    # are listed one by one when they are the library's) or cuFFT's
    own = {k: v for k, v in kern.items() if k != "fft" and not (k == "kspace" and "fft_i_kspace" in kern)}
    dom = max(own, key=lambda k: own[k]["ms"])
    ach = kern[dom]["achieved_gbs"]
    step_bytes = sum(v for k, v in algo.items() if k in ("stage1", "fft", "kspace", "stage2"))  # FFT once, one pass
    step_s = L32["ms"] / K / 1e3
    ref_bytes = reference_formulation_bytes(w, gws) * sites
    roofline = {"bound": "hbm", "achieved": ach, "peak": hbm_peak, "unit": "GB/s", "frac": ach / hbm_peak,
                "traffic": traffic_scaled(dom, "fp32", N), "kernel": dom, "peak_kind": peak_kind,
                "step_algorithmic_bytes": step_bytes,
                "step_achieved_gbs": step_bytes / step_s / 1e9,
                "step_frac": step_bytes / step_s / 1e9 / hbm_peak,
                "reference_formulation_bytes_per_site": reference_formulation_bytes(w, gws),
                "reference_formulation_gbs": ref_bytes / step_s / 1e9,
                "reference_formulation_frac": ref_bytes / step_s / 1e9 / hbm_peak,
                "kernels": kern}
    extra = {}
    if "fp64" in legs:
        L64 = legs["fp64"]
        v64 = world * sites * K / (L64["ms"] / 1e3)
        extra["fp64"] = {"value": v64, "ms_per_step": L64["ms"] / K,
                         "e2e": world * sites * K / (L64["ms_e2e"] / 1e3) if L64["ms_e2e"] else None,
                         "phases_ms": L64["phases"]}
        extra["fp32_over_fp64"] = value / v64
        if L32["energies"] and L64["energies"]:
            extra["energy_rel_diff_fp32_vs_fp64"] = {
                k: abs(L32["energies"][k] - L64["energies"][k]) / abs(L64["energies"][k])
                for k in ("kin", "pot", "grad", "rho", "a", "adot")}
    h2d = 2 * 2 * sites * 8 / K
    d2h = (K * 48 + gb.numbins(N) * 8 * 8 + 2 * 2 * sites * 8) / K
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": L32["ms"] / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"GABE RK2 step, {N}^3 lattice, GWs on, FP32 storage / FP64 scalars",
                   "N": N, "gws": int(gws), "L": 20.0, "dt": 0.01, "model": "lambda phi^4, g^2/lambda=100",
                   "ic": "Gaussian random field with the reference's randInit distribution (torch generator)",
                   "l2": "inputs larger than L2 (state alone is 2 GiB)",
                   **({"lattice_flags": args.lattice_flags} if args.lattice_flags else {})},
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "ms_total": L32["ms_e2e"]},
        "roofline": roofline,
        "gpu_launches": K * L32["launches_per_step"],
        "clocks": clocks,
        "finite": L32["finite"],
        "tile": {"fp32": L32["tile"], "fp64": legs.get("fp64", {}).get("tile")},
        "graph_active": L32["graph_active"],
        "device_bytes": L32["device_bytes"],
    }
    line.update(extra)
    if not args.no_ensemble:
        line["ensemble"] = ensemble_leg(args, rank, world, local, dist, barrier, max_over_ranks)
    if not args.no_slab:
        try:
            line["slab"] = slab_leg(args, rank, world, local, dist, barrier, max_over_ranks)
        except Exception as e:  # noqa: BLE001 -- the headline line is still printed
            line["slab"] = {"error": f"{type(e).__name__}: {e}"[:300]}
    if rank == 0 and not args.no_energy:
        try:
            line["energy_conservation"] = energy_conservation(device=local)
        except Exception as e:  # noqa: BLE001 -- the headline line is still printed
            line["energy_conservation"] = {"error": f"{type(e).__name__}: {e}"[:300]}
    if rank == 0 and not args.no_accuracy:
        try:
            line["accuracy"] = accuracy_block(args, local)
        except Exception as e:  # noqa: BLE001 -- the headline line is still printed
            line["accuracy"] = {"error": f"{type(e).__name__}: {e}"[:300]}
    if world == 1 and rank == 0 and not args.no_cpu_baseline:
        v, info = cpu_reference_sample(args.ref_N or N, max(3, args.cpu_baseline_steps), warm=1)
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": info["cores"], "kind": info["kind"],
                                "sample": info["sample"]}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
