"""Spectra emulator on the GPU (include/gabe_mlp.h).

`MLP` mirrors the C ABI: device tensors in, device tensors out, every
product in the library's own kernels.  `Emulator` adds what a parameter
sweep needs around it:

* inputs (log10 g^2/lambda, amplitude multiplier, tau, log2 N) and targets
  (the ensemble's 3 x nlog log10 spectra, NaN where a log bin is empty) are
  standardised with statistics of the training set; NaN targets are
  excluded from the loss.  The lattice size is an input because the GW
  source of the initial vacuum fluctuations is gradient (UV) dominated:
  spectra of the same parameters differ by about a decade between 32^3 and
  128^3, so an emulator trained on an uneven ensemble must know which size
  it is asked for;
* `members` networks from different seeds are trained on the same data; the
  spread of their predictions flags parameter points the emulator should not
  be trusted on, which the lattice then re-runs (`screen`; `screened_sweep`
  answers a whole sweep that way, the flagged points from the lattice).
"""
from __future__ import annotations

import ctypes
import warnings

import numpy as np

from . import GabeError, library

FP32_ACT = 1
NO_GRAPH = 2
MMA_SYNC = 4


class MLPParams(ctypes.Structure):
    _fields_ = [
        ("struct_size", ctypes.c_int32), ("n_in", ctypes.c_int32), ("width", ctypes.c_int32),
        ("depth", ctypes.c_int32), ("n_out", ctypes.c_int32), ("max_rows", ctypes.c_int32),
        ("lr", ctypes.c_float), ("beta1", ctypes.c_float), ("beta2", ctypes.c_float), ("eps", ctypes.c_float),
        ("weight_decay", ctypes.c_float), ("lr_min", ctypes.c_float), ("decay_steps", ctypes.c_int32),
        ("seed", ctypes.c_uint64), ("device", ctypes.c_int32),
        ("flags", ctypes.c_int32),
    ]


def _mlp_lib():
    L = library()
    if not getattr(L, "_mlp_ready", False):
        M = ctypes.c_void_p
        vp, fp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_float)
        L.gabe_mlp_default_params.argtypes = [ctypes.POINTER(MLPParams)]
        L.gabe_mlp_default_params.restype = None
        L.gabe_mlp_create.argtypes = [ctypes.POINTER(MLPParams), ctypes.POINTER(M)]
        L.gabe_mlp_destroy.argtypes = [M]
        L.gabe_mlp_num_params.argtypes = [M]
        L.gabe_mlp_num_params.restype = ctypes.c_int64
        L.gabe_mlp_set_params.argtypes = [M, fp]
        L.gabe_mlp_get_params.argtypes = [M, fp]
        L.gabe_mlp_forward.argtypes = [M, vp, ctypes.c_int64, vp]
        L.gabe_mlp_loss_grad.argtypes = [M, vp, vp, ctypes.c_int64, ctypes.POINTER(ctypes.c_double), fp]
        L.gabe_mlp_train.argtypes = [M, vp, vp, vp, ctypes.c_int32, ctypes.c_int32]
        L.gabe_mlp_reset_batches.argtypes = [M]
        L.gabe_mlp_set_schedule.argtypes = [M, ctypes.c_float, ctypes.c_float, ctypes.c_int32]
        L.gabe_mlp_train_loss.argtypes = [M, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int64)]
        L.gabe_mlp_sync.argtypes = [M]
        L.gabe_mlp_stream.argtypes = [M]
        L.gabe_mlp_stream.restype = ctypes.c_void_p
        L.gabe_mlp_launches_per_train_step.argtypes = [M]
        L.gabe_mlp_launches_per_forward.argtypes = [M]
        L.gabe_mlp_last_error.argtypes = [M]
        L.gabe_mlp_last_error.restype = ctypes.c_char_p
        L.gabe_mlp_forward_form.argtypes = [M, ctypes.c_int32]
        L._mlp_ready = True
    return L


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


class MLP:
    """One network on one GPU.  Tensors passed in must be contiguous CUDA
    float32 (x [n, n_in], t [n, n_out]) on the handle's device."""

    def __init__(self, *, n_in=3, width=256, depth=4, n_out=192, max_rows=65536, lr=1e-3, weight_decay=0.0,
                 seed=1, fp32_act=False, graph=True, device=-1, mma_sync=False):
        L = _mlp_lib()
        p = MLPParams()
        L.gabe_mlp_default_params(ctypes.byref(p))
        p.n_in, p.width, p.depth, p.n_out, p.max_rows = n_in, width, depth, n_out, max_rows
        p.lr, p.weight_decay, p.seed, p.device = lr, weight_decay, seed, device
        p.flags = (FP32_ACT if fp32_act else 0) | (0 if graph else NO_GRAPH) | (MMA_SYNC if mma_sync else 0)
        self.p = p
        self.shape = (n_in, width, depth, n_out)
        self._h = ctypes.c_void_p()
        rc = L.gabe_mlp_create(ctypes.byref(p), ctypes.byref(self._h))
        if rc != 0:
            self._h = None
            raise GabeError(rc, L.gabe_mlp_last_error(None).decode())
        self._perm = None

    def _check(self, rc):
        if rc != 0:
            raise GabeError(rc, _mlp_lib().gabe_mlp_last_error(self._h).decode())

    def close(self):
        if self._h:
            _mlp_lib().gabe_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def num_params(self) -> int:
        return _mlp_lib().gabe_mlp_num_params(self._h)

    @property
    def stream_ptr(self) -> int:
        return _mlp_lib().gabe_mlp_stream(self._h) or 0

    @property
    def launches_per_train_step(self) -> int:
        return _mlp_lib().gabe_mlp_launches_per_train_step(self._h)

    @property
    def launches_per_forward(self) -> int:
        return _mlp_lib().gabe_mlp_launches_per_forward(self._h)

    def get_params(self) -> np.ndarray:
        out = np.empty(self.num_params, dtype=np.float32)
        self._check(_mlp_lib().gabe_mlp_get_params(self._h, _fptr(out)))
        return out

    def set_params(self, params: np.ndarray):
        a = np.ascontiguousarray(params, dtype=np.float32)
        if a.size != self.num_params:
            raise ValueError("parameter count mismatch")
        self._check(_mlp_lib().gabe_mlp_set_params(self._h, _fptr(a)))

    def _after_torch(self):
        """Orders the library's stream after work torch has queued (tensor
        creation and copies on torch's current stream)."""
        import torch

        s = torch.cuda.ExternalStream(self.stream_ptr)
        s.wait_stream(torch.cuda.current_stream())
        return s

    def forward(self, x, out=None):
        """y = net(x); torch's current stream is ordered after the forward."""
        import torch

        x = x.contiguous()
        n = x.shape[0]
        if out is None:
            out = torch.empty((n, self.shape[3]), dtype=torch.float32, device=x.device)
        s = self._after_torch()
        self._check(_mlp_lib().gabe_mlp_forward(self._h, x.data_ptr(), n, out.data_ptr()))
        torch.cuda.current_stream().wait_stream(s)
        return out

    def loss_grad(self, x, t, want_grad=True):
        self._after_torch()
        loss = ctypes.c_double()
        g = np.empty(self.num_params, dtype=np.float32) if want_grad else None
        self._check(_mlp_lib().gabe_mlp_loss_grad(self._h, x.contiguous().data_ptr(), t.contiguous().data_ptr(),
                                                  x.shape[0], ctypes.byref(loss), _fptr(g) if want_grad else None))
        return loss.value, g

    def train_batches(self, x, t, perm, batch: int, nbatch: int):
        """nbatch Adam steps on rows perm[(s0+s)*batch:...] (see gabe_mlp_train)."""
        self._after_torch()
        self._check(_mlp_lib().gabe_mlp_train(self._h, x.data_ptr(), t.data_ptr(), perm.data_ptr(), batch, nbatch))

    def set_schedule(self, lr: float, lr_min: float = 0.0, decay_steps: int = 0):
        self._check(_mlp_lib().gabe_mlp_set_schedule(self._h, lr, lr_min, int(decay_steps)))

    def reset_batches(self):
        self._check(_mlp_lib().gabe_mlp_reset_batches(self._h))

    def train_loss(self):
        m, s = ctypes.c_double(), ctypes.c_int64()
        self._check(_mlp_lib().gabe_mlp_train_loss(self._h, ctypes.byref(m), ctypes.byref(s)))
        return m.value, s.value

    def sync(self):
        """Waits for the handle's stream; raises if a bounded device wait of
        the tensor-core forward gave up."""
        self._check(_mlp_lib().gabe_mlp_sync(self._h))

    def forward_form(self, layer: int) -> str:
        """Kernel of layer `layer`'s forward: "fma" (FP32 FMA), "mma.sync" or
        "tcgen05"."""
        f = _mlp_lib().gabe_mlp_forward_form(self._h, layer)
        if f < 0:
            raise IndexError(layer)
        return ("fma", "mma.sync", "tcgen05")[f]

    def fit(self, x, t, epochs: int, batch: int, seed: int = 0, log_every: int = 0, lr_min: float | None = None):
        """Trains on all rows of x, t (device tensors) for `epochs` passes in
        shuffled batches; the permutations are drawn on the device.  With
        lr_min the learning rate decays from the handle's lr to lr_min over
        the run (cosine).  Returns the mean batch loss per logged epoch."""
        import torch

        n = x.shape[0]
        if n < 1:
            raise ValueError("no training rows")
        batch = min(batch, n)
        nb = n // batch
        if lr_min is not None:
            self.set_schedule(self.p.lr, lr_min, epochs * nb)
        g = torch.Generator(device=x.device)
        g.manual_seed(seed)
        hist = []
        chunk = max(1, min(epochs, (64 << 20) // max(1, n * 4)))  # epochs per permutation upload
        e = 0
        while e < epochs:
            ne = min(chunk, epochs - e)
            self.sync()  # the previous permutation may still be in use
            perm = torch.cat([torch.randperm(n, generator=g, device=x.device)[: nb * batch] for _ in range(ne)])
            self._perm = perm.to(torch.int32).contiguous()
            self.reset_batches()
            for q in range(ne):
                self.train_batches(x, t, self._perm, batch, nb)
                if log_every and (e + q + 1) % log_every == 0:
                    hist.append((e + q + 1, self.train_loss()[0]))
            e += ne
        self.sync()
        return hist


class Emulator:
    """`members` MLPs on standardised (log10 g^2/lambda, amplitude, tau,
    log2 N) -> standardised log spectra."""

    N_IN = 4

    def __init__(self, members: int = 4, *, n_out=192, width=256, depth=4, lr=1e-3, seed=1, fp32_act=False,
                 device=-1):
        self.nets = [MLP(n_in=self.N_IN, n_out=n_out, width=width, depth=depth, lr=lr, seed=seed + 7919 * k,
                         fp32_act=fp32_act, device=device) for k in range(members)]
        self.n_out = n_out
        self.stats = None

    def close(self):
        for n in self.nets:
            n.close()

    @staticmethod
    def features(g2_over_lambda, amplitude, tau, N):
        return np.stack([np.log10(np.asarray(g2_over_lambda, dtype=np.float64)),
                         np.asarray(amplitude, dtype=np.float64), np.asarray(tau, dtype=np.float64),
                         np.log2(np.asarray(N, dtype=np.float64))], axis=-1)

    def fit(self, feats: np.ndarray, targets: np.ndarray, epochs: int, batch: int = 512, seed: int = 0,
            lr_min: float | None = 1e-5):
        import torch

        f = np.asarray(feats, dtype=np.float64)
        y = np.asarray(targets, dtype=np.float64)
        mu_x, sd_x = f.mean(0), f.std(0) + 1e-12
        yn = np.where(np.isfinite(y), y, np.nan)
        with warnings.catch_warnings():
            warnings.simplefilter("ignore", RuntimeWarning)  # outputs no lattice reaches
            mu_y = np.nanmean(yn, axis=0)
            sd_y = np.nanstd(yn, axis=0)
        mu_y = np.where(np.isfinite(mu_y), mu_y, 0.0)
        sd_y = np.where(np.isfinite(sd_y) & (sd_y > 1e-6), sd_y, 1.0)
        self.stats = (mu_x, sd_x, mu_y, sd_y)
        xs = torch.tensor((f - mu_x) / sd_x, dtype=torch.float32, device="cuda")
        ys = torch.tensor((y - mu_y) / sd_y, dtype=torch.float32, device="cuda")  # NaN stays NaN
        hist = []
        for k, net in enumerate(self.nets):
            hist.append(net.fit(xs, ys, epochs, batch, seed=seed + k, log_every=max(1, epochs // 10), lr_min=lr_min))
        return hist

    def predict_members(self, feats: np.ndarray):
        import torch

        mu_x, sd_x, mu_y, sd_y = self.stats
        xs = torch.tensor((np.asarray(feats, dtype=np.float64) - mu_x) / sd_x, dtype=torch.float32, device="cuda")
        outs = []
        for net in self.nets:
            y = net.forward(xs)
            net.sync()
            outs.append(y.cpu().numpy().astype(np.float64) * sd_y + mu_y)
        return np.stack(outs)

    def predict(self, feats: np.ndarray):
        """(mean prediction, member spread) per output, log10 units."""
        P = self.predict_members(feats)
        return P.mean(0), P.std(0)

    def screen(self, feats: np.ndarray, threshold: float, valid_mask: np.ndarray | None = None):
        """Flags rows whose largest member spread over the (valid) outputs
        exceeds `threshold` dex: those points go back to the lattice."""
        mean, spread = self.predict(feats)
        s = spread if valid_mask is None else np.where(valid_mask, spread, 0.0)
        return mean, s.max(axis=-1) > threshold, s.max(axis=-1)


def nearest_neighbour(train_feats: np.ndarray, train_targets: np.ndarray, query_feats: np.ndarray):
    """The lookup a sweep without the emulator has: the target of the
    training sample nearest in standardised (log g, amplitude) among those
    of the nearest lattice size and, within it, the nearest tau."""
    tf = np.asarray(train_feats, dtype=np.float64)
    qf = np.asarray(query_feats, dtype=np.float64)
    sd = tf.std(0) + 1e-12
    out = np.empty((len(qf), train_targets.shape[1]))
    for i, q in enumerate(qf):
        dn = np.abs(tf[:, 3] - q[3])
        same = dn == dn.min()
        dtau = np.where(same, np.abs(tf[:, 2] - q[2]), np.inf)
        cand = np.flatnonzero(dtau == dtau.min())
        d = (((tf[cand, :2] - q[:2]) / sd[:2]) ** 2).sum(1)
        out[i] = train_targets[cand[np.argmin(d)]]
    return out


def per_bin_error(pred: np.ndarray, truth: np.ndarray):
    """Mean absolute error in dex per output over rows where the truth is
    finite (NaN where no row is)."""
    pred, truth = np.asarray(pred, dtype=np.float64), np.asarray(truth, dtype=np.float64)
    ok = np.isfinite(truth) & np.isfinite(pred)
    err = np.zeros(truth.shape)
    err[ok] = np.abs(pred[ok] - truth[ok])
    n = ok.sum(0)
    return np.where(n > 0, err.sum(0) / np.maximum(n, 1), np.nan)


def _nanmean(x) -> float:
    """Mean of the finite entries (NaN when there are none, without a warning)."""
    x = np.asarray(x, dtype=np.float64)
    ok = np.isfinite(x)
    return float(x[ok].mean()) if ok.any() else float("nan")


def queries_per_second(net: MLP, n: int = 1 << 20, reps: int = 5):
    """Forward throughput on n random queries, device-timed."""
    import torch

    x = torch.randn((n, net.shape[0]), device="cuda", dtype=torch.float32)
    y = torch.empty((n, net.shape[3]), device="cuda", dtype=torch.float32)
    s = torch.cuda.ExternalStream(net.stream_ptr)
    net.forward(x, y)
    net.sync()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(reps):
        net.forward(x, y)
    e1.record(s)
    e1.synchronize()
    net.sync()
    ms = e0.elapsed_time(e1) / reps
    flops = 2.0 * n * (net.num_params - sum([net.shape[1]] * net.shape[2]) - net.shape[3])
    return n / (ms / 1e3), {"ms": ms, "rows": n, "gflops": flops / (ms / 1e3) / 1e9}


__all__ = ["MLP", "Emulator", "nearest_neighbour", "per_bin_error", "queries_per_second"]


# ---------------------------------------------------------------------------
# The parameter-sweep workflow: ensembles -> training set -> emulator ->
# held-out lattice re-runs as the check.
# ---------------------------------------------------------------------------
def ensemble_samples(N, g, amp, seeds, steps: int, every: int, nlog: int = 64, dt: float = 0.01, device: int = -1,
                     log_top_bin: int | None = None):
    """Evolves one batched ensemble and returns (features [T*nlat, 4],
    targets [T*nlat, 3*nlog], lattice index per row, device ms).  The log
    bins end at native bin `log_top_bin` (default: that of the largest sweep
    size, 128^3), the same for every ensemble of a sweep."""
    import torch

    from . import Ensemble, numbins
    from .ensemble import SIZES, evolve_and_record

    top = log_top_bin if log_top_bin is not None else numbins(max(SIZES))
    ens = Ensemble(N, g, amp, seeds, nlog=nlog, dt=dt, device=device, tiles="auto", log_top_bin=top)
    s = torch.cuda.ExternalStream(ens.stream_ptr)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    ens.init()
    taus, logs, _ = evolve_and_record(ens, steps, every, dt)
    e1.record(s)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    ens.close()
    T, nlat = logs.shape[:2]
    feats = Emulator.features(np.tile(g, T), np.tile(amp, T), np.repeat(taus, nlat), np.tile(N, T))
    targets = logs.reshape(T * nlat, 3 * nlog)
    lat = np.tile(np.arange(nlat), T)
    return feats, targets, lat, ms


def output_times(steps: int, every: int, dt: float = 0.01) -> np.ndarray:
    """The times at which evolve_and_record reads the spectra: step 0 and
    every `every` steps up to `steps`."""
    return np.arange(0, steps + 1, every) * dt


def screened_sweep(emu, threshold: float, N, g, amp, seeds, steps: int, every: int, nlog: int = 64,
                   dt: float = 0.01, valid_mask=None, runner=None):
    """Answers a parameter sweep with the emulator as screen and the lattice
    as fallback: every (point, output time) is predicted by the emulator,
    and every point whose largest member spread over its output times and
    (valid) bins exceeds `threshold` dex is evolved on the lattice instead
    and answered by it.

    N, g, amp, seeds: per point (lattice size, g^2/lambda, amplitude
    multiplier, seed).  valid_mask: None, [3 nlog] or [points, 3 nlog] bins
    that count for the spread.  runner(N, g, amp, seeds, steps, every, nlog,
    dt=dt) -> (features, targets, lattice, ms) in ensemble_samples' row order
    (time-major, point-minor); by default one batched ensemble of the flagged
    points.  Returns (answers [T * points, 3 nlog] in the same row order, NaN
    where a flagged point's log bin holds no modes; flagged [points]; spread
    [points])."""
    N, g, amp, seeds = (np.asarray(v) for v in (N, g, amp, seeds))
    P = len(g)
    taus = output_times(steps, every, dt)
    T = len(taus)
    feats = Emulator.features(np.tile(g, T), np.tile(amp, T), np.repeat(taus, P), np.tile(N, T))
    mean, spread = emu.predict(feats)
    spread = spread.reshape(T, P, -1)
    if valid_mask is not None:
        vm = np.asarray(valid_mask, dtype=bool)
        spread = np.where(vm if vm.ndim == 1 else vm[None, :, :], spread, 0.0)
    pt_spread = spread.max(axis=(0, 2))
    flagged = pt_spread > threshold
    answers = np.array(mean, dtype=np.float64).reshape(T, P, -1)
    idx = np.flatnonzero(flagged)
    if len(idx):
        run = runner if runner is not None else ensemble_samples
        _, y, _, _ = run(N[idx], g[idx], amp[idx], seeds[idx], steps, every, nlog, dt=dt)
        answers[:, idx, :] = np.asarray(y, dtype=np.float64).reshape(T, len(idx), -1)
    return answers.reshape(T * P, -1), flagged, pt_spread


def run_sweep(*, nlat=256, ensembles=2, steps=2000, every=50, nlog=64, holdout=32, holdout_N=64, members=4,
              epochs=1000, batch=512, lr=1e-3, master_seed=20261203, flag_quantile=0.9, sizes=None, log=print):
    """Trains the emulator on `ensembles` uneven ensembles of `nlat`
    lattices and checks it on `holdout` new parameter points evolved at
    holdout_N^3.  Returns the report dict."""
    import time

    import torch

    from .ensemble import SIZES, sample_parameters

    sizes = tuple(sizes) if sizes else SIZES
    report = {"config": dict(nlat=nlat, ensembles=ensembles, steps=steps, every=every, nlog=nlog, holdout=holdout,
                             holdout_N=holdout_N, members=members, epochs=epochs, batch=batch, lr=lr,
                             master_seed=master_seed, flag_quantile=flag_quantile, sizes=list(sizes))}
    F, Y, LAT = [], [], []
    ens_ms, sites = 0.0, 0.0
    for e in range(ensembles):
        N, g, amp, seeds = sample_parameters(nlat, master_seed + e, sizes=sizes)
        f, y, lat, ms = ensemble_samples(N, g, amp, seeds, steps, every, nlog)
        F.append(f)
        Y.append(y)
        LAT.append(lat + e * nlat)
        ens_ms += ms
        sites += float(np.sum(np.asarray(N, dtype=np.float64) ** 3))
        log(f"ensemble {e}: {len(f)} samples in {ms / 1e3:.1f} s")
    F, Y, LAT = np.concatenate(F), np.concatenate(Y), np.concatenate(LAT)
    report["training_samples"] = int(len(F))
    report["ensemble_lattice_runs_per_s"] = ensembles * nlat / (ens_ms / 1e3)
    report["ensemble_site_updates_per_s"] = sites * steps / (ens_ms / 1e3)
    # validation split by lattice (10 %) for the flagging threshold
    rng = np.random.default_rng(master_seed)
    val_lat = rng.choice(ensembles * nlat, size=max(1, ensembles * nlat // 10), replace=False)
    is_val = np.isin(LAT, val_lat)
    emu = Emulator(members, n_out=3 * nlog, lr=lr, seed=master_seed % 100000)
    t0 = time.perf_counter()
    hist = emu.fit(F[~is_val], Y[~is_val], epochs=epochs, batch=batch, seed=master_seed % 1000)
    torch.cuda.synchronize()
    report["train_s"] = time.perf_counter() - t0
    report["train_loss_history"] = [[int(a), float(b)] for a, b in hist[0]]
    steps_taken = emu.nets[0].train_loss()[1]
    report["adam_steps_per_member"] = int(steps_taken)
    # threshold: quantile of the per-point max spread on validation lattices
    taus = np.unique(F[:, 2])
    _, vspread = emu.predict(F[is_val])
    vmask = np.isfinite(Y[is_val])
    vpt = np.where(vmask, vspread, 0.0).max(1)
    vlat = LAT[is_val]
    per_point = np.array([vpt[vlat == l].max() for l in np.unique(vlat)])
    thr = float(np.quantile(per_point, flag_quantile))
    report["flag_threshold_dex"] = thr
    # held-out parameter points, re-run on the lattice as the check
    _, gh, ah, sh = sample_parameters(holdout, master_seed + 1000)
    Nh = np.full(holdout, holdout_N, dtype=np.int32)
    fh, yh, lath, ms_h = ensemble_samples(Nh, gh, ah, sh, steps, every, nlog)
    report["holdout_lattice_runs_per_s"] = holdout / (ms_h / 1e3)
    report["holdout_ms"] = ms_h
    mean, spread = emu.predict(fh)
    ok = np.isfinite(yh)
    pt_spread = np.array([np.where(ok, spread, 0.0)[lath == l].max() for l in range(holdout)])
    flagged = pt_spread > thr
    nn = nearest_neighbour(F[~is_val], Y[~is_val], fh)
    report["mae_dex_by_tau"] = {
        "tau": [float(t) for t in np.unique(fh[:, 2])],
        "emulator": [[_nanmean(per_bin_error(mean[fh[:, 2] == t], yh[fh[:, 2] == t]).reshape(3, nlog)[s])
                      for s in range(3)] for t in np.unique(fh[:, 2])],
        "nearest_neighbour": [[_nanmean(per_bin_error(nn[fh[:, 2] == t], yh[fh[:, 2] == t]).reshape(3, nlog)[s])
                               for s in range(3)] for t in np.unique(fh[:, 2])],
    }
    err_em = per_bin_error(mean, yh)
    err_nn = per_bin_error(nn, yh)
    keep = ~flagged[lath]
    err_unflagged = per_bin_error(mean[keep], yh[keep]) if keep.any() else np.full(3 * nlog, np.nan)

    def summary(err):
        e = err.reshape(3, nlog)
        return {"phi": _nanmean(e[0]), "chi": _nanmean(e[1]), "gw": _nanmean(e[2]), "all": _nanmean(err)}

    report["per_bin_mae_dex"] = {"emulator": err_em.reshape(3, nlog).tolist(),
                                 "nearest_neighbour": err_nn.reshape(3, nlog).tolist()}
    report["mae_dex"] = {"emulator": summary(err_em), "nearest_neighbour": summary(err_nn),
                         "emulator_unflagged": summary(err_unflagged)}
    report["flagged_points"] = [int(i) for i in np.flatnonzero(flagged)]
    report["n_flagged"] = int(flagged.sum())
    qps, qinfo = queries_per_second(emu.nets[0])
    report["emulator_queries_per_s"] = qps
    report["emulator_forward"] = qinfo
    # a lattice run yields one spectrum set per output time; the emulator
    # answers one (parameter, time) query with one spectrum set
    report["spectra_per_s_emulator_over_lattice"] = qps / (report["holdout_lattice_runs_per_s"] * len(taus))
    emu.close()
    return report


def main():
    import argparse
    import json

    ap = argparse.ArgumentParser(description="emulator sweep: ensembles -> training -> held-out lattice check")
    ap.add_argument("--lattices", type=int, default=256)
    ap.add_argument("--ensembles", type=int, default=2)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--every", type=int, default=50)
    ap.add_argument("--holdout", type=int, default=32)
    ap.add_argument("--members", type=int, default=4)
    ap.add_argument("--epochs", type=int, default=1000)
    ap.add_argument("--batch", type=int, default=512)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=20261203)
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    rep = run_sweep(nlat=a.lattices, ensembles=a.ensembles, steps=a.steps, every=a.every, holdout=a.holdout,
                    members=a.members, epochs=a.epochs, batch=a.batch, lr=a.lr, master_seed=a.seed)
    s = json.dumps(rep)
    if a.out:
        with open(a.out, "w") as fh:
            fh.write(s)
    short = {k: v for k, v in rep.items() if k not in ("per_bin_mae_dex", "train_loss_history")}
    print(json.dumps(short, indent=1))


if __name__ == "__main__":
    main()
