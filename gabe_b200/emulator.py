"""Spectra emulator on the GPU (include/gabe_mlp.h).

`MLP` mirrors the C ABI: device tensors in, device tensors out, every
product in the library's own kernels.  `Emulator` adds what a parameter
sweep needs around it:

* inputs (log10 g^2/lambda, amplitude multiplier, tau) and targets (the
  ensemble's 3 x nlog log10 spectra, NaN where a log bin is empty) are
  standardised with statistics of the training set; NaN targets are
  excluded from the loss;
* `members` networks from different seeds are trained on the same data; the
  spread of their predictions flags parameter points the emulator should not
  be trusted on, which the lattice then re-runs (`screen`).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import GabeError, library

FP32_ACT = 1
NO_GRAPH = 2


class MLPParams(ctypes.Structure):
    _fields_ = [
        ("struct_size", ctypes.c_int32), ("n_in", ctypes.c_int32), ("width", ctypes.c_int32),
        ("depth", ctypes.c_int32), ("n_out", ctypes.c_int32), ("max_rows", ctypes.c_int32),
        ("lr", ctypes.c_float), ("beta1", ctypes.c_float), ("beta2", ctypes.c_float), ("eps", ctypes.c_float),
        ("weight_decay", ctypes.c_float), ("seed", ctypes.c_uint64), ("device", ctypes.c_int32),
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
        L.gabe_mlp_train_loss.argtypes = [M, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int64)]
        L.gabe_mlp_sync.argtypes = [M]
        L.gabe_mlp_stream.argtypes = [M]
        L.gabe_mlp_stream.restype = ctypes.c_void_p
        L.gabe_mlp_launches_per_train_step.argtypes = [M]
        L.gabe_mlp_launches_per_forward.argtypes = [M]
        L.gabe_mlp_last_error.argtypes = [M]
        L.gabe_mlp_last_error.restype = ctypes.c_char_p
        L._mlp_ready = True
    return L


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


class MLP:
    """One network on one GPU.  Tensors passed in must be contiguous CUDA
    float32 (x [n, n_in], t [n, n_out]) on the handle's device."""

    def __init__(self, *, n_in=3, width=256, depth=4, n_out=192, max_rows=65536, lr=1e-3, weight_decay=0.0,
                 seed=1, fp32_act=False, graph=True, device=-1):
        L = _mlp_lib()
        p = MLPParams()
        L.gabe_mlp_default_params(ctypes.byref(p))
        p.n_in, p.width, p.depth, p.n_out, p.max_rows = n_in, width, depth, n_out, max_rows
        p.lr, p.weight_decay, p.seed, p.device = lr, weight_decay, seed, device
        p.flags = (FP32_ACT if fp32_act else 0) | (0 if graph else NO_GRAPH)
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

    def reset_batches(self):
        self._check(_mlp_lib().gabe_mlp_reset_batches(self._h))

    def train_loss(self):
        m, s = ctypes.c_double(), ctypes.c_int64()
        self._check(_mlp_lib().gabe_mlp_train_loss(self._h, ctypes.byref(m), ctypes.byref(s)))
        return m.value, s.value

    def sync(self):
        self._check(_mlp_lib().gabe_mlp_sync(self._h))

    def fit(self, x, t, epochs: int, batch: int, seed: int = 0, log_every: int = 0):
        """Trains on all rows of x, t (device tensors) for `epochs` passes in
        shuffled batches; the permutations of all epochs are drawn up front
        and kept on the device.  Returns the mean batch loss per logged
        epoch."""
        import torch

        n = x.shape[0]
        nb = n // batch
        if nb < 1:
            raise ValueError("fewer rows than one batch")
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
    """`members` MLPs on standardised (log10 g^2/lambda, amplitude, tau) ->
    standardised log spectra."""

    def __init__(self, members: int = 4, *, n_out=192, width=256, depth=4, lr=1e-3, seed=1, fp32_act=False,
                 device=-1):
        self.nets = [MLP(n_out=n_out, width=width, depth=depth, lr=lr, seed=seed + 7919 * k, fp32_act=fp32_act,
                         device=device) for k in range(members)]
        self.n_out = n_out
        self.stats = None

    def close(self):
        for n in self.nets:
            n.close()

    @staticmethod
    def features(g2_over_lambda, amplitude, tau):
        return np.stack([np.log10(np.asarray(g2_over_lambda, dtype=np.float64)),
                         np.asarray(amplitude, dtype=np.float64), np.asarray(tau, dtype=np.float64)], axis=-1)

    def fit(self, feats: np.ndarray, targets: np.ndarray, epochs: int, batch: int = 512, seed: int = 0):
        import torch

        f = np.asarray(feats, dtype=np.float64)
        y = np.asarray(targets, dtype=np.float64)
        mu_x, sd_x = f.mean(0), f.std(0) + 1e-12
        with np.errstate(invalid="ignore"):
            mu_y = np.nanmean(np.where(np.isfinite(y), y, np.nan), axis=0)
            sd_y = np.nanstd(np.where(np.isfinite(y), y, np.nan), axis=0)
        mu_y = np.where(np.isfinite(mu_y), mu_y, 0.0)
        sd_y = np.where(np.isfinite(sd_y) & (sd_y > 1e-6), sd_y, 1.0)
        self.stats = (mu_x, sd_x, mu_y, sd_y)
        xs = torch.tensor((f - mu_x) / sd_x, dtype=torch.float32, device="cuda")
        ys = torch.tensor((y - mu_y) / sd_y, dtype=torch.float32, device="cuda")  # NaN stays NaN
        hist = []
        for k, net in enumerate(self.nets):
            hist.append(net.fit(xs, ys, epochs, batch, seed=seed + k, log_every=max(1, epochs // 10)))
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
    training sample nearest in standardised (log g, amplitude) at the same
    tau (nearest tau if none matches)."""
    tf = np.asarray(train_feats, dtype=np.float64)
    qf = np.asarray(query_feats, dtype=np.float64)
    sd = tf.std(0) + 1e-12
    out = np.empty((len(qf), train_targets.shape[1]))
    for i, q in enumerate(qf):
        dtau = np.abs(tf[:, 2] - q[2])
        cand = np.flatnonzero(dtau == dtau.min())
        d = (((tf[cand, :2] - q[:2]) / sd[:2]) ** 2).sum(1)
        out[i] = train_targets[cand[np.argmin(d)]]
    return out


def per_bin_error(pred: np.ndarray, truth: np.ndarray):
    """Mean absolute error in dex per output over rows where the truth is
    finite (NaN where no row is)."""
    ok = np.isfinite(truth) & np.isfinite(pred)
    err = np.where(ok, np.abs(pred - truth), 0.0)
    n = ok.sum(0)
    with np.errstate(invalid="ignore"):
        return np.where(n > 0, err.sum(0) / np.maximum(n, 1), np.nan)


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
    ms = e0.elapsed_time(e1) / reps
    flops = 2.0 * n * (net.num_params - sum([net.shape[1]] * net.shape[2]) - net.shape[3])
    return n / (ms / 1e3), {"ms": ms, "rows": n, "gflops": flops / (ms / 1e3) / 1e9}


__all__ = ["MLP", "Emulator", "nearest_neighbour", "per_bin_error", "queries_per_second"]
