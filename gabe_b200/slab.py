"""A lattice split along i into slabs of whole planes (gabe_slab_*).

The reference evolves one lattice in one process.  A lattice that does not
fit one GPU is split here into slabs, one per rank (one GPU each).  A step is
the whole-lattice step of the reference (step(), g2functions.cpp:234-271)
with two exchanges between the ranks, and a third with GWs:

  sweep A on every slab -> all-reduce of the 8 FP64 stage sums ->
  finish (adot0, a[1], adot[1]) -> [GWs: 2-D transforms of the own source
  planes into per-rank blocks -> all-to-all -> pass along i and the h/l
  update of the rank's ky columns] -> sweep B -> boundary-plane exchange.

The spectra take the same transpose with the two fields.  FP64 or FP32
storage (FP32 with GWs or spectra: N in {64, 128, 256, 512}).

`SlabLattice` drives the slabs of one rank through a communicator:
`DistComm` (torch.distributed: all-reduce and a ring of point-to-point
transfers, NCCL on GPUs, gloo on CPUs) or `LocalComm` (all slabs of the
lattice in this process; the sums are added on the host in rank order and
the halos copied device to device).

    from gabe_b200.slab import SlabLattice, DistComm
    lat = SlabLattice(N, DistComm(), precision=FP32)      # rank's planes: lat.planes
    lat.upload(field_local, dfield_local, a0, adot0)       # [2][nplanes][N][N] each
    lat.step(100)
    sc = lat.scalars()                                     # identical on every rank
"""
from __future__ import annotations

import contextlib
import ctypes

import numpy as np

from . import FP32, FP64, MODEL_LPHI4, GabeError, Params, _dp, library, lphi4_constants

KNV = 8  # stage sums per sweep


class SlabParams(ctypes.Structure):
    _fields_ = [("struct_size", ctypes.c_int32), ("plane0", ctypes.c_int32), ("nplanes", ctypes.c_int32),
                ("nranks", ctypes.c_int32)]


_bound = False


def _lib():
    global _bound
    L = library()
    if not _bound:
        H = ctypes.c_void_p
        L.gabe_slab_create.argtypes = [ctypes.POINTER(Params), ctypes.POINTER(SlabParams), ctypes.POINTER(H)]
        L.gabe_slab_destroy.argtypes = [H]
        L.gabe_slab_last_error.argtypes = [H]
        L.gabe_slab_last_error.restype = ctypes.c_char_p
        L.gabe_slab_upload.argtypes = [H, _dp, _dp, _dp, ctypes.c_double, ctypes.c_double]
        L.gabe_slab_download.argtypes = [H, _dp, _dp]
        L.gabe_slab_buffers.argtypes = [H, ctypes.POINTER(_dp)] + [ctypes.POINTER(H)] * 4 + [ctypes.POINTER(ctypes.c_size_t)]
        for f in ("gabe_slab_sweep", "gabe_slab_finish"):
            getattr(L, f).argtypes = [H, ctypes.c_int]
        for f in ("gabe_slab_pack", "gabe_slab_unpack", "gabe_slab_sync"):
            getattr(L, f).argtypes = [H]
        L.gabe_slab_stream.argtypes = [H, ctypes.POINTER(H)]
        L.gabe_slab_scalars.argtypes = [H, _dp]
        i64p = ctypes.POINTER(ctypes.c_int64)
        L.gabe_slab_gw_buffers.argtypes = [H, ctypes.POINTER(H), ctypes.POINTER(H), i64p, i64p]
        for f in ("gabe_slab_gw_transform", "gabe_slab_gw_update"):
            getattr(L, f).argtypes = [H]
        L.gabe_slab_gw_download.argtypes = [H, _dp, _dp]
        L.gabe_slab_spectra_buffers.argtypes = [H, ctypes.POINTER(H), ctypes.POINTER(H), i64p, i64p]
        L.gabe_slab_spectra_transform.argtypes = [H]
        L.gabe_slab_spectra_raw.argtypes = [H, _dp, _dp]
        L.gabe_spectra_from_sums.argtypes = [ctypes.POINTER(Params), ctypes.c_double, _dp, _dp, ctypes.c_int, _dp,
                                             ctypes.c_int]
        _bound = True
    return L


def split_planes(N: int, world: int) -> list[tuple[int, int]]:
    """(plane0, nplanes) of every rank: contiguous, sizes differing by at most one."""
    if world < 1 or world > N:
        raise ValueError(f"cannot split {N} planes over {world} ranks")
    base, extra = divmod(N, world)
    out, p0 = [], 0
    for r in range(world):
        n = base + (1 if r < extra else 0)
        out.append((p0, n))
        p0 += n
    return out


class _DeviceView:
    """A raw device allocation as a zero-copy torch tensor (__cuda_array_interface__)."""

    def __init__(self, ptr: int, nbytes: int, typestr: str, itemsize: int):
        self.__cuda_array_interface__ = {"shape": (nbytes // itemsize,), "typestr": typestr,
                                         "data": (int(ptr), False), "version": 3, "strides": None}


class Slab:
    """One slab on one GPU: the C handle and views of its exchange buffers."""

    def __init__(self, N: int, plane0: int, nplanes: int, *, L: float = 20.0, dt: float = 0.01,
                 model: int = MODEL_LPHI4, model_c=None, precision: int = FP64, device: int = -1,
                 tile_shape: int = -1, tile_ci: int = 0, expansion: int = 1, gws: bool = False, nranks: int = 1):
        lib = _lib()
        p = Params()
        lib.gabe_default_params(ctypes.byref(p), int(N))
        p.L, p.dt, p.gws_on, p.model, p.precision = float(L), float(dt), int(bool(gws)), int(model), int(precision)
        if model_c is None:
            model_c = lphi4_constants() if model == MODEL_LPHI4 else (1e-6, 2.5e-7)
        p.model_c[0], p.model_c[1] = float(model_c[0]), float(model_c[1])
        p.device, p.tile_shape, p.tile_ci, p.expansion = int(device), int(tile_shape), int(tile_ci), int(expansion)
        sp = SlabParams(ctypes.sizeof(SlabParams), int(plane0), int(nplanes), int(nranks))
        self.params = p
        self.N, self.plane0, self.nplanes, self.precision = int(N), int(plane0), int(nplanes), int(precision)
        self.gws, self.nranks = bool(gws), int(nranks)
        self._h = ctypes.c_void_p()
        rc = lib.gabe_slab_create(ctypes.byref(p), ctypes.byref(sp), ctypes.byref(self._h))
        if rc != 0:
            self._h = None
            raise GabeError(rc, lib.gabe_slab_last_error(None).decode())
        sums = _dp()
        bufs = [ctypes.c_void_p() for _ in range(4)]
        nb = ctypes.c_size_t()
        self._check(lib.gabe_slab_buffers(self._h, ctypes.byref(sums), *[ctypes.byref(b) for b in bufs], ctypes.byref(nb)))
        self._ptrs = {"sums": ctypes.cast(sums, ctypes.c_void_p).value, "send_lo": bufs[0].value,
                      "send_hi": bufs[1].value, "recv_lo": bufs[2].value, "recv_hi": bufs[3].value}
        self.halo_bytes = int(nb.value)
        st = ctypes.c_void_p()
        self._check(lib.gabe_slab_stream(self._h, ctypes.byref(st)))
        self.stream_ptr = st.value or 0
        spec = (self.precision == FP64 or self.N in (64, 128, 256, 512)) and self.nranks >= 1
        kinds = (["gw"] if self.gws else []) + (["spec"] if spec else [])
        for kind in kinds:  # all-to-all buffers of the GW sources and of the spectra's two fields
            snd, rcv = ctypes.c_void_p(), ctypes.c_void_p()
            sb = (ctypes.c_int64 * self.nranks)()
            rb = (ctypes.c_int64 * self.nranks)()
            fn = lib.gabe_slab_gw_buffers if kind == "gw" else lib.gabe_slab_spectra_buffers
            self._check(fn(self._h, ctypes.byref(snd), ctypes.byref(rcv), sb, rb))
            self._ptrs[f"{kind}_send"], self._ptrs[f"{kind}_recv"] = snd.value, rcv.value
            setattr(self, f"{kind}_send_bytes", list(sb))
            setattr(self, f"{kind}_recv_bytes", list(rb))

    def _check(self, rc: int):
        if rc != 0:
            raise GabeError(rc, _lib().gabe_slab_last_error(self._h).decode())

    def close(self):
        if self._h:
            _lib().gabe_slab_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- buffers as torch tensors (CUDA) -----------------------------------
    def tensor(self, name: str):
        import torch

        if name == "sums":
            return torch.as_tensor(_DeviceView(self._ptrs["sums"], KNV * 8, "<f8", 8), device="cuda")
        if name.endswith("_send") or name.endswith("_recv"):  # all-to-all buffers, as float32
            nbytes = sum(getattr(self, f"{name}_bytes"))
            return torch.as_tensor(_DeviceView(self._ptrs[name], nbytes, "<f4", 4), device="cuda")
        return torch.as_tensor(_DeviceView(self._ptrs[name], self.halo_bytes, "|u1", 1), device="cuda")

    # -- the stage calls ----------------------------------------------------
    def upload(self, field0: np.ndarray, dfield0: np.ndarray, mean, a0: float, adot0: float):
        f = np.ascontiguousarray(field0, dtype=np.float64)
        d = np.ascontiguousarray(dfield0, dtype=np.float64)
        want = (2, self.nplanes, self.N, self.N)
        if f.shape != want or d.shape != want:
            raise ValueError(f"slab arrays must have shape {want}")
        m = None if mean is None else np.ascontiguousarray(mean, dtype=np.float64)
        self._check(_lib().gabe_slab_upload(self._h, f.ctypes.data_as(_dp), d.ctypes.data_as(_dp),
                                            None if m is None else m.ctypes.data_as(_dp), float(a0), float(adot0)))

    def download(self):
        f = np.empty((2, self.nplanes, self.N, self.N))
        d = np.empty_like(f)
        self._check(_lib().gabe_slab_download(self._h, f.ctypes.data_as(_dp), d.ctypes.data_as(_dp)))
        return f, d

    def sweep(self, which: int):
        self._check(_lib().gabe_slab_sweep(self._h, int(which)))

    def finish(self, which: int):
        self._check(_lib().gabe_slab_finish(self._h, int(which)))

    def pack(self):
        self._check(_lib().gabe_slab_pack(self._h))

    def unpack(self):
        self._check(_lib().gabe_slab_unpack(self._h))

    def sync(self):
        self._check(_lib().gabe_slab_sync(self._h))

    def scalars(self) -> np.ndarray:
        out = np.empty(12)
        self._check(_lib().gabe_slab_scalars(self._h, out.ctypes.data_as(_dp)))
        return out

    def gw_transform(self):
        self._check(_lib().gabe_slab_gw_transform(self._h))

    def gw_update(self):
        self._check(_lib().gabe_slab_gw_update(self._h))

    def spectra_transform(self):
        self._check(_lib().gabe_slab_spectra_transform(self._h))

    def spectra_raw(self):
        nb = int(np.sqrt(3.0) * self.N / 2 + 1)
        ns = 2 + int(self.gws)
        sums, cnt = np.zeros((ns, nb)), np.zeros(nb)
        self._check(_lib().gabe_slab_spectra_raw(self._h, sums.ctypes.data_as(_dp), cnt.ctypes.data_as(_dp)))
        return sums, cnt

    def gw_download(self):
        """h, l of this slab's k-points, [12][N][nplanes][N/2+1] each (ky = plane0 + y)."""
        shape = (12, self.N, self.nplanes, self.N // 2 + 1)
        h, l = np.empty(shape), np.empty(shape)
        self._check(_lib().gabe_slab_gw_download(self._h, h.ctypes.data_as(_dp), l.ctypes.data_as(_dp)))
        return h, l


def _on_slab_stream(s):
    """Torch work inside this context is ordered on the slab's CUDA stream
    (after the library's kernels, before its next ones), so no host
    synchronisation is needed around it; CPU stand-ins need none."""
    if s.tensor("sums").is_cuda:
        import torch

        return torch.cuda.stream(torch.cuda.ExternalStream(s.stream_ptr))
    return contextlib.nullcontext()


def _sync_devices(slabs):
    """Wait for the copies between slabs (CUDA); CPU stand-ins need nothing."""
    if slabs[0].tensor("sums").is_cuda:
        import torch

        torch.cuda.synchronize()


class LocalComm:
    """Every slab of the lattice in this process (one GPU or several):
    sums added on the host in rank order, halos copied device to device.
    A single slab needs neither: its sums are the totals, and its halos are
    copies of its own end planes, taken on its stream."""

    def __init__(self, world: int):
        self.world = int(world)

    def allreduce_sums(self, slabs):
        if len(slabs) == 1:
            return
        for s in slabs:
            s.sync()
        tot = np.zeros(KNV)
        views = [s.tensor("sums") for s in slabs]
        for v in views:
            tot += v.cpu().numpy()
        import torch

        t = torch.from_numpy(tot)
        for v in views:
            v.copy_(t)
        _sync_devices(slabs)

    def exchange(self, slabs):
        import torch

        if len(slabs) == 1:
            (s,) = slabs
            with _on_slab_stream(s):
                s.tensor("recv_lo").copy_(s.tensor("send_hi"))
                s.tensor("recv_hi").copy_(s.tensor("send_lo"))
            return
        for s in slabs:
            s.sync()
        W = len(slabs)
        for r, s in enumerate(slabs):
            s.tensor("recv_lo").copy_(slabs[(r - 1) % W].tensor("send_hi"))
            s.tensor("recv_hi").copy_(slabs[(r + 1) % W].tensor("send_lo"))
        _sync_devices(slabs)

    def all_to_all(self, slabs, kind: str = "gw"):
        """Transpose (kind "gw": the sources, "spec": the two fields): block r'
        of slab r's send buffer -> slab r''s receive buffer, at r."""
        import torch

        if len(slabs) == 1:
            (s,) = slabs
            with _on_slab_stream(s):
                s.tensor(f"{kind}_recv").copy_(s.tensor(f"{kind}_send"))
            return
        for s in slabs:
            s.sync()
        W = len(slabs)
        for src in range(W):
            snd = slabs[src].tensor(f"{kind}_send")
            soff = np.cumsum([0] + [b // 4 for b in getattr(slabs[src], f"{kind}_send_bytes")])
            for dst in range(W):
                rcv = slabs[dst].tensor(f"{kind}_recv")
                roff = np.cumsum([0] + [b // 4 for b in getattr(slabs[dst], f"{kind}_recv_bytes")])
                rcv[roff[src]:roff[src + 1]].copy_(snd[soff[dst]:soff[dst + 1]])
        _sync_devices(slabs)

    def allreduce_host(self, v: np.ndarray) -> np.ndarray:
        return v


class DistComm:
    """One slab per rank of a torch.distributed process group: the sums by
    all_reduce, the boundary planes by a ring of point-to-point transfers
    (rank r sends its top plane to r+1 and its bottom plane to r-1,
    periodic).  `device` is where the exchanged tensors live ("cuda" with
    NCCL, "cpu" with gloo)."""

    def __init__(self, group=None):
        import torch.distributed as dist

        self.dist, self.group = dist, group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)

    def allreduce_sums(self, slabs):
        (s,) = slabs
        with _on_slab_stream(s):  # NCCL: ordered on the slab's stream, no host round trip
            self.dist.all_reduce(s.tensor("sums"), group=self.group)

    def exchange(self, slabs):
        (s,) = slabs
        W, r, d = self.world, self.rank, self.dist
        with _on_slab_stream(s):
            if W == 1:
                s.tensor("recv_lo").copy_(s.tensor("send_hi"))
                s.tensor("recv_hi").copy_(s.tensor("send_lo"))
                return
            lo, hi = (r - 1) % W, (r + 1) % W
            g = lambda p: d.get_global_rank(self.group, p) if self.group is not None else p  # noqa: E731
            ops = [d.P2POp(d.isend, s.tensor("send_hi"), g(hi), self.group, tag=1),
                   d.P2POp(d.isend, s.tensor("send_lo"), g(lo), self.group, tag=0),
                   d.P2POp(d.irecv, s.tensor("recv_lo"), g(lo), self.group, tag=1),
                   d.P2POp(d.irecv, s.tensor("recv_hi"), g(hi), self.group, tag=0)]
            for w in d.batch_isend_irecv(ops):
                w.wait()  # NCCL: the slab's stream waits; gloo: the host waits

    def all_to_all(self, slabs, kind: str = "gw"):
        """Transpose: block r of the send buffer to rank r, arriving at this rank's place."""
        (s,) = slabs
        with _on_slab_stream(s):
            self.dist.all_to_all_single(s.tensor(f"{kind}_recv"), s.tensor(f"{kind}_send"),
                                        output_split_sizes=[b // 4 for b in getattr(s, f"{kind}_recv_bytes")],
                                        input_split_sizes=[b // 4 for b in getattr(s, f"{kind}_send_bytes")],
                                        group=self.group)

    def allreduce_host(self, v: np.ndarray) -> np.ndarray:
        import torch

        t = torch.from_numpy(np.ascontiguousarray(v, dtype=np.float64))
        if self.dist.get_backend(self.group) == "nccl":
            t = t.cuda()
        self.dist.all_reduce(t, group=self.group)
        return t.cpu().numpy()


class SlabLattice:
    """The slabs of one rank (DistComm: one; LocalComm: all of them) and the
    step sequence.  Scalars are the same on every slab."""

    def __init__(self, N: int, comm, *, precision: int = FP64, device: int = -1, gws: bool = False, slab_factory=None,
                 **kw):
        self.N, self.comm, self.precision, self.gws = int(N), comm, int(precision), bool(gws)
        parts = split_planes(self.N, comm.world)
        mine = [comm.rank] if hasattr(comm, "rank") else list(range(comm.world))
        make = slab_factory or (lambda p0, n: Slab(self.N, p0, n, precision=precision, device=device, gws=gws,
                                                   nranks=comm.world, **kw))
        self.parts = [parts[r] for r in mine]
        self.slabs = [make(p0, n) for p0, n in self.parts]

    def close(self):
        for s in self.slabs:
            s.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def planes(self):
        return self.parts

    def _exchange(self):
        for s in self.slabs:
            s.pack()
        self.comm.exchange(self.slabs)
        for s in self.slabs:
            s.unpack()

    def _reduce_and_finish(self, which: int):
        self.comm.allreduce_sums(self.slabs)
        for s in self.slabs:
            s.finish(which)

    def upload(self, fields, dfields, a0: float, adot0: float, mean=None):
        """fields/dfields: per slab of this rank, [2][nplanes][N][N] each (a
        list, or for a single slab the arrays).  mean: <phi>, <chi>, <phidot>,
        <chidot> of the whole lattice (FP32 storage); by default summed over
        the ranks' planes.  Then the halos and the energies, as the
        reference's calcEnergy(0) after its initialisation."""
        if not isinstance(fields, (list, tuple)):
            fields, dfields = [fields], [dfields]
        if mean is None and self.precision == FP32:
            loc = np.zeros(4)
            for f, d in zip(fields, dfields):
                loc += np.concatenate([np.asarray(f).reshape(2, -1).sum(axis=1), np.asarray(d).reshape(2, -1).sum(axis=1)])
            mean = self._allreduce_host(loc) / float(self.N) ** 3
        for s, f, d in zip(self.slabs, fields, dfields):
            s.upload(f, d, mean, a0, adot0)
        self._exchange()
        self.energies()

    def _allreduce_host(self, v: np.ndarray) -> np.ndarray:
        return self.comm.allreduce_host(v)

    def energies(self):
        for s in self.slabs:
            s.sweep(2)
        self._reduce_and_finish(2)

    def step(self, nsteps: int = 1):
        for _ in range(int(nsteps)):
            for s in self.slabs:
                s.sweep(0)
            self._reduce_and_finish(0)
            if self.gws:  # sources of this step: 2-D transforms, transpose, pass along i, h/l update
                for s in self.slabs:
                    s.gw_transform()
                self.comm.all_to_all(self.slabs)
                for s in self.slabs:
                    s.gw_update()
            for s in self.slabs:
                s.sweep(1)
            self._exchange()

    def scalars(self) -> np.ndarray:
        """a, adot, edkin, edpot, edgrad, edrho (two stages each) after the
        energies of the current state."""
        self.energies()
        out = [s.scalars() for s in self.slabs]
        return out[0]

    def download(self):
        return [s.download() for s in self.slabs]

    def spectra(self) -> np.ndarray:
        """The table of gabe_spectra (specOut's columns) of the whole lattice,
        the same on every rank: each rank bins its k-points after the fields'
        transpose, the sums are added over the ranks and normalised with the
        stage-0 energy density."""
        sc = self.scalars()
        for s in self.slabs:
            s.spectra_transform()
        self.comm.all_to_all(self.slabs, "spec")
        raw = [s.spectra_raw() for s in self.slabs]
        sums = sum(r[0] for r in raw)
        cnt = sum(r[1] for r in raw)
        flat = self._allreduce_host(np.concatenate([sums.ravel(), cnt]))
        ns, nb = sums.shape
        sums, cnt = np.ascontiguousarray(flat[:ns * nb].reshape(ns, nb)), np.ascontiguousarray(flat[ns * nb:])
        ncols = 5 + (3 if self.gws else 0)
        out = np.zeros((nb, ncols))
        s0 = self.slabs[0]
        rc = _lib().gabe_spectra_from_sums(ctypes.byref(s0.params), float(sc[10]), sums.ctypes.data_as(_dp),
                                           cnt.ctypes.data_as(_dp), nb, out.ctypes.data_as(_dp), ncols)
        if rc != 0:
            raise GabeError(rc, "gabe_spectra_from_sums")
        return out

    def download_gw(self):
        """(h, l) per slab of this rank: its ky columns of the reference's
        [12][N][N][N/2+1] arrays."""
        return [s.gw_download() for s in self.slabs]
