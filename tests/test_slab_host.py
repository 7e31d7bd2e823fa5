"""Host side of the slab decomposition (gabe_b200.slab, gabe_slab_*), on the
CPU: the plane split, gabe_slab_create's parameter checks (made before any
CUDA call), and the per-step protocol -- all-reduce of the stage sums and
the periodic ring exchange of boundary planes -- through a world-size-3 gloo
process group with stand-in slabs that hold CPU tensors."""
import ctypes
import datetime
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import gabe_b200 as gb
from gabe_b200 import slab as gs


@pytest.mark.parametrize("N,world", [(32, 1), (32, 3), (64, 4), (48, 5), (16, 16)])
def test_split_planes_covers_the_lattice(N, world):
    parts = gs.split_planes(N, world)
    assert len(parts) == world
    assert parts[0][0] == 0 and sum(n for _, n in parts) == N
    for (p0, n), (q0, _) in zip(parts, parts[1:]):
        assert q0 == p0 + n
    sizes = [n for _, n in parts]
    assert max(sizes) - min(sizes) <= 1 and min(sizes) >= 1


def test_split_planes_rejects_more_ranks_than_planes():
    with pytest.raises(ValueError):
        gs.split_planes(16, 17)


@pytest.mark.parametrize("case", ["gws", "gws_expansion2", "gws_split", "planes_hi", "planes_neg", "empty", "N",
                                  "size"])
def test_slab_create_rejects_bad_params(case):
    lib = gs._lib()
    p = gb.Params()
    lib.gabe_default_params(ctypes.byref(p), 32)
    sp = gs.SlabParams(ctypes.sizeof(gs.SlabParams), 0, 8, 0)
    if case == "gws":
        p.gws_on, p.precision = 1, gb.FP32  # FP32 GWs need N in {64, ..., 512}
    elif case == "gws_expansion2":  # a valid split of 64 planes over 4 ranks; only the expansion type is wrong
        p.N, p.gws_on, p.precision, p.expansion, sp.nplanes, sp.nranks = 64, 1, gb.FP32, 2, 16, 4
    elif case == "gws_split":  # planes [0, 8) are not a rank's share of 64 planes over 3 ranks (22, 21, 21)
        p.N, p.gws_on, p.precision, sp.nranks = 64, 1, gb.FP32, 3
    elif case == "planes_hi":
        sp.plane0, sp.nplanes = 28, 8
    elif case == "planes_neg":
        sp.plane0 = -1
    elif case == "empty":
        sp.nplanes = 0
    elif case == "N":
        p.N = 40
    elif case == "size":
        sp.struct_size = 4
    h = ctypes.c_void_p()
    assert lib.gabe_slab_create(ctypes.byref(p), ctypes.byref(sp), ctypes.byref(h)) == 1
    assert not h.value
    msg = lib.gabe_slab_last_error(None)
    assert msg
    if case == "gws_expansion2":
        assert b"expansion_type 1" in msg
    elif case == "gws_split":
        assert b"share" in msg


@pytest.mark.parametrize("N,world,rank", [(48, 3, 1), (64, 2, 0), (80, 5, 4)])
def test_fp64_slabs_with_gws_pass_the_parameter_checks(N, world, rank):
    """FP64 slabs take GWs and spectra at any N that is a multiple of 16 (the
    pass along i is a cuFFT plan): with a rank's standard share the checks
    pass and creation goes on to the device (none here: a CUDA error, not a
    parameter error)."""
    lib = gs._lib()
    p = gb.Params()
    lib.gabe_default_params(ctypes.byref(p), N)
    p.gws_on, p.precision = 1, gb.FP64
    p0, n = gs.split_planes(N, world)[rank]
    sp = gs.SlabParams(ctypes.sizeof(gs.SlabParams), p0, n, world)
    h = ctypes.c_void_p()
    rc = lib.gabe_slab_create(ctypes.byref(p), ctypes.byref(sp), ctypes.byref(h))
    if rc == 0:  # a machine with a GPU
        assert lib.gabe_slab_destroy(h) == 0
    else:
        assert rc != 1 and not h.value, lib.gabe_slab_last_error(None)


def test_c_and_python_plane_splits_agree():
    """gabe_slab_create checks a rank's planes against the C split
    (slabsplit.h) before any CUDA call; gabe_b200.slab.split_planes is the
    Python one.  Every Python share passes that check, and a share moved by
    one plane does not."""
    lib = gs._lib()
    for N in (16, 48, 80, 112):
        for world in range(1, 8):
            for rank, (p0, n) in enumerate(gs.split_planes(N, world)):
                p = gb.Params()
                lib.gabe_default_params(ctypes.byref(p), N)
                # shares hold >= 2 planes here, so a share moved by one is never another rank's
                for q0, m, ok in ((p0, n, True), (p0 + 1, n, False)):
                    if q0 + m > N:
                        continue
                    sp = gs.SlabParams(ctypes.sizeof(gs.SlabParams), q0, m, world)
                    h = ctypes.c_void_p()
                    rc = lib.gabe_slab_create(ctypes.byref(p), ctypes.byref(sp), ctypes.byref(h))
                    if h.value:
                        lib.gabe_slab_destroy(h)
                    if ok:
                        assert rc != 1, (N, world, rank, lib.gabe_slab_last_error(None))
                    else:
                        assert rc == 1 and b"share" in lib.gabe_slab_last_error(None), (N, world, rank, q0, m)


class FakeSlab:
    """Stands in for gs.Slab: CPU tensors for the sums and boundary planes,
    and a log of the stage calls.  Its 'sweeps' put rank-dependent values in
    the sums; 'pack' writes a pattern naming the rank and the side."""

    def __init__(self, rank, plane0, nplanes, log):
        self.rank, self.plane0, self.nplanes, self.log = rank, plane0, nplanes, log
        self.t = {"sums": torch.zeros(gs.KNV, dtype=torch.float64)}
        for k in ("send_lo", "send_hi", "recv_lo", "recv_hi"):
            self.t[k] = torch.zeros(16, dtype=torch.uint8)
        self.finished = []

    def tensor(self, name):
        return self.t[name]

    def sync(self):
        pass

    def sweep(self, which):
        self.log.append(("sweep", which))
        if which in (0, 2):
            self.t["sums"][:] = torch.arange(gs.KNV, dtype=torch.float64) + 10.0 * (self.rank + 1) + which

    def finish(self, which):
        self.log.append(("finish", which))
        self.finished.append(self.t["sums"].clone())

    def pack(self):
        self.log.append(("pack",))
        self.t["send_lo"][:] = 10 * self.rank + 1
        self.t["send_hi"][:] = 10 * self.rank + 2

    def unpack(self):
        self.log.append(("unpack",))

    def gw_setup(self, world):
        """Send block for rank r': 6 floats per (own rank, destination) pair, distinct per pair."""
        self.gws = True
        self.gw_send_bytes = [4 * 6 * (r + 1) for r in range(world)]
        self.gw_recv_bytes = [4 * 6 * (self.rank + 1)] * world
        self.t["gw_send"] = torch.zeros(sum(self.gw_send_bytes) // 4, dtype=torch.float32)
        self.t["gw_recv"] = torch.full((sum(self.gw_recv_bytes) // 4,), -1.0, dtype=torch.float32)

    def gw_transform(self):
        self.log.append(("gw_transform",))
        off = 0
        for r, b in enumerate(self.gw_send_bytes):
            self.t["gw_send"][off:off + b // 4] = 100.0 * self.rank + r
            off += b // 4

    def gw_update(self):
        self.log.append(("gw_update",))

    def upload(self, f, d, mean, a0, adot0):
        self.log.append(("upload", None if mean is None else tuple(np.round(mean, 12))))

    def close(self):
        pass


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _protocol_worker(rank, world, port, N, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        log = []
        made = []

        def factory(p0, n):
            made.append(FakeSlab(rank, p0, n, log))
            return made[-1]

        lat = gs.SlabLattice(N, gs.DistComm(), precision=gb.FP32, slab_factory=factory)
        (s,) = made
        ok = lat.planes == [gs.split_planes(N, world)[rank]]
        # upload: the whole lattice's means come from the ranks' own planes
        p0, n = lat.planes[0]
        f = np.zeros((2, n, N, N))
        f[0] += 1.0 + p0  # phi differs per rank
        d = np.ones((2, n, N, N))
        lat.upload(f, d, 1.0, 0.5)
        want_phi = sum((1.0 + a) * b for a, b in gs.split_planes(N, world)) * N * N / float(N) ** 3
        ok &= log[0][0] == "upload" and abs(log[0][1][0] - want_phi) < 1e-12 and log[0][1][2] == 1.0
        log.clear()
        s.finished.clear()
        lat.step(2)
        want_log = [("sweep", 0), ("finish", 0), ("sweep", 1), ("pack",), ("unpack",)] * 2
        ok &= log == want_log
        # every rank finished with the sum over ranks of its stage sums
        tot = sum(torch.arange(gs.KNV, dtype=torch.float64) + 10.0 * (r + 1) for r in range(world))
        ok &= all(torch.equal(t, tot) for t in s.finished)
        # ring: recv_lo holds the top plane of the rank below, recv_hi the bottom plane of the rank above
        lo, hi = (rank - 1) % world, (rank + 1) % world
        ok &= bool((s.tensor("recv_lo") == 10 * lo + 2).all()) and bool((s.tensor("recv_hi") == 10 * hi + 1).all())
        q.put(bool(ok))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_slab_protocol_over_gloo_ranks(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_protocol_worker, args=(r, world, port, 24, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs)
    assert all(q.get(timeout=5) for _ in range(world))


@pytest.mark.parametrize("gws", [False, True])
def test_local_comm_protocol_with_three_slabs(gws):
    """All slabs in one process (LocalComm): every stage runs on every slab
    before the exchange that follows it, each slab finishes with the sum of
    all slabs' sums, the ring and the transpose land as over gloo."""
    world, log, made = 3, [], []

    def factory(p0, n):
        s = FakeSlab(len(made), p0, n, log)
        if gws:
            s.gw_setup(world)
        made.append(s)
        return s

    lat = gs.SlabLattice(24, gs.LocalComm(world), precision=gb.FP32, gws=gws, slab_factory=factory)
    assert lat.parts == gs.split_planes(24, world)
    lat.step(1)
    each = lambda *ev: [ev] * world  # noqa: E731
    want = each("sweep", 0) + each("finish", 0)
    if gws:
        want += each("gw_transform") + each("gw_update")
    want += each("sweep", 1) + each("pack") + each("unpack")
    assert log == want
    tot = sum(torch.arange(gs.KNV, dtype=torch.float64) + 10.0 * (r + 1) for r in range(world))
    for rank, s in enumerate(made):
        assert [torch.equal(t, tot) for t in s.finished] == [True]
        lo, hi = (rank - 1) % world, (rank + 1) % world
        assert bool((s.tensor("recv_lo") == 10 * lo + 2).all()) and bool((s.tensor("recv_hi") == 10 * hi + 1).all())
        if gws:
            recv, off = s.tensor("gw_recv"), 0
            for r, b in enumerate(s.gw_recv_bytes):
                assert bool((recv[off:off + b // 4] == 100.0 * r + rank).all())
                off += b // 4


def _gw_worker(rank, world, port, N, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        log, made = [], []

        def factory(p0, n):
            made.append(FakeSlab(rank, p0, n, log))
            made[-1].gw_setup(world)
            return made[-1]

        lat = gs.SlabLattice(N, gs.DistComm(), precision=gb.FP32, gws=True, slab_factory=factory)
        (s,) = made
        lat.step(1)
        ok = log == [("sweep", 0), ("finish", 0), ("gw_transform",), ("gw_update",), ("sweep", 1), ("pack",),
                     ("unpack",)]
        # block from source rank r sits at r's place: the value 100 r + this rank
        recv = s.tensor("gw_recv")
        off = 0
        for r, b in enumerate(s.gw_recv_bytes):
            ok &= bool((recv[off:off + b // 4] == 100.0 * r + rank).all())
            off += b // 4
        q.put(bool(ok))
    finally:
        dist.destroy_process_group()


def test_slab_gw_transpose_over_gloo_ranks():
    world = 3
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gw_worker, args=(r, world, port, 24, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs)
    assert all(q.get(timeout=5) for _ in range(world))

