"""Host-side reader of gabe_dump.h files: the reference-layout state dumps
(written by the reference harness, the oracle and gabe_save_state) and the
restart block that gabe_save_state appends.

The reference itself has no restartable output -- its field slices are
sampled %e text (g2output.cpp:25-68) -- so this format carries its full
state: field[0], dfield[0] (g2header.h:54-55), h[0], l[0]
(g2header.h:171-172) and the per-stage scalars a, adot, edkin, edpot,
edgrad, edrho (g2header.h:58-63)."""
from __future__ import annotations

import struct

import numpy as np

DUMP_MAGIC = b"GABEDMP1"
RESTART_MAGIC = b"GABERST1"
_HDR = struct.Struct("<8s6iqddd12d96x")           # gabe_dump_header, 256 bytes
_RST = struct.Struct("<8s8iqq72x")                # gabe_restart_header, 128 bytes
assert _HDR.size == 256 and _RST.size == 128
SCALAR_NAMES = ("a", "adot", "edkin", "edpot", "edgrad", "edrho")


def read_header(path: str) -> dict:
    with open(path, "rb") as fh:
        raw = fh.read(_HDR.size)
    if len(raw) != _HDR.size:
        raise ValueError(f"{path}: shorter than a dump header")
    magic, ver, N, nflds, gws, eb, model, step, t, L, dt, *v = _HDR.unpack(raw)
    if magic != DUMP_MAGIC or ver != 1 or eb != 8:
        raise ValueError(f"{path} is not a gabe_dump.h state dump")
    sc = {name: (v[2 * i], v[2 * i + 1]) for i, name in enumerate(SCALAR_NAMES)}
    return {"N": N, "nflds": nflds, "gws": gws, "model": model, "step": step, "t": t, "L": L, "dt": dt,
            "scalars": sc}


def _payload_bytes(hd: dict) -> int:
    N = hd["N"]
    nf = hd["nflds"] * N ** 3
    ng = 12 * N * N * (N // 2 + 1)
    return 8 * (2 * nf + (2 * ng if hd["gws"] else 0))


def read_state(path: str) -> dict:
    """The FP64 arrays in the reference's layout: field, dfield
    [nflds][N][N][N] and, with GWs, h, l [12][N][N][N/2+1]."""
    hd = read_header(path)
    N, nfl = hd["N"], hd["nflds"]
    out = dict(hd)
    shapes = [("field", (nfl, N, N, N)), ("dfield", (nfl, N, N, N))]
    if hd["gws"]:
        shapes += [("h", (12, N, N, N // 2 + 1)), ("l", (12, N, N, N // 2 + 1))]
    with open(path, "rb") as fh:
        fh.seek(_HDR.size)
        for name, shape in shapes:
            want = int(np.prod(shape))
            arr = np.fromfile(fh, np.float64, want)
            if arr.size != want:
                raise ValueError(f"{path} is truncated: {name} holds {arr.size} of {want} values")
            out[name] = arr.reshape(shape)
    return out


def read_restart_header(path: str) -> dict | None:
    """The restart block's header, or None for a dump without one (such as
    the reference harness's)."""
    hd = read_header(path)
    with open(path, "rb") as fh:
        fh.seek(_HDR.size + _payload_bytes(hd))
        raw = fh.read(_RST.size)
    if len(raw) != _RST.size:
        return None
    magic, prec, layout, expansion, shape, ci, stale, sbytes, eb, fbytes, gbytes = _RST.unpack(raw)
    if magic != RESTART_MAGIC:
        return None
    return {"precision": prec, "gw_layout": layout, "expansion": expansion, "tile_shape": shape, "tile_ci": ci,
            "e0_stale": stale, "scalar_bytes": sbytes, "elem_bytes": eb, "field_bytes": fbytes, "gw_bytes": gbytes}
