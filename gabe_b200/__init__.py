"""gabe_b200 -- B200 (sm_100a) implementation of GABE's lattice-evolution path.

The product is the C-ABI library libgabe_b200.so (include/gabe.h).  This
module is its host-side mirror for Python callers: `Lattice` wraps one
handle and exposes the reference's operations on that path under their
reference names and meanings --

    Lattice.step()          step()            g2functions.cpp:201-304
    Lattice.calc_energy()   calcEnergy(0)     g2functions.cpp:168-174
    Lattice.adf()           adf(0)            g2functions.cpp:188-191
    Lattice.spec_out()      specOut(first)    g2spectra.cpp:23-234
    Lattice.meansvars()     meansvars()       g2output.cpp:70-121

with host arrays in the reference layout (field/dfield [nflds][N][N][N],
h/l [12][N][N][N/2+1], FP64).  There is no CPU fallback: without the built
library or a CUDA device every call raises.
"""
from __future__ import annotations

import ctypes
import math
import os

import numpy as np

__all__ = [
    "GabeError", "Params", "Lattice", "library", "lib_path", "lphi4_constants",
    "FP64", "FP32", "MODEL_QUADRATIC", "MODEL_LPHI4", "numbins", "wait_probe",
]

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(HERE, "libgabe_b200.so")

FP64, FP32 = 0, 1
MODEL_QUADRATIC, MODEL_LPHI4 = 0, 1
FLAG_NO_GRAPH = 1
FLAG_NO_OVERLAP = 2
FLAG_OWN_FFT = 16
FLAG_CUFFT_3D = 64
FLAG_TRANSPOSED_FFT = 128

STATUS = {
    0: "GABE_OK", 1: "GABE_ERR_PARAM", 2: "GABE_ERR_CUDA", 3: "GABE_ERR_CUFFT", 4: "GABE_ERR_NOMEM",
    5: "GABE_ERR_NONFINITE", 6: "GABE_ERR_TIMEOUT", 7: "GABE_ERR_STATE",
}


class GabeError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


class Params(ctypes.Structure):
    _fields_ = [
        ("struct_size", ctypes.c_int32), ("N", ctypes.c_int32), ("nflds", ctypes.c_int32),
        ("gws_on", ctypes.c_int32), ("expansion", ctypes.c_int32), ("model", ctypes.c_int32),
        ("precision", ctypes.c_int32), ("gw_spec_quirk", ctypes.c_int32),
        ("L", ctypes.c_double), ("dt", ctypes.c_double), ("model_c", ctypes.c_double * 2),
        ("device", ctypes.c_int32), ("flags", ctypes.c_int32), ("tile_ci", ctypes.c_int32),
        ("tile_shape", ctypes.c_int32), ("reserved", ctypes.c_int64 * 4),
    ]


_lib = None
_dp = ctypes.POINTER(ctypes.c_double)


def lib_path() -> str:
    return _LIB_PATH


def library():
    """Loads libgabe_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        raise RuntimeError(f"{_LIB_PATH} is missing; build it with `python -m gabe_b200.build`")
    L = ctypes.CDLL(_LIB_PATH)
    H = ctypes.c_void_p
    L.gabe_default_params.argtypes = [ctypes.POINTER(Params), ctypes.c_int]
    L.gabe_default_params.restype = None
    L.gabe_create.argtypes = [ctypes.POINTER(Params), ctypes.POINTER(H)]
    L.gabe_destroy.argtypes = [H]
    L.gabe_upload_state.argtypes = [H, _dp, _dp, _dp, _dp, ctypes.c_double, ctypes.c_double]
    L.gabe_step.argtypes = [H, ctypes.c_int]
    L.gabe_sync.argtypes = [H]
    L.gabe_energies.argtypes = [H, _dp, _dp, _dp]
    L.gabe_scalars.argtypes = [H, _dp]
    L.gabe_download_state.argtypes = [H, _dp, _dp, _dp, _dp]
    L.gabe_spectra_numbins.argtypes = [ctypes.c_int]
    L.gabe_spectra.argtypes = [H, _dp, ctypes.c_int, ctypes.c_int]
    L.gabe_spectra_raw.argtypes = [H, _dp, _dp, ctypes.c_int, ctypes.c_int]
    L.gabe_meansvars.argtypes = [H, _dp]
    L.gabe_field_slice_rows.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int]
    L.gabe_field_slice_rows.restype = ctypes.c_size_t
    L.gabe_field_slice.argtypes = [H, ctypes.c_int, ctypes.c_int, _dp, ctypes.c_size_t]
    L.gabe_last_error.argtypes = [H]
    L.gabe_last_error.restype = ctypes.c_char_p
    L.gabe_device_bytes.argtypes = [H]
    L.gabe_device_bytes.restype = ctypes.c_size_t
    L.gabe_launches_per_step.argtypes = [H]
    L.gabe_graph_active.argtypes = [H]
    L.gabe_profile_steps.argtypes = [H, ctypes.c_int, _dp]
    L.gabe_profile_fft_passes.argtypes = [H, ctypes.c_int, _dp]
    L.gabe_stream.argtypes = [H, ctypes.POINTER(ctypes.c_void_p)]
    L.gabe_energy_noalloc.argtypes = [ctypes.POINTER(Params), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double,
                                      ctypes.c_void_p, ctypes.c_void_p]
    L.gabe_save_state.argtypes = [H, ctypes.c_char_p]
    L.gabe_load_state.argtypes = [H, ctypes.c_char_p, ctypes.POINTER(ctypes.c_int)]
    _lib = L
    return L


def numbins(N: int) -> int:
    return int(math.sqrt(3.0) * N / 2 + 1)


def wait_probe(limit_ns: int) -> tuple[int, int, int]:
    """gabe_wait_probe: the library's bounded device wait run on a barrier
    nothing arrives at.  Returns (return code, device status word, GPU ns
    waited); the code is 6 (GABE_ERR_TIMEOUT) when the wait gave up as
    designed."""
    L = library()
    if not getattr(L, "_probe_ready", False):
        L.gabe_wait_probe.argtypes = [ctypes.c_int64, ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_int64)]
        L._probe_ready = True
    st, w = ctypes.c_uint32(), ctypes.c_int64()
    rc = L.gabe_wait_probe(int(limit_ns), ctypes.byref(st), ctypes.byref(w))
    return rc, st.value, w.value


def lphi4_constants(g2_over_lambda: float = 100.0, phi0: float = 0.342) -> tuple[float, float]:
    """(lam_pr, gsq_pr) of V = lambda phi^4/4 + g^2 phi^2 chi^2/2 in program
    units with B = sqrt(lambda) phi0 (the reference's rescaling,
    g2model.cpp:12-18)."""
    return 1.0 / (phi0 * phi0), g2_over_lambda / (phi0 * phi0)


def _ptr(a):
    if a is None:
        return None
    if not (a.dtype == np.float64 and a.flags.c_contiguous):
        raise ValueError("arrays must be C-contiguous float64")
    return a.ctypes.data_as(_dp)


class Lattice:
    """One lattice on one GPU (a gabe_handle)."""

    def __init__(self, N: int, *, L: float = 20.0, dt: float = 0.01, gws: bool = False,
                 model: int = MODEL_LPHI4, model_c=None, precision: int = FP64, device: int = -1,
                 gw_spec_quirk: bool = True, flags: int = 0, tile_ci: int = 0, tile_shape=-1, expansion: int = 1):
        """tile_shape="auto" takes the tile the autotuner cached for this GPU,
        N, precision and GW setting (gabe_b200.autotune), if any.  expansion
        is the reference's expansion_type (g2parameters.h:62): 1 self-consistent
        Friedmann expansion, 0 none, 2 type 1 without tensor-mode evolution."""
        lib = library()
        if tile_shape == "auto":
            from .autotune import lookup

            hit = lookup(int(N), int(precision), bool(gws))
            tile_shape, tile_ci = hit if hit else (-1, tile_ci)
        p = Params()
        lib.gabe_default_params(ctypes.byref(p), int(N))
        p.L, p.dt, p.gws_on, p.model, p.precision = float(L), float(dt), int(bool(gws)), int(model), int(precision)
        if model_c is None:
            model_c = lphi4_constants() if model == MODEL_LPHI4 else (1e-6, 2.5e-7)
        p.model_c[0], p.model_c[1] = float(model_c[0]), float(model_c[1])
        p.device, p.gw_spec_quirk, p.flags = int(device), int(bool(gw_spec_quirk)), int(flags)
        p.tile_ci, p.tile_shape = int(tile_ci), int(tile_shape)
        p.expansion = int(expansion)
        self.params = p
        self.N, self.gws, self.precision = int(N), bool(gws), int(precision)
        self.nz = self.N // 2 + 1
        self._h = ctypes.c_void_p()
        rc = lib.gabe_create(ctypes.byref(p), ctypes.byref(self._h))
        if rc != 0:
            msg = lib.gabe_last_error(None).decode()
            self._h = None
            raise GabeError(rc, msg)

    # -- plumbing ---------------------------------------------------------
    def _check(self, rc: int):
        if rc != 0:
            raise GabeError(rc, library().gabe_last_error(self._h).decode())

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            library().gabe_destroy(self._h)
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
    def device_bytes(self) -> int:
        return library().gabe_device_bytes(self._h)

    @property
    def launches_per_step(self) -> int:
        return library().gabe_launches_per_step(self._h)

    @property
    def graph_active(self) -> int:
        """1: steps replay the captured CUDA graphs; 0: direct launches; -1: before the first step."""
        return library().gabe_graph_active(self._h)

    # -- state ------------------------------------------------------------
    def upload_state(self, field0, dfield0, h0=None, l0=None, *, a0: float = 1.0, adot0: float):
        N = self.N
        f = np.ascontiguousarray(field0, dtype=np.float64).reshape(2, N, N, N)
        d = np.ascontiguousarray(dfield0, dtype=np.float64).reshape(2, N, N, N)
        hh = ll = None
        if self.gws:
            if h0 is not None:
                hh = np.ascontiguousarray(h0, dtype=np.float64).reshape(12, N, N, self.nz)
            if l0 is not None:
                ll = np.ascontiguousarray(l0, dtype=np.float64).reshape(12, N, N, self.nz)
        self._check(library().gabe_upload_state(self._h, _ptr(f), _ptr(d), _ptr(hh), _ptr(ll), a0, adot0))

    def upload_ptrs(self, field0: int, dfield0: int, h0: int | None, l0: int | None, a0: float, adot0: float):
        """Upload from raw host addresses (e.g. pinned buffers)."""
        c = lambda v: ctypes.cast(ctypes.c_void_p(v), _dp) if v else None
        self._check(library().gabe_upload_state(self._h, c(field0), c(dfield0), c(h0), c(l0), a0, adot0))

    def download_state(self, want_gw: bool = True):
        N = self.N
        f = np.empty((2, N, N, N))
        d = np.empty((2, N, N, N))
        hh = ll = None
        if self.gws and want_gw:
            hh = np.empty((12, N, N, self.nz))
            ll = np.empty((12, N, N, self.nz))
        self._check(library().gabe_download_state(self._h, _ptr(f), _ptr(d), _ptr(hh), _ptr(ll)))
        return f, d, hh, ll

    def download_ptrs(self, field0: int, dfield0: int, h0: int | None = None, l0: int | None = None):
        c = lambda v: ctypes.cast(ctypes.c_void_p(v), _dp) if v else None
        self._check(library().gabe_download_state(self._h, c(field0), c(dfield0), c(h0), c(l0)))

    # -- hot path ---------------------------------------------------------
    def step(self, n: int = 1):
        self._check(library().gabe_step(self._h, int(n)))

    def profile_steps(self, n: int) -> dict:
        """Mean ms per step of each phase (direct launches with CUDA events)."""
        out = (ctypes.c_double * 4)()
        self._check(library().gabe_profile_steps(self._h, int(n), out))
        return {"stage1": out[0], "fft": out[1], "kspace": out[2], "stage2": out[3]}

    def profile_fft_passes(self, n: int) -> dict:
        """Mean ms of each pass of the library's own transforms (raises
        GabeError GABE_ERR_STATE for a handle that uses cuFFT's plan).  The
        three-pass 3-D FFT: {fft_rows, fft_j, fft_i}, run on the source buffer.
        The transposed form (FLAG_TRANSPOSED_FFT): {fft_rows, fft_j,
        fft_i_kspace}, timed inside n full steps (the state advances n steps)."""
        out = (ctypes.c_double * 3)()
        self._check(library().gabe_profile_fft_passes(self._h, int(n), out))
        last = "fft_i_kspace" if self.launches_per_step == 5 else "fft_i"  # 5: the transposed form
        return {"fft_rows": out[0], "fft_j": out[1], last: out[2]}

    @property
    def stream_ptr(self) -> int:
        s = ctypes.c_void_p()
        self._check(library().gabe_stream(self._h, ctypes.byref(s)))
        return s.value or 0

    def sync(self):
        self._check(library().gabe_sync(self._h))

    def calc_energy(self) -> dict:
        e = (ctypes.c_double * 4)()
        a = ctypes.c_double()
        ad = ctypes.c_double()
        self._check(library().gabe_energies(self._h, e, ctypes.byref(a), ctypes.byref(ad)))
        return {"kin": e[0], "pot": e[1], "grad": e[2], "rho": e[3], "a": a.value, "adot": ad.value}

    energies = calc_energy

    def adf(self) -> float:
        return self.calc_energy()["adot"]

    def scalars(self) -> dict:
        out = (ctypes.c_double * 12)()
        self._check(library().gabe_scalars(self._h, out))
        names = ("a", "adot", "edkin", "edpot", "edgrad", "edrho")
        return {n: (out[2 * i], out[2 * i + 1]) for i, n in enumerate(names)}

    # -- checkpoint / restart ---------------------------------------------
    def save(self, path: str) -> None:
        """Checkpoint to a gabe_dump.h file with the library's restart block
        (gabe_save_state)."""
        self._check(library().gabe_save_state(self._h, os.fsencode(path)))

    def load(self, path: str) -> bool:
        """Loads a gabe_dump.h file (gabe_load_state): True when its restart
        block became the state (bit-exact continuation), False when its FP64
        arrays were uploaded as an initial state."""
        restored = ctypes.c_int(0)
        self._check(library().gabe_load_state(self._h, os.fsencode(path), ctypes.byref(restored)))
        return bool(restored.value)

    # -- analysis ---------------------------------------------------------
    def spec_out(self) -> np.ndarray:
        nb = numbins(self.N)
        nc = 8 if self.gws else 5
        out = np.zeros((nb, nc))
        self._check(library().gabe_spectra(self._h, _ptr(out), nb, nc))
        return out

    spectra = spec_out

    def spectra_raw(self):
        nb = numbins(self.N)
        ns = 3 if self.gws else 2
        sums = np.zeros((ns, nb))
        cnt = np.zeros(nb)
        self._check(library().gabe_spectra_raw(self._h, _ptr(sums), _ptr(cnt), nb, ns))
        return sums, cnt

    def meansvars(self) -> np.ndarray:
        """Mean and variance of each field (meansvars, g2output.cpp:70-121),
        reduced on the device: rows (mean, var) per field.  Raises
        GabeError(GABE_ERR_NONFINITE) where the reference would exit(1)."""
        out = np.zeros(4)
        self._check(library().gabe_meansvars(self._h, _ptr(out)))
        return out.reshape(2, 2)

    def field_slice(self, outdim: int = 2, skip: int = 2) -> np.ndarray:
        """The rows outputfield (g2output.cpp:25-68) writes for field_outdim
        `outdim` and field_sliceskip `skip`: (phi, chi, calcrho) per sampled
        point, in the reference's loop order, computed on the device."""
        rows = library().gabe_field_slice_rows(self.N, int(outdim), int(skip))
        out = np.zeros((rows, 3))
        self._check(library().gabe_field_slice(self._h, int(outdim), int(skip), _ptr(out), out.size))
        return out


class EnsParams(ctypes.Structure):
    _fields_ = [
        ("struct_size", ctypes.c_int32), ("nlat", ctypes.c_int32),
        ("N", ctypes.POINTER(ctypes.c_int32)), ("g2_over_lambda", ctypes.POINTER(ctypes.c_double)),
        ("amplitude", ctypes.POINTER(ctypes.c_double)), ("seed", ctypes.POINTER(ctypes.c_uint64)),
        ("tile_shape", ctypes.POINTER(ctypes.c_int32)), ("tile_ci", ctypes.POINTER(ctypes.c_int32)),
        ("L", ctypes.c_double), ("dt", ctypes.c_double),
        ("lam", ctypes.c_double), ("phi0", ctypes.c_double), ("dphi0", ctypes.c_double),
        ("gws_on", ctypes.c_int32), ("device", ctypes.c_int32), ("nlog", ctypes.c_int32),
        ("gw_spec_quirk", ctypes.c_int32), ("flags", ctypes.c_int32), ("log_top_bin", ctypes.c_int32),
        ("spec_cut_off", ctypes.c_double), ("spec_smooth", ctypes.c_double),
        ("ic_deterministic", ctypes.c_int32), ("reserved", ctypes.c_int32),
    ]


def _ens_lib():
    L = library()
    if not getattr(L, "_ens_ready", False):
        E = ctypes.c_void_p
        L.gabe_ensemble_create.argtypes = [ctypes.POINTER(EnsParams), ctypes.POINTER(E)]
        L.gabe_ensemble_destroy.argtypes = [E]
        L.gabe_ensemble_init.argtypes = [E]
        L.gabe_ensemble_upload.argtypes = [E, ctypes.c_int, _dp, _dp, ctypes.c_double, ctypes.c_double]
        L.gabe_ensemble_step.argtypes = [E, ctypes.c_int]
        L.gabe_ensemble_sync.argtypes = [E]
        L.gabe_ensemble_scalars.argtypes = [E, _dp]
        L.gabe_ensemble_native_bins.argtypes = [E]
        L.gabe_ensemble_log_spectra.argtypes = [E, _dp, _dp, _dp]
        L.gabe_ensemble_download.argtypes = [E, ctypes.c_int, _dp, _dp, _dp, _dp]
        L.gabe_ensemble_last_error.argtypes = [E]
        L.gabe_ensemble_last_error.restype = ctypes.c_char_p
        L.gabe_ensemble_device_bytes.argtypes = [E]
        L.gabe_ensemble_device_bytes.restype = ctypes.c_size_t
        L.gabe_ensemble_stream.argtypes = [E]
        L.gabe_ensemble_stream.restype = ctypes.c_void_p
        L.gabe_ensemble_launches_per_step.argtypes = [E]
        L.gabe_ensemble_graph_active.argtypes = [E]
        L._ens_ready = True
    return L


class Ensemble:
    """Many independent lattices evolved together (gabe_ensemble_*): FP32
    storage, FP64 scalars, the lambda phi^4 + g^2 phi^2 chi^2 model with a
    per-lattice g^2/lambda, fluctuation amplitude multiplier and seed."""

    def __init__(self, N, g2_over_lambda, amplitude, seed, *, L: float = 20.0, dt: float = 0.01,
                 lam: float = 9e-14, phi0: float = 0.342, dphi0: float = 0.0, gws: bool = True, nlog: int = 64,
                 tiles="auto", device: int = -1, flags: int = 0, gw_spec_quirk: bool = True, log_top_bin: int = 0,
                 spec_cut_off: float | None = None, spec_smooth: float = 0.5, full_rand: bool = True):
        lib = _ens_lib()
        self.N = np.ascontiguousarray(N, dtype=np.int32)
        self.nlat = len(self.N)
        self._g = np.ascontiguousarray(g2_over_lambda, dtype=np.float64)
        self._amp = np.ascontiguousarray(amplitude, dtype=np.float64)
        self._seed = np.ascontiguousarray(seed, dtype=np.uint64)
        self.gws, self.nlog = bool(gws), int(nlog)
        shapes = cis = None
        if tiles == "auto":
            from .autotune import lookup_ensemble

            st = [lookup_ensemble(int(n)) for n in self.N]
            if all(t is not None for t in st):
                shapes = np.array([t[0] for t in st], dtype=np.int32)
                cis = np.array([t[1] for t in st], dtype=np.int32)
        elif tiles is not None:
            shapes = np.ascontiguousarray(tiles[0], dtype=np.int32)
            cis = np.ascontiguousarray(tiles[1], dtype=np.int32)
        self._shapes, self._cis = shapes, cis
        p = EnsParams()
        p.struct_size = ctypes.sizeof(EnsParams)
        p.nlat = self.nlat
        p.N = self.N.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
        p.g2_over_lambda = self._g.ctypes.data_as(_dp)
        p.amplitude = self._amp.ctypes.data_as(_dp)
        p.seed = self._seed.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))
        if shapes is not None:
            p.tile_shape = shapes.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
            p.tile_ci = cis.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
        p.L, p.dt, p.lam, p.phi0, p.dphi0 = L, dt, lam, phi0, dphi0
        p.gws_on, p.device, p.nlog, p.gw_spec_quirk, p.flags = int(gws), device, nlog, int(gw_spec_quirk), flags
        p.log_top_bin = int(log_top_bin)
        # the reference's spec_cut_off / spec_smooth / field_full_rand (as gabe_b200.ic.random_state)
        p.spec_cut_off = float(spec_cut_off) if spec_cut_off is not None else 0.0
        p.spec_smooth = float(spec_smooth)
        p.ic_deterministic = 0 if full_rand else 1
        self._p = p
        self._h = ctypes.c_void_p()
        rc = lib.gabe_ensemble_create(ctypes.byref(p), ctypes.byref(self._h))
        if rc != 0:
            self._h = None
            raise GabeError(rc, lib.gabe_ensemble_last_error(None).decode())
        self.nb = lib.gabe_ensemble_native_bins(self._h)

    def _check(self, rc):
        if rc != 0:
            raise GabeError(rc, _ens_lib().gabe_ensemble_last_error(self._h).decode())

    def close(self):
        if self._h:
            _ens_lib().gabe_ensemble_destroy(self._h)
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
    def device_bytes(self) -> int:
        return _ens_lib().gabe_ensemble_device_bytes(self._h)

    @property
    def stream_ptr(self) -> int:
        return _ens_lib().gabe_ensemble_stream(self._h) or 0

    @property
    def launches_per_step(self) -> int:
        return _ens_lib().gabe_ensemble_launches_per_step(self._h)

    @property
    def graph_active(self) -> int:
        """1: steps replay the captured CUDA graph; 0: direct launches; -1: before the first step."""
        return _ens_lib().gabe_ensemble_graph_active(self._h)

    def init(self):
        self._check(_ens_lib().gabe_ensemble_init(self._h))

    def upload(self, lat: int, field0, dfield0, *, a0: float = 1.0, adot0: float):
        """Replaces lattice `lat`'s state (gabe_ensemble_upload); init() must
        have drawn every lattice's state first (GabeError GABE_ERR_STATE)."""
        n = int(self.N[lat])
        f = np.ascontiguousarray(field0, dtype=np.float64).reshape(2, n, n, n)
        d = np.ascontiguousarray(dfield0, dtype=np.float64).reshape(2, n, n, n)
        self._check(_ens_lib().gabe_ensemble_upload(self._h, int(lat), _ptr(f), _ptr(d), a0, adot0))

    def step(self, n: int = 1):
        self._check(_ens_lib().gabe_ensemble_step(self._h, int(n)))

    def sync(self):
        self._check(_ens_lib().gabe_ensemble_sync(self._h))

    def scalars(self) -> np.ndarray:
        """[nlat][12]: a[0], a[1], adot[0], adot[1], edkin[0..1], edpot, edgrad, edrho."""
        out = np.zeros((self.nlat, 12))
        self._check(_ens_lib().gabe_ensemble_scalars(self._h, _ptr(out)))
        return out

    def log_spectra(self):
        logs = np.zeros((self.nlat, 3, self.nlog))
        cnt = np.zeros((self.nlat, self.nlog))
        nat = np.zeros((self.nlat, 4, self.nb))
        self._check(_ens_lib().gabe_ensemble_log_spectra(self._h, _ptr(logs), _ptr(cnt), _ptr(nat)))
        return logs, cnt, nat

    def download(self, lat: int, want_gw: bool = True):
        n = int(self.N[lat])
        f = np.empty((2, n, n, n))
        d = np.empty((2, n, n, n))
        hh = ll = None
        if self.gws and want_gw:
            hh = np.empty((12, n, n, n // 2 + 1))
            ll = np.empty((12, n, n, n // 2 + 1))
        self._check(_ens_lib().gabe_ensemble_download(self._h, int(lat), _ptr(f), _ptr(d), _ptr(hh), _ptr(ll)))
        return f, d, hh, ll


def rebin_log(native: np.ndarray, N: int, nlog: int, nb_max: int, L: float, rho0: float) -> np.ndarray:
    """Log-binned (Delta^2_phi, Delta^2_chi, Omega_gw) from native bin sums
    and counts -- the rule of gabe_ensemble_log_spectra, for checks and for
    single lattices (use gabe_spectra_raw's sums/counts as `native`
    [4][nb]: phi, chi, GW sums and counts)."""
    nbe = int(math.sqrt(3.0) * N / 2 + 1)
    spec_norm = (L / N) ** 6 * (2 * math.pi / L) ** 3
    hub = math.sqrt(8 * math.pi / 3) * math.sqrt(rho0)
    norm1 = 4.e-5 / 100. ** .333 / 24. / math.pi / math.pi / L ** 3 / hub ** 2
    out = np.full((3, nlog), np.nan)
    cnt = np.zeros(nlog)
    lo, hi = 1.0, float(nb_max)
    for q in range(nlog):
        e0 = lo * (hi / lo) ** (q / nlog)
        e1 = lo * (hi / lo) ** ((q + 1) / nlog)
        bs = [b for b in range(1, nbe) if b >= e0 and (b < e1 if q + 1 < nlog else b <= e1)]
        n = sum(native[3][b] for b in bs)
        cnt[q] = n
        if n > 0:
            k3 = [(b * 2 * math.pi / L) ** 3 for b in bs]
            s = [sum(k * native[c][b] for k, b in zip(k3, bs)) for c in range(3)]
            with np.errstate(divide="ignore"):
                out[0, q] = np.log10(spec_norm * s[0] / n / 2 / math.pi / math.pi)
                out[1, q] = np.log10(spec_norm * s[1] / n / 2 / math.pi / math.pi)
                out[2, q] = np.log10(norm1 * s[2] / n)
    return out, cnt
