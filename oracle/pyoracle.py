"""ctypes binding of liboracle.so (the CPU restatement) -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg import
this module, and only as the checker.  It also reads/writes the binary state
dumps (include/gabe_dump.h) and runs the reference binaries under
oracle/_ref when they exist.
"""
from __future__ import annotations

import ctypes
import math
import os
import struct
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

MODEL_QUADRATIC = 0
MODEL_LPHI4 = 1

# Physical constants of the two models (oracle/ref_cfg/g2parameters.h).
LPHI4 = dict(lambda_phys=9e-14, g2_over_lambda=100.0, phi0=0.342, dphi0=0.0)
QUAD = dict(mphi=1e-6, phi0=0.193, gsq=2.5e-7, dphi0=-0.142231)


class _Params(ctypes.Structure):
    _fields_ = [
        ("N", ctypes.c_int), ("nflds", ctypes.c_int),
        ("L", ctypes.c_double), ("dt", ctypes.c_double),
        ("model", ctypes.c_int), ("gws", ctypes.c_int),
        ("gw_spec_quirk", ctypes.c_int), ("expansion", ctypes.c_int),
        ("mc", ctypes.c_double * 6),
        ("ic_variant", ctypes.c_int), ("ic_pad", ctypes.c_int),
        ("spec_cut", ctypes.c_double), ("spec_smooth", ctypes.c_double),
    ]


class _Scalars(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double * 2) for n in ("a", "adot", "edkin", "edpot", "edgrad", "edrho")]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} missing: run `make -C oracle`")
        L = ctypes.CDLL(LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        P = ctypes.POINTER(_Params)
        S = ctypes.POINTER(_Scalars)
        L.ora_model_constants.argtypes = [P, ctypes.c_double, ctypes.c_double]
        L.ora_potential.argtypes = [P, ctypes.c_double, ctypes.c_double]
        L.ora_potential.restype = ctypes.c_double
        L.ora_dvdf.argtypes = [P, ctypes.c_int, ctypes.c_double, ctypes.c_double]
        L.ora_dvdf.restype = ctypes.c_double
        L.ora_calc_energy.argtypes = [P, dp, dp, ctypes.c_double, dp]
        L.ora_adf.argtypes = [ctypes.c_double, ctypes.c_double]
        L.ora_adf.restype = ctypes.c_double
        L.ora_init.argtypes = [P, ctypes.c_int, dp, dp, ctypes.c_double, dp, dp, S]
        L.ora_step.argtypes = [P, dp, dp, dp, dp, dp, S]
        L.ora_fft_stresstensor.argtypes = [P, dp, dp]
        L.ora_tt_point.argtypes = [ctypes.POINTER(ctypes.c_int), ctypes.c_double, dp, dp]
        L.ora_spectra_numbins.argtypes = [ctypes.c_int]
        L.ora_spectra_numbins.restype = ctypes.c_int
        L.ora_spectra.argtypes = [P, dp, dp, ctypes.c_double, dp]
        L.ora_spectra.restype = ctypes.c_int
        L.fftw_plan_with_nthreads.argtypes = [ctypes.c_int]
        _lib = L
    return _lib


def _dp(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def model_constants(model: int):
    """(c0, c1, rescale_B, f0, df0) for the oracle models."""
    if model == MODEL_QUADRATIC:
        q = QUAD
        return q["mphi"], q["gsq"], q["mphi"], (q["phi0"], 0.0), (q["dphi0"], 0.0)
    m = LPHI4
    phi0 = m["phi0"]
    lam_pr = 1.0 / (phi0 * phi0)
    gsq_pr = m["g2_over_lambda"] / (phi0 * phi0)
    B = math.sqrt(m["lambda_phys"]) * phi0
    return lam_pr, gsq_pr, B, (phi0, 0.0), (m["dphi0"], 0.0)


@dataclass
class Config:
    N: int
    L: float = 20.0
    dt: float = 0.01
    model: int = MODEL_LPHI4
    gws: int = 0
    gw_spec_quirk: int = 1
    expansion: int = 1  # expansion_type (g2parameters.h:62)
    ic_variant: int = 0  # 0 field_full_rand 1; 1 with spec_cut_off; 2 field_full_rand 0 (g2init.cpp:117-165)
    spec_cut: float = math.sqrt(3.) / 8.  # spec_cut_off, spec_smooth (the reference's g2parameters.h:73-74)
    spec_smooth: float = 0.5

    def params(self) -> _Params:
        p = _Params()
        p.N, p.nflds, p.L, p.dt = self.N, 2, self.L, self.dt
        p.model, p.gws, p.gw_spec_quirk = self.model, self.gws, self.gw_spec_quirk
        p.expansion = self.expansion
        p.ic_variant, p.spec_cut, p.spec_smooth = self.ic_variant, self.spec_cut, self.spec_smooth
        c0, c1, *_ = model_constants(self.model)
        lib().ora_model_constants(ctypes.byref(p), c0, c1)
        return p


@dataclass
class State:
    """Reference-layout FP64 state: both RK2 stages, like g2main.cpp:49-99."""
    cfg: Config
    field: np.ndarray
    dfield: np.ndarray
    h: np.ndarray | None
    l: np.ndarray | None
    sc: _Scalars = field(default_factory=_Scalars)
    step: int = 0

    @staticmethod
    def empty(cfg: Config) -> "State":
        N = cfg.N
        f = np.zeros((2, 2, N, N, N))
        d = np.zeros((2, 2, N, N, N))
        h = l = None
        if cfg.gws:
            h = np.zeros((2, 12, N, N, N // 2 + 1))
            l = np.zeros((2, 12, N, N, N // 2 + 1))
        return State(cfg, f, d, h, l)

    def scalars(self, s: int = 0) -> dict:
        return {k: getattr(self.sc, k)[s] for k in ("a", "adot", "edkin", "edpot", "edgrad", "edrho")}

    def copy(self) -> "State":
        st = State(self.cfg, self.field.copy(), self.dfield.copy(),
                   None if self.h is None else self.h.copy(),
                   None if self.l is None else self.l.copy(), step=self.step)
        ctypes.memmove(ctypes.byref(st.sc), ctypes.byref(self.sc), ctypes.sizeof(_Scalars))
        return st


def init_state(cfg: Config, seed: int = 44463132) -> State:
    """The reference's initialisation sequence (see ora_init)."""
    st = State.empty(cfg)
    c0, c1, B, f0, df0 = model_constants(cfg.model)
    p = cfg.params()
    f0a = (ctypes.c_double * 2)(*f0)
    df0a = (ctypes.c_double * 2)(*df0)
    lib().ora_init(ctypes.byref(p), seed, f0a, df0a, B, _dp(st.field), _dp(st.dfield), ctypes.byref(st.sc))
    return st


def step(st: State, n: int = 1, T_gw: np.ndarray | None = None) -> State:
    p = st.cfg.params()
    if st.cfg.gws and T_gw is None:
        N = st.cfg.N
        T_gw = np.zeros((2, 12, N, N, N // 2 + 1))
    for _ in range(n):
        lib().ora_step(ctypes.byref(p), _dp(st.field), _dp(st.dfield), _dp(st.h), _dp(st.l),
                       _dp(T_gw), ctypes.byref(st.sc))
        st.step += 1
    return st


def calc_energy(cfg: Config, f: np.ndarray, df: np.ndarray, a: float) -> np.ndarray:
    out = np.zeros(4)
    f = np.ascontiguousarray(f, dtype=np.float64)
    df = np.ascontiguousarray(df, dtype=np.float64)
    lib().ora_calc_energy(ctypes.byref(cfg.params()), _dp(f), _dp(df), a, _dp(out))
    return out


def adf(rho: float, a: float) -> float:
    return lib().ora_adf(rho, a)


def fft_stresstensor(cfg: Config, f_stage: np.ndarray) -> np.ndarray:
    N = cfg.N
    T = np.zeros((12, N, N, N // 2 + 1))
    f_stage = np.ascontiguousarray(f_stage, dtype=np.float64)
    lib().ora_fft_stresstensor(ctypes.byref(cfg.params()), _dp(f_stage), _dp(T))
    return T


def tt_point(n, nm: float, S: np.ndarray) -> np.ndarray:
    nn = (ctypes.c_int * 3)(*[int(v) for v in n])
    S = np.ascontiguousarray(S, dtype=np.float64)
    T = np.zeros(12)
    lib().ora_tt_point(nn, nm, _dp(S), _dp(T))
    return T


def numbins(N: int) -> int:
    return lib().ora_spectra_numbins(N)


def spectra(cfg: Config, field0: np.ndarray, l0: np.ndarray | None, edrho0: float) -> np.ndarray:
    nb = numbins(cfg.N)
    ncol = 1 + 4 + (3 if cfg.gws else 0)
    out = np.zeros((nb, ncol))
    field0 = np.ascontiguousarray(field0, dtype=np.float64)
    l0c = None if l0 is None else np.ascontiguousarray(l0, dtype=np.float64)
    lib().ora_spectra(ctypes.byref(cfg.params()), _dp(field0), _dp(l0c), edrho0, _dp(out))
    return out


def meansvars(field0: np.ndarray) -> np.ndarray:
    """meansvars (g2output.cpp:70-121): rows (mean, variance) per field, the
    variance as the reference forms it, sum(f^2 - mean^2) / N^3 (numpy's sum
    order, not the reference's serial one)."""
    out = np.zeros((field0.shape[0], 2))
    for q in range(field0.shape[0]):
        f = field0[q]
        av = f.sum() / f.size
        out[q] = av, (f * f - av * av).sum() / f.size
    return out


def _potential(cfg: Config, P: np.ndarray, C: np.ndarray) -> np.ndarray:
    """potential (g2model.cpp:66-69; lphi4 in ref_cfg/g2model_lphi4.cpp), operation order kept."""
    mc = list(cfg.params().mc)
    if cfg.model == MODEL_QUADRATIC:
        return 0.5 * P * P + mc[1] * P * P * C * C
    return mc[2] * P * P * P * P + mc[3] * P * P * C * C


def field_slice(cfg: Config, field0: np.ndarray, dfield0: np.ndarray, a0: float, outdim: int, skip: int) -> np.ndarray:
    """The rows outputfield (g2output.cpp:25-68) writes: per sampled point
    (i stepping by skip if outdim > 2 else 0, j likewise if outdim > 1, k),
    the two field values and calcrho(0, i, j, k) (g2functions.cpp:176-186)
    with the fourth-order gradients dfdi/dfdj/dfdk (:70-98) and gradF2
    (:118-122), each in the reference's operation order."""
    N = cfg.N
    dx = cfg.L / float(N)

    def d4(f, axis):
        r = lambda s: np.roll(f, s, axis=axis)  # r(2)[i] = f[i-2]
        return ((1. / 12.) * r(2) + ((-2.) / 3.) * r(1) + (2. / 3.) * r(-1) + ((-1.) / 12.) * r(-2)) / dx

    rho = _potential(cfg, field0[0], field0[1])
    for q in range(2):
        gi, gj, gk = d4(field0[q], 0), d4(field0[q], 1), d4(field0[q], 2)
        g2 = gi * gi + gj * gj + gk * gk
        rho = rho + (.5 * dfield0[q] * dfield0[q] + .5 * g2 / a0 / a0)
    ii = range(0, N, skip) if outdim > 2 else [0]
    jj = range(0, N, skip) if outdim > 1 else [0]
    kk = range(0, N, skip)
    rows = [(field0[0, i, j, k], field0[1, i, j, k], rho[i, j, k]) for i in ii for j in jj for k in kk]
    return np.array(rows)


# ---------------------------------------------------------------------------
# binary dumps (include/gabe_dump.h)
# ---------------------------------------------------------------------------
_HDR = struct.Struct("<8s6iqddd12d96x")
assert _HDR.size == 256


def write_dump(path: str, st: State, s: int = 0) -> None:
    cfg = st.cfg
    sc = st.sc
    vals = []
    for name in ("a", "adot", "edkin", "edpot", "edgrad", "edrho"):
        vals += [getattr(sc, name)[0], getattr(sc, name)[1]]
    hdr = _HDR.pack(b"GABEDMP1", 1, cfg.N, 2, cfg.gws, 8, cfg.model, st.step, 0.0, cfg.L, cfg.dt, *vals)
    with open(path, "wb") as fh:
        fh.write(hdr)
        fh.write(np.ascontiguousarray(st.field[s]).tobytes())
        fh.write(np.ascontiguousarray(st.dfield[s]).tobytes())
        if cfg.gws:
            fh.write(np.ascontiguousarray(st.h[s]).tobytes())
            fh.write(np.ascontiguousarray(st.l[s]).tobytes())


def read_dump(path: str, cfg: Config | None = None) -> State:
    with open(path, "rb") as fh:
        raw = fh.read()
    magic, ver, N, nflds, gws, eb, model, stepn, t, L, dt, *v = _HDR.unpack_from(raw, 0)
    assert magic == b"GABEDMP1" and ver == 1 and eb == 8 and nflds == 2
    if cfg is None:
        cfg = Config(N=N, L=L, dt=dt, model=model, gws=gws)
    st = State.empty(cfg)
    off = 256
    n3 = N ** 3
    st.field[0] = np.frombuffer(raw, np.float64, 2 * n3, off).reshape(2, N, N, N); off += 16 * n3
    st.dfield[0] = np.frombuffer(raw, np.float64, 2 * n3, off).reshape(2, N, N, N); off += 16 * n3
    if gws:
        M = 12 * N * N * (N // 2 + 1)
        hh = np.frombuffer(raw, np.float64, M, off).reshape(12, N, N, N // 2 + 1); off += 8 * M
        ll = np.frombuffer(raw, np.float64, M, off).reshape(12, N, N, N // 2 + 1); off += 8 * M
        if cfg.gws:
            st.h[0] = hh
            st.l[0] = ll
    for i, name in enumerate(("a", "adot", "edkin", "edpot", "edgrad", "edrho")):
        getattr(st.sc, name)[0] = v[2 * i]
        getattr(st.sc, name)[1] = v[2 * i + 1]
    st.step = stepn
    return st


def ref_binary(model: int, N: int, gws: int, parallel: int, expansion: int = 1, ic_variant: int = 0) -> str:
    suffix = ("" if expansion == 1 else f"_e{expansion}") + ("", "_rc", "_rd")[ic_variant]
    return os.path.join(REF_DIR, f"ref_m{model}_n{N}_g{gws}_p{parallel}{suffix}")


def run_ref(binary: str, args: list[str], cwd: str, threads: int | None = None, timeout: float = 600) -> str:
    env = dict(os.environ)
    if threads is not None:
        env["GABE_REF_THREADS"] = str(threads)
    os.makedirs(os.path.join(cwd, "slices"), exist_ok=True)
    r = subprocess.run([binary] + args, cwd=cwd, env=env, capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"{binary} failed ({r.returncode}): {r.stderr[-2000:]}")
    return r.stdout
