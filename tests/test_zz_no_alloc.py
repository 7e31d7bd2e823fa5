"""gabe_energy_noalloc: the stage-0 energy reduction for callers that cannot
allocate device memory (their pool allocator owns it, or a cudaMalloc would
synchronise the device).  Its scratch is a fixed file-scope device array, so
the check here is that, called twice in a row through the C ABI on states
the test places in device memory, it returns what gabe_energies returns for
the same states, and that a grid larger than its scratch is refused.

Collected last on purpose (tests/test_zz_*): if it fails, every other test
has already run."""
import ctypes

import numpy as np
import pytest

import gabe_b200 as gb
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


def _tol(name, want, rho):
    # same bounds as the FP64 parity tests: 1e-12, gradient energy against rho
    return 1e-12 * (abs(rho) if name == "grad" else abs(want))


# the default tile plan, and 4x4 tiles with one plane per block (8 x 8 x 32 =
# 2048 blocks): another arm of the entry point's tile dispatch, many planes
@pytest.mark.parametrize("tile_shape,tile_ci", [(-1, 0), (5, 1)])
def test_energy_noalloc_matches_handle_energies_twice(tile_shape, tile_ci):
    import torch

    lib = gb.library()
    cfg = po.Config(N=32, model=po.MODEL_LPHI4, gws=0)
    st = po.init_state(cfg)
    first = st.copy()
    po.step(st, 20)
    c0, c1, *_ = po.model_constants(cfg.model)
    for state in (first, st):  # two calls in a row, different states
        with gb.Lattice(cfg.N, L=cfg.L, dt=cfg.dt, model=cfg.model, model_c=(c0, c1), device=0,
                        tile_shape=tile_shape, tile_ci=tile_ci) as lat:
            lat.upload_state(state.field[0], state.dfield[0], a0=state.sc.a[0], adot0=state.sc.adot[0])
            want = lat.calc_energy()
            params = lat.params
        f = torch.tensor(state.field[0], dtype=torch.float64, device="cuda")
        d = torch.tensor(state.dfield[0], dtype=torch.float64, device="cuda")
        out = torch.full((4,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        rc = lib.gabe_energy_noalloc(ctypes.byref(params), f.data_ptr(), d.data_ptr(), state.sc.a[0],
                                     out.data_ptr(), None)
        torch.cuda.synchronize()
        assert rc == 0
        got = out.cpu().numpy()
        for q, name in enumerate(("kin", "pot", "grad", "rho")):
            assert abs(got[q] - want[name]) <= _tol(name, want[name], want["rho"]), (name, got[q], want[name])


def test_energy_noalloc_refuses_grids_beyond_its_scratch():
    lib = gb.library()
    p = gb.Params()
    lib.gabe_default_params(ctypes.byref(p), 512)
    p.tile_shape, p.tile_ci = 5, 1  # 4x4 tiles, one plane per block: 8.4M blocks
    out = ctypes.c_void_p(0x1000)
    rc = lib.gabe_energy_noalloc(ctypes.byref(p), ctypes.c_void_p(0x1000), ctypes.c_void_p(0x1000), 1.0, out, None)
    assert rc == 1
