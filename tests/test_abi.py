"""The C-ABI library: it loads, exports every entry point include/*.h
declares, and rejects bad input before touching a GPU.  No compute calls
here -- those are the gpu-marked tests."""
import ctypes
import glob
import os
import re
import subprocess

import pytest

import gabe_b200 as gb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for hdr in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(hdr).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(gabe_[a-z0-9_]+)\s*\(", src, re.M):
            names.add(m.group(1))
    # static inline helpers of the dump format are not library exports
    return sorted(n for n in names if not n.startswith("gabe_dump_"))


def test_library_exports_every_declared_symbol():
    lib = gb.library()
    names = declared_functions()
    assert "gabe_step" in names and "gabe_create" in names
    out = subprocess.run(["nm", "-D", "--defined-only", gb.lib_path()], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (gabe_\w+)", out))
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    for n in names:
        getattr(lib, n)


def test_params_struct_matches_header():
    lib = gb.library()
    p = gb.Params()
    lib.gabe_default_params(ctypes.byref(p), 64)
    assert p.struct_size == ctypes.sizeof(gb.Params)
    assert p.N == 64 and p.nflds == 2 and p.expansion == 1
    assert gb.numbins(64) == lib.gabe_spectra_numbins(64) == 56
    assert gb.numbins(256) == 222 and gb.numbins(512) == 444 and gb.numbins(1024) == 887


@pytest.mark.parametrize("field,value", [("N", 63), ("N", 2), ("nflds", 3), ("expansion", 3), ("expansion", -1),
                                         ("model", 7), ("precision", 5), ("dt", -1.0), ("gws_on", 2)])
def test_create_rejects_bad_params(field, value):
    lib = gb.library()
    p = gb.Params()
    lib.gabe_default_params(ctypes.byref(p), 32)
    setattr(p, field, value)
    h = ctypes.c_void_p()
    rc = lib.gabe_create(ctypes.byref(p), ctypes.byref(h))
    assert rc == 1 and not h.value
    assert lib.gabe_last_error(None)


def test_null_handles_are_errors_not_crashes():
    lib = gb.library()
    assert lib.gabe_destroy(None) == 0
    assert lib.gabe_step(None, 1) == 1
    assert lib.gabe_sync(None) == 1


def test_oracle_library_loads():
    from oracle import pyoracle as po
    assert po.numbins(64) == 56
