"""Generate tests/golden fixtures by running the reference itself.

Runs the reference binaries that `make -C oracle ref` compiles from the
unmodified reference sources (oracle/_ref/ref_<cfg>, one thread, so rand()
runs in loop order) and records, for each configuration and step:

  * SHA-256 of field[0], dfield[0], h[0], l[0] as the reference wrote them;
  * the 12 per-stage scalars (a, adot, edkin, edpot, edgrad, edrho) as exact
    hex floats, and the L2 norm of every array;
  * the reference's own spectra files (slices_spectra_<n>.dat) as numbers.

plus the complete state of the smallest GW configuration at one step
(ref_m1_n16_g1_step10.npz) for tolerance-based checks.

Usage (needs the reference tree, so it runs only where it is mounted):
    make -C oracle ref && python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle import pyoracle as po  # noqa: E402

CASES = [
    # (model, N, gws, steps at which to dump, steps at which to write spectra[, expansion_type])
    (1, 16, 1, [0, 1, 2, 5, 10, 50], [0, 10, 50]),
    (0, 32, 1, [0, 1, 10, 50], [0, 50]),
    (1, 32, 0, [0, 1, 10, 100, 200], [0, 200]),
    (1, 64, 0, [0, 1, 10, 100, 200], [0, 200]),
    (1, 64, 1, [0, 1, 10], [0, 10]),
    # expansion_type 0 (no expansion) and 2 (type 1 without tensor modes; the
    # harness starts the user-defined expansion as type 1)
    (1, 32, 0, [0, 1, 10, 100], [0, 100], 0),
    (1, 32, 1, [0, 1, 10, 50], [0, 50], 0),
    (1, 32, 1, [0, 1, 10, 50], [0, 50], 2),
    # initial spectra with spec_cut_off (randInit variant 1) and field_full_rand 0 (variant 2)
    (1, 32, 0, [0, 1, 10], [0, 10], 1, 1),
    (1, 32, 0, [0, 1, 10], [0, 10], 1, 2),
]


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


def record(st: po.State) -> dict:
    out = {
        "field": sha(st.field[0]), "dfield": sha(st.dfield[0]),
        "norm_field": float(np.linalg.norm(st.field[0])), "norm_dfield": float(np.linalg.norm(st.dfield[0])),
        "scalars": {k: [float(getattr(st.sc, k)[s]).hex() for s in (0, 1)]
                    for k in ("a", "adot", "edkin", "edpot", "edgrad", "edrho")},
    }
    if st.cfg.gws:
        out.update({"h": sha(st.h[0]), "l": sha(st.l[0]),
                    "norm_h": float(np.linalg.norm(st.h[0])), "norm_l": float(np.linalg.norm(st.l[0]))})
    return out


def main() -> None:
    golden = {"generator": "tests/golden/make_golden.py", "seed": 44463132, "L": 20.0, "dt": 0.01, "cases": {}}
    for model, N, gws, dumps, specs, *rest in CASES:
        expansion = rest[0] if rest else 1
        ic = rest[1] if len(rest) > 1 else 0
        name = f"m{model}_n{N}_g{gws}" + ("" if expansion == 1 else f"_e{expansion}") + ("", "_rc", "_rd")[ic]
        binary = po.ref_binary(model, N, gws, 0, expansion, ic)
        with tempfile.TemporaryDirectory() as d:
            steps = max(dumps + specs)
            po.run_ref(binary, ["--steps", str(steps), "--dump-prefix", "s_", "--dump-at", ",".join(map(str, dumps)),
                                "--spectra-at", ",".join(map(str, specs))], d)
            cfg = po.Config(N=N, model=model, gws=gws, expansion=expansion, ic_variant=ic)
            entry = {"model": model, "N": N, "gws": gws, "steps": {}, "spectra": {}}
            if expansion != 1:
                entry["expansion"] = expansion
            if ic:
                entry["ic_variant"] = ic
            for s in dumps:
                st = po.read_dump(os.path.join(d, f"s_{s}.bin"), cfg)
                entry["steps"][str(s)] = record(st)
                if name == "m1_n16_g1" and s == 10:
                    np.savez_compressed(os.path.join(HERE, "ref_m1_n16_g1_step10.npz"),
                                        field=st.field[0], dfield=st.dfield[0], h=st.h[0], l=st.l[0],
                                        scalars=np.array([[getattr(st.sc, k)[q] for q in (0, 1)] for k in
                                                          ("a", "adot", "edkin", "edpot", "edgrad", "edrho")]))
                if name == "m1_n16_g1" and s == 0:
                    np.savez_compressed(os.path.join(HERE, "ref_m1_n16_g1_step0.npz"),
                                        field=st.field[0], dfield=st.dfield[0],
                                        scalars=np.array([[getattr(st.sc, k)[q] for q in (0, 1)] for k in
                                                          ("a", "adot", "edkin", "edpot", "edgrad", "edrho")]))
            for n, s in enumerate(specs):
                tab = np.loadtxt(os.path.join(d, "slices", f"slices_spectra_{n}.dat"))
                entry["spectra"][str(s)] = tab.tolist()
        golden["cases"][name] = entry
        print(name, "done", flush=True)
    with open(os.path.join(HERE, "golden.json"), "w") as fh:
        json.dump(golden, fh, indent=1)


if __name__ == "__main__":
    main()
