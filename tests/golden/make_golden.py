"""Generate the committed golden fixtures of tests/golden.

1. ``fd_kat_si216.json``: the Md = 6 finite-difference table RSDFT prints in
   init_kinetic (kinetic_module.f90:94-112) for Hgrid = 0.6413125, read from
   the reference's committed run log examples/Si216/a.log:249-273 (and
   coef_lap0 from the same block).  This is the reference's own known-answer
   output for the hot path's set-up.
2. ``gaunt_l1.json``: the coupling coefficients of the force's derivative
   table for projector angular momenta L = 0 and 1 -- the entries
   Y1/Y2/Y3(L, m, L1, L1z) that get_gaunt_coefficient_L1 assigns
   (force_sub_sub_module.f90:64-387), read from that source file as text.
3. ``oracle_si8_g12.npz``: sampled outputs of the oracle (hpsi, one CG sweep,
   Gram-Schmidt, subspace diagonalisation, nonlocal force) on the seeded
   12^3 cell, so that later edits of the oracle cannot drift unnoticed.

Run from the repository root:
``python tests/golden/make_golden.py --reference <path of the RSDFT tree>``
writes all three; ``--oracle-only`` rewrites only the oracle fixture (no
reference tree needed).
"""
from __future__ import annotations

import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def fd_kat(reference: str) -> dict:
    log = open(os.path.join(reference, "examples", "Si216", "a.log")).read().splitlines()
    start = next(i for i, l in enumerate(log) if "lap" in l and "coef_lap" in l)
    lap, coef, nab, coefn = {}, {}, {}, {}
    i = start + 1
    while "nab" not in log[i]:
        t = log[i].split()
        n = int(t[0])
        lap[n] = t[1]
        coef[n] = t[2:]
        i += 1
    i += 1
    while i < len(log) and re.match(r"^\s+\d+\s", log[i]):
        t = log[i].split()
        nab[int(t[0])] = t[1]
        coefn[int(t[0])] = t[2:]
        i += 1
    return {
        "source": "examples/Si216/a.log:249-273 (init_kinetic, kinetic_module.f90:94-112)",
        "Md": 6,
        "Hgrid": 0.6413125,
        "print_format": "f20.15",
        "lap": [float(lap[n]) for n in range(7)],
        "coef_lap0": float(coef[0][0]),
        "coef_lap": [float(coef[n][0]) for n in range(1, 7)],
        "nab": [float(nab[n]) for n in range(1, 7)],
        "coef_nab": [float(coefn[n][0]) for n in range(1, 7)],
    }


def gaunt_l1(reference: str, lmax: int = 1) -> dict:
    """Y1/Y2/Y3(L, m, L1, L1z) entries with L <= lmax, as assigned in
    get_gaunt_coefficient_L1 (values printed with 15 decimals)."""
    path = os.path.join(reference, "src", "force_sub_sub_module.f90")
    src = open(path).read()
    body = src[src.index("SUBROUTINE get_gaunt_coefficient_L1"):src.index("END SUBROUTINE get_gaunt_coefficient_L1")]
    pat = re.compile(r"(Y[123])\(\s*(-?\d+)\s*,\s*(-?\d+)\s*,\s*(-?\d+)\s*,\s*(-?\d+)\s*\)\s*=\s*([-+.\dEeDd]+)")
    out = {"Y1": [], "Y2": [], "Y3": []}
    for m in pat.finditer(body):
        name, L, mm, L1, L1z, v = m.groups()
        if int(L) <= lmax:
            out[name].append([int(L), int(mm), int(L1), int(L1z), float(v.lower().replace("d", "e"))])
    return {"source": "force_sub_sub_module.f90:64-387 (get_gaunt_coefficient_L1), entries with L <= %d" % lmax,
            "note": "Y1, Y2, Y3 couple through the l = 1 harmonics of m = 1, -1, 0 (x, y, z)", **out}


def oracle_fixture() -> dict:
    from oracle import oracle as O
    from rsdft_b200.cell import build_cell

    c = build_cell("si8_g12")
    o = O.Oracle(c)
    psi = np.asfortranarray(c.psi0())
    rng = np.random.default_rng(12)
    idx = rng.choice(c.ML, 256, replace=False)
    h = o.hamiltonian(psi[:, :4])
    q = o.gram_schmidt_t(psi)
    u, esp, res, _ = o.conjugate_gradient(q, 4, 3)
    u2 = o.gram_schmidt_t(u)
    u3, w, _ = o.subspace_diag_la(u2)
    occ = c.occupations()
    f = o.force_nloc(u3, occ)
    return {
        "idx": idx,
        "hpsi": h[idx, :],
        "gs": q[idx, :4],
        "cg_esp": esp,
        "cg_res": res,
        "sub_esp": w,
        "force": f,
    }


if __name__ == "__main__":
    import argparse

    ap = argparse.ArgumentParser()
    g = ap.add_mutually_exclusive_group(required=True)
    g.add_argument("--reference", help="root of the RSDFT source tree (read-only)")
    g.add_argument("--oracle-only", action="store_true")
    args = ap.parse_args()
    if args.reference:
        with open(os.path.join(HERE, "fd_kat_si216.json"), "w") as fh:
            json.dump(fd_kat(args.reference), fh, indent=1)
        print("wrote fd_kat_si216.json")
        with open(os.path.join(HERE, "gaunt_l1.json"), "w") as fh:
            json.dump(gaunt_l1(args.reference), fh, indent=1)
        print("wrote gaunt_l1.json")
    np.savez_compressed(os.path.join(HERE, "oracle_si8_g12.npz"), **oracle_fixture())
    print("wrote oracle_si8_g12.npz")
