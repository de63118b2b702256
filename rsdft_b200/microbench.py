"""Small timing drivers for single pieces of the eigensolver, for profiling.

``python -m rsdft_b200.microbench hpsi --workload si216 --bands 64``
    H psi through ``rsdft_gpu_hamiltonian`` on device arrays (warm-up calls,
    then ``--reps`` timed calls); prints ms per call and the algorithmic
    bytes rate.  ``--no-nonlocal`` uploads an empty projector table first, so
    the stencil and Vloc part is timed alone.
``python -m rsdft_b200.microbench iteration --workload si216 --mode fp64``
    eigensolver iterations (CG -> Gram-Schmidt -> subspace) from the seeded
    start, ``--warmup`` untimed and ``--steps`` timed.
``python -m rsdft_b200.microbench rr --workload si216 --mode mixed-bf16``
    the Gram-Schmidt + Rayleigh-Ritz step alone (``rsdft_gpu_orth_subspace_diag``)
    on orthonormalised seeded bands; ``--ngrid`` / ``--bands`` shrink the cell
    (same atoms, coarser grid) for small profiler captures.
``python -m rsdft_b200.microbench table --workloads si8,si64,si216``
    per workload: hpsi on all bands (GB/s, fraction of the measured HBM
    copy bandwidth), FP64 and mixed iteration times, one adjoint force.
``python -m rsdft_b200.microbench large --workload si512``
    the large-cell run: FP64 and mixed iterations from one start (each timed),
    the FP64 closing pass, one adjoint force evaluation per form, eigenvalue
    and force differences between the forms, hpsi bandwidth on all bands.

All run on cuda:0 with the library on a dedicated torch stream; timings are
CUDA events on that stream.
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

MODES = {"fp64": 0, "mixed-bf16x3": 1, "mixed-tf32": 2, "mixed-bf16x2": 3}


def _setup(workload: str, ngrid: int = 0, bands: int = 0):
    import dataclasses

    import torch

    from rsdft_b200 import api
    from rsdft_b200.cell import WORKLOADS, build_cell

    st = torch.cuda.Stream()
    torch.cuda.set_stream(st)
    g = api.RsdftGpu(0)
    g.set_stream(st.cuda_stream)
    w = WORKLOADS[workload]
    if ngrid or bands:
        w = dataclasses.replace(w, ngrid=ngrid or w.ngrid, nband=bands or w.nband,
                                nocc=min(w.nocc, bands or w.nband))
    cell = build_cell(w)
    g.setup(cell)
    psi = torch.from_numpy(np.ascontiguousarray(cell.psi0().T)).cuda().t()
    return torch, api, g, cell, st, psi


def _timed(torch, st, fn, warmup: int, reps: int) -> float:
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(reps):
        fn()
    e1.record(st)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def run_hpsi(args) -> dict:
    torch, api, g, cell, st, psi = _setup(args.workload)
    from rsdft_b200 import _lib

    if args.no_nonlocal:
        lp = np.zeros(1, np.int32)
        _lib.call("rsdft_gpu_set_nonlocal", 0, lp.ctypes.data, None, None, None, None, cell.natom, None)
    nb = min(args.bands, cell.nband)
    p = psi[:, :nb]
    h = api.fortran_empty(cell.ML, nb)
    ms = _timed(torch, st, lambda: g.hamiltonian(1, 1, p, h, 1, cell.ML, 1, nb), args.warmup, args.reps)
    nnz = 0 if args.no_nonlocal else int(cell.lma_ptr[-1])
    nbytes = nb * cell.ML * 16 + cell.ML * 8 + nnz * 12
    return {"what": "hpsi", "workload": args.workload, "bands": nb, "nonlocal": not args.no_nonlocal,
            "ms": ms, "bytes": nbytes, "gbs": nbytes / (ms * 1e-3) / 1e9}


def run_iteration(args) -> dict:
    torch, api, g, cell, st, psi = _setup(args.workload, args.ngrid, args.bands)
    MB = cell.nband
    u = api.fortran_copy(psi)
    g.gram_schmidt(1, MB, 1, 1, u)
    esp = torch.zeros(MB, dtype=torch.float64, device="cuda")
    res = torch.zeros_like(esp)
    mode = MODES[args.mode]
    ms = _timed(torch, st, lambda: g.eigensolver_iteration(u, esp, res, ncg=args.ncg, mloop=args.mloop, mode=mode),
                args.warmup, args.steps)
    return {"what": "iteration", "workload": args.workload, "grid": list(cell.ngrid), "bands": MB, "mode": args.mode,
            "ms_per_iter": ms}


def run_rr(args) -> dict:
    torch, api, g, cell, st, psi = _setup(args.workload, args.ngrid, args.bands)
    MB = cell.nband
    u = api.fortran_copy(psi)
    g.gram_schmidt(1, MB, 1, 1, u)
    esp = torch.zeros(MB, dtype=torch.float64, device="cuda")
    mode = MODES[args.mode]
    ms = _timed(torch, st, lambda: g.orth_subspace_diag(1, 1, u, esp, mode=mode), args.warmup, args.reps)
    return {"what": "rr", "workload": args.workload, "grid": list(cell.ngrid), "bands": MB, "mode": args.mode,
            "ms": ms}


def run_large(args) -> dict:
    """The large-cell workload: from the same start, ``--steps`` FP64 and mixed
    iterations (each timed), the FP64 closing pass on the mixed bands, then
    one adjoint force evaluation per form; eigenvalue and force differences
    mixed vs FP64, hpsi bandwidth on all bands."""
    torch, api, g, cell, st, psi = _setup(args.workload)
    MB, ML = cell.nband, cell.ML
    start = api.fortran_copy(psi)
    g.gram_schmidt(1, MB, 1, 1, start)
    occ = np.zeros(MB)
    occ[: cell.nocc] = 2.0
    out = {"what": "large", "workload": args.workload, "grid": list(cell.ngrid), "bands": MB, "steps": args.steps}
    res = {}
    for name, mode in (("fp64", 0), ("mixed-bf16x3", 1)):
        u = api.fortran_copy(start)
        esp = torch.zeros(MB, dtype=torch.float64, device="cuda")
        r = torch.zeros_like(esp)
        times = []
        for _ in range(args.steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            g.eigensolver_iteration(u, esp, r, ncg=args.ncg, mloop=args.mloop, mode=mode)
            e1.record(st)
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
        if mode != 0:
            g.finalize_fp64(u, esp, r)
        dv = torch.zeros(ML, dtype=torch.float64, device="cuda")
        dr = torch.zeros(3 * cell.natom, dtype=torch.float64, device="cuda")
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(st)
        g.hpsi_adjoint(u, occ=occ, dl_dv=dv, dl_dr=dr)
        f1.record(st)
        torch.cuda.synchronize()
        res[name] = (esp.cpu().numpy(), dr.cpu().numpy())
        out[name] = {"ms_per_iter": times, "ms_per_iter_last": times[-1],
                     "adjoint_force_ms": f0.elapsed_time(f1)}
        del u
    occn = cell.nocc
    out["eig_err_max_occupied_ha"] = float(np.abs(res["fp64"][0][:occn] - res["mixed-bf16x3"][0][:occn]).max())
    out["force_err_max_ha_bohr"] = float(np.abs(res["fp64"][1] - res["mixed-bf16x3"][1]).max())
    h = api.fortran_empty(ML, MB)
    ms = _timed(torch, st, lambda: g.hamiltonian(1, 1, start, h, 1, ML, 1, MB), 2, 5)
    nbytes = MB * ML * 16 + ML * 8 + int(cell.lma_ptr[-1]) * 12
    out["hpsi"] = {"ms": ms, "gbs": nbytes / (ms * 1e-3) / 1e9}
    return out


def _hbm_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def run_table(args) -> dict:
    """Per workload: hpsi on all bands, FP64 and mixed iterations from the
    same Gram-Schmidt'd seeded start, one adjoint force evaluation (lowest
    nocc bands doubly occupied) on the FP64 bands."""
    import torch

    from rsdft_b200 import api
    from rsdft_b200.cell import build_cell

    peak, src = _hbm_peak()
    st = torch.cuda.Stream()
    torch.cuda.set_stream(st)
    g = api.RsdftGpu(0)
    g.set_stream(st.cuda_stream)
    rows = {}
    for name in args.workloads.split(","):
        cell = build_cell(name)
        g.setup(cell)
        MB, ML = cell.nband, cell.ML
        start = torch.from_numpy(np.ascontiguousarray(cell.psi0().T)).cuda().t()
        g.gram_schmidt(1, MB, 1, 1, start)
        h = api.fortran_empty(ML, MB)
        ms = _timed(torch, st, lambda: g.hamiltonian(1, 1, start, h, 1, ML, 1, MB), 2, 5)
        nbytes = MB * ML * 16 + ML * 8 + int(cell.lma_ptr[-1]) * 12
        row = {"grid": list(cell.ngrid), "bands": MB,
               "hpsi": {"ms": ms, "gbs": nbytes / (ms * 1e-3) / 1e9, "frac": nbytes / (ms * 1e-3) / 1e9 / peak,
                        "peak_source": src}}
        for form, mode in (("fp64", 0), ("mixed-bf16x3", 1)):
            u = api.fortran_copy(start)
            esp = torch.zeros(MB, dtype=torch.float64, device="cuda")
            res = torch.zeros_like(esp)
            it = _timed(torch, st, lambda: g.eigensolver_iteration(u, esp, res, ncg=4, mloop=3, mode=mode),
                        args.warmup, args.steps)
            row[form] = {"ms_per_iter": it}
            if mode == 0:
                occ = np.zeros(MB)
                occ[: cell.nocc] = 2.0
                dv = torch.zeros(ML, dtype=torch.float64, device="cuda")
                dr = torch.zeros(3 * cell.natom, dtype=torch.float64, device="cuda")
                row["adjoint_force_ms"] = _timed(torch, st, lambda: g.hpsi_adjoint(u, occ=occ, dl_dv=dv, dl_dr=dr),
                                                 1, 3)
            del u
        rows[name] = row
    return {"what": "table", "rows": rows}


def main(argv=None) -> None:
    p = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    sub = p.add_subparsers(dest="what", required=True)
    h = sub.add_parser("hpsi")
    h.add_argument("--workload", default="si216")
    h.add_argument("--bands", type=int, default=64)
    h.add_argument("--warmup", type=int, default=3)
    h.add_argument("--reps", type=int, default=10)
    h.add_argument("--no-nonlocal", action="store_true")
    it = sub.add_parser("iteration")
    it.add_argument("--workload", default="si216")
    it.add_argument("--mode", default="fp64", choices=sorted(MODES))
    it.add_argument("--ncg", type=int, default=4)
    it.add_argument("--mloop", type=int, default=3)
    it.add_argument("--warmup", type=int, default=3)
    it.add_argument("--steps", type=int, default=2)
    it.add_argument("--ngrid", type=int, default=0)
    it.add_argument("--bands", type=int, default=0)
    rr = sub.add_parser("rr")
    rr.add_argument("--workload", default="si216")
    rr.add_argument("--mode", default="mixed-bf16x3", choices=sorted(MODES))
    rr.add_argument("--ngrid", type=int, default=0)
    rr.add_argument("--bands", type=int, default=0)
    rr.add_argument("--warmup", type=int, default=2)
    rr.add_argument("--reps", type=int, default=5)
    lg = sub.add_parser("large")
    lg.add_argument("--workload", default="si512")
    lg.add_argument("--ncg", type=int, default=4)
    lg.add_argument("--mloop", type=int, default=3)
    lg.add_argument("--steps", type=int, default=5)
    tb = sub.add_parser("table")
    tb.add_argument("--workloads", default="si8,si64,si216")
    tb.add_argument("--warmup", type=int, default=2)
    tb.add_argument("--steps", type=int, default=3)
    args = p.parse_args(argv)
    out = {"hpsi": run_hpsi, "iteration": run_iteration, "rr": run_rr, "large": run_large,
           "table": run_table}[args.what](args)
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
