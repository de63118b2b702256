"""Benchmark of the Kohn-Sham eigensolver inner loop on B200.

Workload (default): the 216-atom Si cell, 72^3 grid (373,248 points), Md = 6,
480 bands; one step = one eigensolver iteration as calc_sweep runs it
(sweep_module.f90:150-155): CG (Ncg = 4, mloop = 3, IPC = 4) -> Gram-Schmidt
-> subspace diagonalisation, starting from seeded random bands.

Printed JSON line (rank 0):
  value        eigensolver iterations/s of the headline form over all ranks,
               inputs resident in HBM (device-timed with CUDA events)
  e2e          the same through the C ABI with the wavefunction in pinned host
               memory: every step is one eigensolver_sweep call on the host
               array, which uploads it (band blocks overlapped with the CG),
               runs the iteration and downloads it with the eigenvalues
  roofline     hpsi (projection + fused stencil/Vloc/nonlocal kernels) on all
               bands: algorithmic bytes / measured duration vs measured HBM peak
  cpu_baseline the oracle (C/OpenMP + numpy BLAS) on the host cores: one
               whole iteration of the same workload, every band (rank 0,
               N = 1)
``--impl reference`` times only that CPU implementation (the reference is
Fortran and cannot be built in this image; the oracle restates it).
Multi-GPU (torchrun): independent replicas, one per GPU ("scaling": "weak").
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

MODES = {"fp64": 0, "mixed-bf16x3": 1, "mixed-tf32": 2, "mixed-bf16x2": 3}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default="si216")
    p.add_argument("--mode", default="auto", choices=["auto"] + sorted(MODES))
    p.add_argument("--ncg", type=int, default=4)
    p.add_argument("--mloop", type=int, default=3)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-accuracy", action="store_true", help="skip the 10-iteration accuracy comparison")
    p.add_argument("--cpu-table", default="", help="comma-separated workloads: print the CPU rows of the "
                   "per-configuration table (oracle hpsi, nonlocal force, and whole iterations for "
                   "--cpu-table-iter) and exit")
    p.add_argument("--cpu-table-iter", default="si8,si64")
    return p.parse_args()


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clock / throttle samples (every 100 ms), each stamped by
    nvidia-smi itself, so the ones inside a timed window can be picked out.
    Started well before the window (nvidia-smi takes a few hundred ms to
    print its first sample)."""

    FIELDS = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)  # the reader has taken every line once the pipe closes

    @classmethod
    def parse(cls, lines):
        """(epoch seconds, sm MHz, max sm MHz, set of active reasons) per sample."""
        out = []
        for ln in lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 10:
                continue
            try:
                ts = time.mktime(time.strptime(f[0].split(".")[0], "%Y/%m/%d %H:%M:%S"))
                ts += float("0." + f[0].split(".")[1]) if "." in f[0] else 0.0
                sm, mx = float(f[2]), float(f[3])
            except ValueError:
                continue
            reasons = {n for n, v in zip(cls.REASONS, f[6:10]) if v.lower().startswith("active")}
            out.append((ts, sm, mx, reasons))
        return out

    @classmethod
    def summarize(cls, samples, t0, t1):
        """Samples inside [t0, t1] (host wall clock); when the window is
        shorter than the sampling period, the nearest sample on each side
        (within 0.3 s: the GPU is busy with warm-up before and the next
        phase after)."""
        inside = [s for s in samples if t0 <= s[0] <= t1]
        if not inside:
            before = [s for s in samples if t0 - 0.3 <= s[0] < t0]
            after = [s for s in samples if t1 < s[0] <= t1 + 0.3]
            inside = before[-1:] + after[:1]
        if not inside:
            return None
        reasons = set().union(*(s[3] for s in inside))
        return {"sm_mhz": statistics.median(s[1] for s in inside), "sm_max_mhz": inside[-1][2],
                "reasons": sorted(reasons), "samples": len(inside),
                "window_s": round(t1 - t0, 3)}


# ------------------------------------------------------------ CPU baseline
def host_info():
    """CPU model, logical cores and the BLAS numpy/scipy call (the oracle's
    dense steps)."""
    model = "unknown"
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.lower().startswith("model name"):
                model = ln.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    blas = "unknown"
    try:
        cfg = np.show_config(mode="dicts")["Build Dependencies"]["blas"]
        blas = f"{cfg.get('name', '?')} {cfg.get('version', '')}".strip()
    except Exception:  # noqa: BLE001 - numpy builds without the dict form
        pass
    return {"cpu_model": model, "logical_cores": os.cpu_count(), "blas": blas}


def cpu_iteration(o, cell, psi, ncg: int, mloop: int):
    """One full eigensolver iteration on the oracle, as calc_sweep runs it
    (sweep_module.f90:150-155): conjugate_gradient_1 on every band (band by
    band, cg_module.f90:97-430), the literal recursive gram_schmidt_t
    (gram_schmidt_t_module.f90:84-316), then subspace_diag_la with H psi of
    every band, dsyr2k, DSYEV and the rotation (subspace_diag_la_module.f90:
    18-232).  Returns the new bands and the seconds of each step."""
    t0 = time.perf_counter()
    u, _, _, _ = o.conjugate_gradient(psi, ncg, mloop)
    t1 = time.perf_counter()
    u = o.gram_schmidt_t(u)
    t2 = time.perf_counter()
    u, _, _ = o.subspace_diag_la(u)
    t3 = time.perf_counter()
    return np.asfortranarray(u), {"cg": t1 - t0, "gram_schmidt": t2 - t1, "subspace_diag": t3 - t2}


def cpu_baseline_run(cell, ncg: int, mloop: int, steps: int, warmup: int):
    """The oracle (C/OpenMP on all host threads + numpy/OpenBLAS) timed on
    whole iterations of the full workload (every band), continuing from the
    seeded start bands after Gram-Schmidt: `warmup` untimed iterations, then
    `steps` timed ones; median seconds per iteration."""
    from oracle import oracle as O  # CPU baseline leg only

    o = O.Oracle(cell)
    psi = o.gram_schmidt_t(np.asfortranarray(cell.psi0()))
    for _ in range(warmup):
        psi, _ = cpu_iteration(o, cell, psi, ncg, mloop)
    per, parts = [], []
    for _ in range(steps):
        t0 = time.perf_counter()
        psi, sec = cpu_iteration(o, cell, psi, ncg, mloop)
        per.append(time.perf_counter() - t0)
        parts.append(sec)
    threads = int(O.lib().oracle_num_threads())
    med = statistics.median(per)
    info = host_info()
    return {
        "value": 1.0 / med,
        "unit": "iter/s",
        "cores": threads,
        "kind": "port",
        "sample": (f"oracle (C/OpenMP, {threads} threads, + numpy/{info['blas']}): {steps} whole iteration(s) of "
                   f"{cell.nband} bands x {cell.ML} points after {warmup} untimed, median; no scaling"),
        "steps": steps,
        "warmup": warmup,
        "seconds_per_iter": per,
        "seconds": {k: statistics.median(p[k] for p in parts) for k in parts[0]},
        "host": info,
    }


def cpu_table(workloads, ncg: int, mloop: int, iter_workloads):
    """The CPU rows of the per-configuration table: the oracle on the host
    cores, per workload hpsi on every band, one nonlocal force evaluation
    (lowest nocc bands doubly occupied) and, for the workloads in
    iter_workloads, one whole iteration as cpu_iteration runs it."""
    from oracle import oracle as O  # CPU baseline leg only

    rows = {}
    for name in workloads:
        from rsdft_b200.cell import build_cell

        cell = build_cell(name)
        o = O.Oracle(cell)
        psi = o.gram_schmidt_t(np.asfortranarray(cell.psi0()))
        o.hamiltonian(np.asfortranarray(psi[:, :2]))  # threads and tables warm
        t0 = time.perf_counter()
        o.hamiltonian(psi)
        row = {"hpsi_s": time.perf_counter() - t0}
        occ = np.zeros(cell.nband)
        occ[: cell.nocc] = 2.0
        t0 = time.perf_counter()
        o.force_nloc(psi, occ)
        row["force_nloc_s"] = time.perf_counter() - t0
        if name in iter_workloads:
            _, sec = cpu_iteration(o, cell, psi, ncg, mloop)
            row["iteration_s"] = sum(sec.values())
        rows[name] = row
    return {"what": "cpu_table", "threads": int(O.lib().oracle_num_threads()), "host": host_info(), "rows": rows}


def metric_name(cell, ncg):
    """The headline metric's label for a workload ("Si216 72^3, 480 bands" by default)."""
    n1 = cell.ngrid[0]
    return (f"eigensolver iter/s ({cell.name.split('_')[0].capitalize()} {n1}^3, {cell.nband} bands, "
            f"CG Ncg={ncg} + GS + subspace)")


def run_reference(args, rank, world):
    """The reference arm: the reference's CPU path (its Fortran cannot be
    built in this image, so the oracle's restatement of it) on the host
    cores, rank 0 only.  Whole iterations of the full workload: at most 3
    timed after at most 1 untimed (about 20-40 s each), and the line says
    how many ran."""
    if rank != 0:
        return
    from rsdft_b200.cell import build_cell

    cell = build_cell(args.workload)
    steps = max(1, min(args.steps, 3))
    warmup = max(0, min(args.warmup, 1))
    t0 = time.perf_counter()
    r = cpu_baseline_run(cell, args.ncg, args.mloop, steps, warmup)
    wall = time.perf_counter() - t0
    v = r["value"]
    out = {
        "impl": "reference",
        "metric": metric_name(cell, args.ncg),
        "value": v,
        "unit": "iter/s",
        "n_gpus": world,
        "ranks_used": 1,
        "steps": steps,
        "warmup": warmup,
        "ms_per_step": 1000.0 / v,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded Si cell, random start bands)",
        "config": {"workload": f"{args.workload}", "grid": list(cell.ngrid), "bands": cell.nband, "Md": cell.md,
                   "ncg": args.ncg, "mloop": args.mloop},
        "cpu_baseline": {k: r[k] for k in ("value", "unit", "cores", "kind", "sample", "steps", "warmup", "host")},
        "e2e": {"value": v, "unit": "iter/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "seconds": r["seconds"],
        "note": ("The reference is Fortran+MPI; no Fortran compiler exists in this image, so its CPU path is "
                 "timed through the oracle's line-by-line restatement, on one process (rank 0) whatever the "
                 "number of ranks launched."),
        "wall_s": wall,
    }
    print(json.dumps(out), flush=True)


# ------------------------------------------------------------- our arm
# DRAM bytes (read + write) of one hpsi call per band, from the ncu capture of
# the three hpsi kernels on Si216 with 64 bands (k_nl_project 167.8 MB,
# k_stencil_tma 379.7 MB, k_nl_scatter 210.8 MB), scaled by the band count.
HPSI_TRAFFIC_PER_BAND = {"si216": (167.8e6 + 379.7e6 + 210.8e6) / 64}


def hpsi_bytes(cell, nb):
    return nb * cell.ML * 16 + cell.ML * 8 + int(cell.lma_ptr[-1]) * 12


def main():
    args = parse()
    from rsdft_b200 import replicas

    rank, world, local = replicas.rank_info()
    if args.cpu_table:
        if rank == 0:
            print(json.dumps(cpu_table(args.cpu_table.split(","), args.ncg, args.mloop,
                                       set(args.cpu_table_iter.split(",")))), flush=True)
        return
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    import torch.distributed as dist

    from rsdft_b200 import _lib, api
    from rsdft_b200.cell import build_cell

    torch.cuda.set_device(local)
    pg = replicas.init(world, "nccl")
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)  # torch and the library share this stream
    g = api.RsdftGpu(local)
    g.set_stream(stream.cuda_stream)
    cell = build_cell(args.workload)
    g.setup(cell)
    ML, MB = cell.ML, cell.nband

    psi0 = np.asfortranarray(cell.psi0())
    start = torch.from_numpy(np.ascontiguousarray(psi0.T)).cuda().t()  # (ML, MB) Fortran
    g.gram_schmidt(1, MB, 1, 1, start)  # init_wf + gram_schmidt (main.f90:253-257)
    esp = torch.zeros(MB, dtype=torch.float64, device="cuda")
    res = torch.zeros_like(esp)

    def supported(mode):
        u = api.fortran_copy(start)
        try:
            g.gram_schmidt(1, MB, 1, 1, u, mode=mode)
            g.subspace_diag(1, 1, u, esp, mode=mode)
            return True
        except api.RsdftError:
            return False

    modes = ["fp64"]
    if args.mode == "auto":
        for m in ("mixed-bf16x3",):
            if supported(MODES[m]):
                modes.append(m)
                break
        head = modes[-1]
    else:
        head = args.mode
        if head != "fp64":
            modes.append(head)

    def iterate(u, mode):
        g.eigensolver_iteration(u, esp, res, ncg=args.ncg, mloop=args.mloop, mode=MODES[mode])

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    results = {}
    clocks = None
    launches = 0
    window = None
    sampler = ClockSampler(local)
    sampler.start()
    for mode in modes:
        u = api.fortran_copy(start)
        for _ in range(args.warmup):
            iterate(u, mode)
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        n0 = _lib.load().rsdft_gpu_kernel_launches()
        w0 = time.time()
        e0.record(stream)
        for _ in range(args.steps):
            iterate(u, mode)
        e1.record(stream)
        barrier()
        w1 = time.time()
        n1 = _lib.load().rsdft_gpu_kernel_launches()
        if mode == head:
            window = (w0, w1)
            launches = int(n1 - n0)
        ms = replicas.max_over_ranks(e0.elapsed_time(e1) / args.steps, pg, device="cuda")
        results[mode] = {"ms": ms, "esp": esp.cpu().numpy().copy()}

    # ---- accuracy of the headline form against FP64 from the same start:
    # 10 iterations each (separate copies of the start bands), then the FP64
    # closing pass (CholeskyQR2 + Rayleigh quotients and residuals in FP64)
    # on both; at iteration 3, before the bands converge, the two
    # trajectories' Ritz values and one Rayleigh-Ritz step of the headline
    # form against the FP64 step on the same (FP64 CG) bands
    acc = {}
    if head != "fp64" and not args.no_accuracy:
        niter = 10
        ua = api.fortran_copy(start)
        ub = api.fortran_copy(start)
        ea = torch.zeros_like(esp)
        eb = torch.zeros_like(esp)
        ra = torch.zeros_like(esp)
        rb = torch.zeros_like(esp)
        occ = cell.nocc
        early = {}
        for it in range(1, niter + 1):
            g.eigensolver_iteration(ua, ea, ra, ncg=args.ncg, mloop=args.mloop, mode=0)
            g.eigensolver_iteration(ub, eb, rb, ncg=args.ncg, mloop=args.mloop, mode=MODES[head])
            if it == 3:
                x = api.fortran_copy(ua)
                e0, r0 = torch.zeros_like(esp), torch.zeros_like(esp)
                g.conjugate_gradient(1, ML, MB, 1, 1, x, e0, r0, ncg=args.ncg, mloop=args.mloop, mode=0)
                y = api.fortran_copy(x)
                e1, e2 = torch.zeros_like(esp), torch.zeros_like(esp)
                g.orth_subspace_diag(1, 1, x, e1, mode=0)
                g.orth_subspace_diag(1, 1, y, e2, mode=MODES[head])
                early = {"iteration": it,
                         "trajectory_eig_diff_occupied_ha": float((ea[:occ] - eb[:occ]).abs().max()),
                         "rayleigh_ritz_step_eig_err_occupied_ha": float((e1[:occ] - e2[:occ]).abs().max()),
                         "fp64_residual_max_occupied": float(ra[:occ].max())}
                del x, y
        sub_err = float((ea[:occ] - eb[:occ]).abs().max())
        orth_before = float(((ub.t() @ ub) * cell.dV - torch.eye(MB, dtype=torch.float64, device="cuda")).abs().max())
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g.finalize_fp64(ua, ea, ra)
        f0.record(stream)
        g.finalize_fp64(ub, eb, rb)
        f1.record(stream)
        barrier()
        orth = float(((ub.t() @ ub) * cell.dV - torch.eye(MB, dtype=torch.float64, device="cuda")).abs().max())
        acc = {"iterations": niter,
               "eig_err_max_occupied_ha": float((ea[:occ] - eb[:occ]).abs().max()),
               "eig_err_max_all_ha": float((ea - eb).abs().max()),
               "subspace_eig_err_before_fp64_pass_ha": sub_err,
               "orth_err_after_fp64_pass": orth,
               "orth_err_before_fp64_pass": orth_before,
               "fp64_closing_pass_ms": f0.elapsed_time(f1),
               "residual_max_occupied": float(rb[:occ].max()),
               "unconverged": early}
        del ua, ub

    # ---- hpsi roofline on all bands (device pointers, K launches)
    out = api.fortran_empty(ML, MB)
    for _ in range(3):
        g.hamiltonian(1, 1, start, out, 1, ML, 1, MB)
    reps = 10
    h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    h0.record(stream)
    for _ in range(reps):
        g.hamiltonian(1, 1, start, out, 1, ML, 1, MB)
    h1.record(stream)
    barrier()
    hms = h0.elapsed_time(h1) / reps
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    hb = hpsi_bytes(cell, MB)
    hgbs = hb / (hms * 1e-3) / 1e9
    del out

    # ---- end to end through the C ABI with host buffers
    e2e = None
    if not args.no_e2e:
        host = torch.empty((MB, ML), dtype=torch.float64, pin_memory=True)
        host.copy_(start.t())
        hn = host.numpy().T  # (ML, MB) Fortran view of pinned memory
        esp_h = np.zeros(MB)
        res_h = np.zeros(MB)
        mode_e = MODES[head]
        for _ in range(1):
            g.eigensolver_iteration(hn, esp_h, res_h, ncg=args.ncg, mloop=args.mloop, mode=mode_e)
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            g.eigensolver_iteration(hn, esp_h, res_h, ncg=args.ncg, mloop=args.mloop, mode=mode_e)
        barrier()
        dt = replicas.max_over_ranks((time.perf_counter() - t0) / args.steps, pg, device="cuda")
        e2e = {"value": replicas.whole_job_rate(1.0, world, dt), "unit": "iter/s", "h2d_bytes_per_step": ML * MB * 8,
               "d2h_bytes_per_step": ML * MB * 8 + 2 * MB * 8}

    # clocks during the headline form's timed window (the sampler has run
    # since before the first form's warm-up)
    if window is not None and time.time() < window[1] + 0.35:
        time.sleep(window[1] + 0.35 - time.time())
    sampler.stop()
    clocks = ClockSampler.summarize(ClockSampler.parse(sampler.lines), *window) if window else None

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_run(cell, args.ncg, args.mloop, 1, 0)

    if rank == 0:
        ms = results[head]["ms"]
        line = {
            "metric": metric_name(cell, args.ncg),
            "value": replicas.whole_job_rate(1000.0, world, ms),
            "unit": "iter/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64" if head == "fp64" else ("bf16(3-term)+f32+f64" if head == "mixed-bf16x3" else "bf16(2-term)+f32+f64"),
            "data": "synthetic (seeded Si cell, random start bands)",
            "config": {"workload": args.workload, "grid": list(cell.ngrid), "bands": MB, "Md": cell.md,
                       "ncg": args.ncg, "mloop": args.mloop, "form": head,
                       "l2": "inputs larger than L2 (psi = %.2f GB)" % (ML * MB * 8 / 1e9),
                       "parallelism": f"replicas x{world}"},
            "forms": {m: {"ms_per_iter": r["ms"], "iter_s": 1000.0 / r["ms"]} for m, r in results.items()},
            "hpsi": {"ms": hms, "gbs": hgbs, "bytes": hb, "frac_of_hbm": hgbs / hbm},
            "roofline": {"bound": "hbm", "achieved": hgbs, "peak": hbm, "unit": "GB/s", "frac": hgbs / hbm,
                         "traffic": (HPSI_TRAFFIC_PER_BAND[args.workload] * MB
                                     if args.workload in HPSI_TRAFFIC_PER_BAND else None),
                         "kernel": "hpsi (k_nl_project + k_stencil_tma + k_nl_scatter), all bands",
                         "peak_source": peak_src},
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clocks,
            "cpu_baseline": cpu,
        }
        if "fp64" in results and head != "fp64":
            line["speedup_vs_fp64"] = results["fp64"]["ms"] / ms
        if acc:
            line["accuracy"] = acc
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
