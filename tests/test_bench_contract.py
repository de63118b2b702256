"""The benchmark's JSON line for the reference arm (the CPU oracle on the host
cores), on the small cell: one line with every key the benchmark contract
names, the time-like fields consistent, and no device bytes moved."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run(*args):
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], capture_output=True, text=True,
                         timeout=300, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out.stdout
    return json.loads(lines[0])


def test_reference_arm_line():
    d = run("--impl", "reference", "--workload", "si8", "--steps", "2", "--warmup", "1")
    assert d["impl"] == "reference"
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["metric"].startswith("eigensolver iter/s (Si8 24^3, 32 bands")
    assert d["unit"] == "iter/s" and d["higher_is_better"] is True and d["value"] > 0
    assert (d["n_gpus"], d["steps"], d["warmup"]) == (1, 2, 1)
    assert abs(d["ms_per_step"] - 1000.0 / d["value"]) <= 1e-6 * d["ms_per_step"]
    assert d["vs_baseline"] is None and d["config"]["workload"] == "si8"
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["sample"]
    # whole iterations actually timed, no scaling; the host is described
    assert (cb["steps"], cb["warmup"]) == (d["steps"], d["warmup"]) and "scaled" not in cb["sample"]
    assert cb["host"]["cpu_model"] and cb["host"]["blas"] and d["ranks_used"] == 1
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == d["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


def test_reference_arm_under_torchrun_prints_once():
    """Launched as the multi-GPU run is (torchrun, 2 ranks), rank 0 alone runs
    the reference arm and prints; the other rank exits 0 without work."""
    import socket

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    out = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
                          "--master-addr", "127.0.0.1", "--master-port", str(port),
                          os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload", "si8", "--steps", "1",
                          "--warmup", "0"], capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["ranks_used"] == 1
