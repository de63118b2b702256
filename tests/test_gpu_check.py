"""The debug build (librsdft_gpu_check.so, -DRSDFT_GPU_CHECK) on the GPU.

Its kernels that index memory through stored tables (the nonlocal
projection, scatter and force gathers) check each index against its array.
A child process loads the debug build (RSDFT_GPU_CHECK=1; one library per
process) and runs small seeded cases of hpsi, the split nonlocal operators,
the CG sweep, Gram-Schmidt + Rayleigh-Ritz and the nonlocal force against the
oracle: results must match to 1e-12 and no check may fail.  Then
rsdft_gpu_selftest_check makes one check fail on purpose (an index one past
its buffer, whose read the check skips): the next synchronize must report
RSDFT_ECHECK with the site and index, clear it, and the context must keep
working.  No access outside a buffer is made on this path.
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
TOL = 1e-12


def child() -> dict:
    sys.path.insert(0, os.path.dirname(HERE))
    import torch

    from oracle import oracle as O
    from rsdft_b200 import _lib, api
    from rsdft_b200.cell import build_cell

    out = {}
    L = _lib.load()
    out["lib"] = os.path.basename(_lib.LIB_PATH)
    out["checked"] = L.rsdft_gpu_checked_build()
    c = build_cell("si8")
    o = O.Oracle(c)
    g = api.RsdftGpu(0)
    g.setup(c)
    rel = lambda a, b: float(np.abs(a - b).max() / np.abs(b).max())  # noqa: E731
    psi = np.asfortranarray(o.gram_schmidt_t(c.psi0()))
    nb = psi.shape[1]
    h = np.zeros_like(psi, order="F")
    g.hamiltonian(1, 1, psi, h, 1, c.ML, 1, nb)
    out["hpsi"] = rel(h, o.hamiltonian(psi))
    # the split operators (projection, then the scatter of a host uVunk)
    uv = np.zeros((c.nzlma, nb), order="F")
    g.op_nonlocal_project(psi, uv)
    h2 = np.zeros_like(psi, order="F")
    g.op_local(1, psi, h2)
    g.op_nonlocal_add(uv, h2)
    out["split"] = rel(h2, o.hamiltonian(psi))
    u = np.array(psi, order="F", copy=True)
    esp, res = np.zeros(nb), np.zeros(nb)
    g.conjugate_gradient(1, c.ML, nb, 1, 1, u, esp, res, ncg=4, mloop=3)
    ru, resp, rres, _ = o.conjugate_gradient(psi, 4, 3)
    out["cg"] = max(rel(esp, resp), rel(res, rres))
    w = np.zeros(nb)
    g.orth_subspace_diag(1, 1, np.array(ru, order="F", copy=True), w)
    _, ref_w, _ = o.subspace_diag_la(o.gram_schmidt_t(ru))
    out["rr_eig"] = rel(w, ref_w)
    occ = np.zeros(nb)
    occ[: nb // 2] = 2.0
    f = np.zeros((3, c.natom), order="F")
    g.calc_force_ps_nloc2(c.natom, f, psi, occ)
    out["force"] = rel(f.T, o.force_nloc(psi, occ))
    out["sync"] = L.rsdft_gpu_synchronize()
    # one check made to fail: reported once, then cleared
    out["selftest"] = L.rsdft_gpu_selftest_check()
    out["sync_after"] = L.rsdft_gpu_synchronize()
    out["message"] = L.rsdft_gpu_last_error().decode()
    out["sync_cleared"] = L.rsdft_gpu_synchronize()
    h3 = np.zeros_like(psi, order="F")
    g.hamiltonian(1, 1, psi, h3, 1, c.ML, 1, nb)
    out["hpsi_after"] = rel(h3, o.hamiltonian(psi))
    torch.cuda.synchronize()
    return out


def test_debug_build_parity_and_check_report():
    from rsdft_b200 import build

    build.build(check=True)
    env = dict(os.environ, RSDFT_GPU_CHECK="1")
    r = subprocess.run([sys.executable, os.path.abspath(__file__)], env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert out["lib"] == "librsdft_gpu_check.so" and out["checked"] == 1
    for k in ("hpsi", "split", "cg", "rr_eig", "force", "hpsi_after"):
        assert out[k] <= TOL, (k, out[k])
    assert out["sync"] == 0, out  # no check failed on valid inputs
    assert out["selftest"] == 0
    assert out["sync_after"] == -8  # RSDFT_ECHECK
    assert "site 99, index 4" in out["message"], out["message"]
    assert out["sync_cleared"] == 0


def test_normal_build_has_no_checks(gpu):
    from rsdft_b200 import _lib

    L = _lib.load()
    assert L.rsdft_gpu_checked_build() == 0
    assert L.rsdft_gpu_selftest_check() == -6  # EUNSUP: nothing launched
    assert L.rsdft_gpu_synchronize() == 0


if __name__ == "__main__":
    print(json.dumps(child()))
