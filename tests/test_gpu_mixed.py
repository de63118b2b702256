"""Mixed-precision forms (tcgen05 split-BF16 / split-TF32 contractions, FP32
CG sweeps) against the FP64 oracle on seeded cells.

Tolerances: the 3-term BF16 split keeps 24 significant bits per operand, the
2-term TF32 split 22 and the 2-term BF16 split 16; the FP32 accumulation is
drained to FP64 every 128 terms, so the 3-term BF16 and the TF32 contractions
agree with FP64 to ~1e-7 .. 1e-6 relative; orthogonality after mixed
CholeskyQR2 is at that level, not the FP64 1e-12 (the FP64 finalisation
restores that).  The 64-atom cell (48^3, 160 bands) is the contraction
workload of the precision comparison: every form's orthogonality and
eigenvalue error against the FP64 oracle is reported by
test_contraction_forms_report.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from rsdft_b200 import api

from test_gpu_parity import dev, host, overlap_check, prepare, rel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode,tol", [(api.MODE_MIXED_BF16X3, 3e-6), (api.MODE_MIXED_TF32, 1e-5), (api.MODE_MIXED_BF16X2, 2e-4)])
@pytest.mark.parametrize("name,nb", [("si8", 32), ("si64", 160)])
def test_mixed_gram_schmidt(gpu, cells, mode, tol, name, nb):
    c, o = prepare(gpu, cells, name)
    psi = np.asfortranarray(c.psi0()[:, :nb])
    ref = o.gram_schmidt_t(psi)
    u = dev(psi)
    gpu.gram_schmidt(1, nb, 1, 1, u, mode=mode)
    torch.cuda.synchronize()
    g = host(u)
    orth = np.abs(g.T @ g * c.dV - np.eye(nb)).max()
    assert orth <= tol, f"orthogonality {orth:.2e}"
    assert rel(g, ref) <= 50 * tol


@pytest.mark.parametrize("mode,tol", [(api.MODE_MIXED_BF16X3, 3e-6), (api.MODE_MIXED_TF32, 1e-5), (api.MODE_MIXED_BF16X2, 1e-4)])
def test_mixed_subspace_diag(gpu, cells, mode, tol):
    c, o = prepare(gpu, cells, "si64")
    nb = 160
    psi = o.gram_schmidt_t(np.asfortranarray(c.psi0()[:, :nb]))
    ref, w, _ = o.subspace_diag_la(psi)
    u = dev(psi)
    esp = torch.zeros(nb, dtype=torch.float64, device="cuda")
    gpu.subspace_diag(1, 1, u, esp, mode=mode)
    torch.cuda.synchronize()
    e = host(esp)
    assert np.abs(e - w).max() <= tol * max(1.0, np.abs(w).max())
    assert overlap_check(host(u), ref, w, c.dV, gap_tol=1e-3) <= 1e3 * tol


@pytest.mark.parametrize("mode,tol", [(api.MODE_MIXED_BF16X3, 3e-6), (api.MODE_MIXED_TF32, 1e-5), (api.MODE_MIXED_BF16X2, 1e-4)])
def test_mixed_orth_subspace_diag(gpu, cells, mode, tol):
    c, o = prepare(gpu, cells, "si64")
    nb = 160
    q = o.gram_schmidt_t(np.asfortranarray(c.psi0()[:, :nb]))
    u0, _, _, _ = o.conjugate_gradient(q, 4, 3)
    ref, w, _ = o.subspace_diag_la(o.gram_schmidt_t(u0))
    u = dev(u0)
    esp = torch.zeros(nb, dtype=torch.float64, device="cuda")
    gpu.orth_subspace_diag(1, 1, u, esp, mode=mode)
    torch.cuda.synchronize()
    g = host(u)
    assert np.abs(host(esp) - w).max() <= tol * max(1.0, np.abs(w).max())
    assert np.abs(g.T @ g * c.dV - np.eye(nb)).max() <= 10 * tol


def test_mixed_sweep_matches_separate_calls(gpu, cells):
    """The one-call sweep (FP32 bands handed to Rayleigh-Ritz) tracks CG +
    orth_subspace_diag made as separate calls."""
    c, o = prepare(gpu, cells, "si64")
    nb = 160
    q = o.gram_schmidt_t(np.asfortranarray(c.psi0()[:, :nb]))
    ua, ub = dev(q), dev(q)
    ea = torch.zeros(nb, dtype=torch.float64, device="cuda")
    eb, ra, rb = torch.zeros_like(ea), torch.zeros_like(ea), torch.zeros_like(ea)
    gpu.conjugate_gradient(1, c.ML, nb, 1, 1, ua, ea, ra, ncg=4, mloop=3, mode=api.MODE_MIXED_BF16X3)
    gpu.orth_subspace_diag(1, 1, ua, ea, mode=api.MODE_MIXED_BF16X3)
    gpu.eigensolver_sweep(1, 1, ub, eb, rb, ncg=4, mloop=3, mode=api.MODE_MIXED_BF16X3)
    torch.cuda.synchronize()
    assert np.abs(host(ea) - host(eb)).max() <= 3e-6 * max(1.0, np.abs(host(ea)).max())
    assert np.abs(host(ra) - host(rb)).max() <= 1e-12 * max(1.0, np.abs(host(ra)).max())
    g = host(ub)
    assert np.abs(g.T @ g * c.dV - np.eye(nb)).max() <= 3e-5


def test_mixed_cg_sweep_fp32(gpu, cells):
    c, o = prepare(gpu, cells, "si8")
    q = o.gram_schmidt_t(c.psi0())
    ru, resp, rres, _ = o.conjugate_gradient(q, 4, 3)
    u = dev(q)
    esp = torch.zeros(c.nband, dtype=torch.float64, device="cuda")
    res = torch.zeros_like(esp)
    gpu.conjugate_gradient(1, c.ML, c.nband, 1, 1, u, esp, res, ncg=4, mloop=3, mode=api.MODE_MIXED_BF16X3)
    torch.cuda.synchronize()
    # FP32 storage and arithmetic in the sweeps: eigenvalue estimates to ~1e-6
    assert np.abs(host(esp) - resp).max() <= 1e-5 * max(1.0, np.abs(resp).max())


def test_mixed_iteration_tracks_fp64(gpu, cells):
    """Three full iterations in the mixed form stay within 1e-5 Ha of FP64."""
    c, o = prepare(gpu, cells, "si8")
    q = o.gram_schmidt_t(c.psi0())
    ua, ub = dev(q), dev(q)
    ea = torch.zeros(c.nband, dtype=torch.float64, device="cuda")
    eb = torch.zeros_like(ea)
    res = torch.zeros_like(ea)
    for _ in range(3):
        gpu.eigensolver_iteration(ua, ea, res, ncg=4, mloop=3, mode=api.MODE_FP64)
        gpu.eigensolver_iteration(ub, eb, res, ncg=4, mloop=3, mode=api.MODE_MIXED_BF16X3)
    torch.cuda.synchronize()
    assert np.abs(host(ea) - host(eb)).max() <= 1e-5


def test_mixed_then_fp64_closing_pass(gpu, cells):
    """Mixed iterations, then the FP64 closing pass: orthogonality at the FP64
    level and Rayleigh quotients close to the all-FP64 run."""
    c, o = prepare(gpu, cells, "si8")
    q = o.gram_schmidt_t(c.psi0())
    ua, ub = dev(q), dev(q)
    ea = torch.zeros(c.nband, dtype=torch.float64, device="cuda")
    eb = torch.zeros_like(ea)
    res = torch.zeros_like(ea)
    for _ in range(4):
        gpu.eigensolver_iteration(ua, ea, res, ncg=4, mloop=3, mode=api.MODE_FP64)
        gpu.eigensolver_iteration(ub, eb, res, ncg=4, mloop=3, mode=api.MODE_MIXED_BF16X3)
    gpu.finalize_fp64(ua, ea, res)
    gpu.finalize_fp64(ub, eb, res)
    torch.cuda.synchronize()
    g = host(ub)
    assert np.abs(g.T @ g * c.dV - np.eye(c.nband)).max() <= 1e-12
    assert np.abs(host(ea) - host(eb)).max() <= 1e-5


@pytest.mark.parametrize("mode,tol", [(api.MODE_MIXED_BF16X3, 3e-6), (api.MODE_MIXED_TF32, 1e-5), (api.MODE_MIXED_BF16X2, 1e-4)])
def test_mixed_general_shapes(gpu, cells, mode, tol):
    """ML = 18^3 (not a multiple of 32: the rotation takes the transposed
    split; FP32 rows of 18 take the general stencil) and 36 bands (the band
    dimension padded to 40): Rayleigh-Ritz step and sweep against the oracle."""
    c, o = prepare(gpu, cells, "si8_g18")
    nb = c.nband
    q = o.gram_schmidt_t(np.asfortranarray(c.psi0()))
    u0, _, _, _ = o.conjugate_gradient(q, 4, 3)
    ref, w, _ = o.subspace_diag_la(o.gram_schmidt_t(u0))
    u = dev(u0)
    esp = torch.zeros(nb, dtype=torch.float64, device="cuda")
    gpu.orth_subspace_diag(1, 1, u, esp, mode=mode)
    torch.cuda.synchronize()
    g = host(u)
    assert np.abs(host(esp) - w).max() <= tol * max(1.0, np.abs(w).max())
    assert np.abs(g.T @ g * c.dV - np.eye(nb)).max() <= 10 * tol
    ub = dev(q)
    eb = torch.zeros(nb, dtype=torch.float64, device="cuda")
    rb = torch.zeros_like(eb)
    gpu.eigensolver_sweep(1, 1, ub, eb, rb, ncg=4, mloop=3, mode=mode)
    torch.cuda.synchronize()
    # FP32 CG sweep: eigenvalue estimates to ~1e-5 of the FP64 sequence (the
    # 22-bit TF32 split 2.5 times looser than the 24-bit BF16 one, as in
    # test_contraction_forms_report)
    sweep_tol = {api.MODE_MIXED_BF16X3: 1e-5, api.MODE_MIXED_TF32: 3e-5}.get(mode, tol)
    assert np.abs(host(eb) - w).max() <= sweep_tol * max(1.0, np.abs(w).max())


def test_mixed_sweep_host_array_overlapped_upload(gpu, cells):
    """A host array in the mixed sweep is uploaded in band blocks on a copy
    stream, each block's CG starting when its upload lands; the bands' CG
    steps are independent, so the result equals the sweep on a device array."""
    c, o = prepare(gpu, cells, "si64")
    nb = 160
    q = np.asfortranarray(o.gram_schmidt_t(np.asfortranarray(c.psi0()[:, :nb])))
    ud = dev(q)
    ed = torch.zeros(nb, dtype=torch.float64, device="cuda")
    rd = torch.zeros_like(ed)
    gpu.eigensolver_sweep(1, 1, ud, ed, rd, ncg=4, mloop=3, mode=api.MODE_MIXED_BF16X3)
    host_pinned = torch.empty((nb, c.ML), dtype=torch.float64, pin_memory=True)
    host_pinned.copy_(torch.from_numpy(np.ascontiguousarray(q.T)))
    uh = host_pinned.numpy().T  # (ML, nb) Fortran view of pinned memory
    eh = np.zeros(nb)
    rh = np.zeros(nb)
    gpu.eigensolver_sweep(1, 1, uh, eh, rh, ncg=4, mloop=3, mode=api.MODE_MIXED_BF16X3)
    torch.cuda.synchronize()
    assert np.array_equal(host(ed), eh) and np.array_equal(host(rd), rh)
    assert np.array_equal(host(ud), uh)


def test_contraction_forms_report(gpu, cells, capsys):
    """The 64-atom cell (48^3, 160 bands): Gram-Schmidt and the Rayleigh-Ritz
    step of every precision form against the FP64 oracle -- orthogonality
    max |dV psi^T psi - I| and the largest eigenvalue error (Ha).  The FP64
    form meets 1e-12; the split forms order by their operand bits."""
    c, o = prepare(gpu, cells, "si64")
    nb = 160
    psi = np.asfortranarray(c.psi0()[:, :nb])
    q = o.gram_schmidt_t(psi)
    u0, _, _, _ = o.conjugate_gradient(q, 4, 3)
    ref, w, _ = o.subspace_diag_la(o.gram_schmidt_t(u0))
    rows = {}
    for name, mode in (("fp64", api.MODE_FP64), ("bf16x3", api.MODE_MIXED_BF16X3), ("tf32", api.MODE_MIXED_TF32),
                       ("bf16x2", api.MODE_MIXED_BF16X2)):
        u = dev(psi)
        gpu.gram_schmidt(1, nb, 1, 1, u, mode=mode)
        g = host(u)
        orth = float(np.abs(g.T @ g * c.dV - np.eye(nb)).max())
        v = dev(u0)
        esp = torch.zeros(nb, dtype=torch.float64, device="cuda")
        gpu.orth_subspace_diag(1, 1, v, esp, mode=mode)
        torch.cuda.synchronize()
        eig = float(np.abs(host(esp) - w).max())
        rows[name] = (orth, eig)
    with capsys.disabled():
        print("\nform    GS orthogonality   Rayleigh-Ritz eigenvalue error (Ha)")
        for name, (orth, eig) in rows.items():
            print(f"{name:7s} {orth:16.2e}   {eig:.2e}")
    assert rows["fp64"][0] <= 1e-12 and rows["fp64"][1] <= 1e-12 * max(1.0, np.abs(w).max())
    assert rows["bf16x3"][1] <= 3e-6 and rows["tf32"][1] <= 1e-5 and rows["bf16x2"][1] <= 1e-4
    assert rows["bf16x2"][1] > rows["bf16x3"][1]
