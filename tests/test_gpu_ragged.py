"""Band counts that fill no tile evenly, through the FP64 path against the
oracle: one band, 37 bands (prime: every tile and chunk of the kernels has
a ragged edge) and 129 bands (one past a 128-band tile) on the 64-atom cell
(48^3 grid), and 37 bands in the 3-term split-BF16 form.

FP64 tolerance 1e-12 relative, the plain form's bar; the split form to the
3e-6 of its own tests."""
import numpy as np
import pytest
import torch

from rsdft_b200 import api

from test_gpu_parity import TOL, dev, host, overlap_check, prepare, rel

pytestmark = pytest.mark.gpu

RAGGED = [1, 37, 129]


@pytest.mark.parametrize("nb", RAGGED)
def test_hpsi_ragged(gpu, cells, nb):
    c, o = prepare(gpu, cells, "si64")
    psi = np.asfortranarray(c.psi0()[:, :nb])
    out = api.fortran_empty(c.ML, nb)
    gpu.hamiltonian(1, 1, dev(psi), out, 1, c.ML, 1, nb)
    torch.cuda.synchronize()
    assert rel(host(out), o.hamiltonian(psi)) <= TOL


@pytest.mark.parametrize("nb", RAGGED)
def test_cg_sweep_ragged(gpu, cells, nb):
    c, o = prepare(gpu, cells, "si64")
    q = o.gram_schmidt_t(np.asfortranarray(c.psi0()[:, :nb]))
    ru, resp, rres, _ = o.conjugate_gradient(q, 4, 3)
    u = dev(q)
    esp = torch.zeros(nb, dtype=torch.float64, device="cuda")
    res = torch.zeros_like(esp)
    gpu.conjugate_gradient(1, c.ML, nb, 1, 1, u, esp, res, ncg=4, mloop=3)
    torch.cuda.synchronize()
    assert rel(host(esp), resp) <= TOL
    assert rel(host(res), rres) <= TOL
    assert rel(host(u), ru) <= TOL


@pytest.mark.parametrize("nb", RAGGED[1:])
def test_rayleigh_ritz_ragged(gpu, cells, nb):
    """gram_schmidt + subspace_diag (one step) on a CG sweep's bands."""
    c, o = prepare(gpu, cells, "si64")
    q = o.gram_schmidt_t(np.asfortranarray(c.psi0()[:, :nb]))
    u0, _, _, _ = o.conjugate_gradient(q, 4, 3)
    ref, w, _ = o.subspace_diag_la(o.gram_schmidt_t(u0))
    u = dev(u0)
    esp = torch.zeros(nb, dtype=torch.float64, device="cuda")
    gpu.orth_subspace_diag(1, 1, u, esp)
    torch.cuda.synchronize()
    g = host(u)
    assert rel(host(esp), w) <= TOL
    assert np.abs(g.T @ g * c.dV - np.eye(nb)).max() <= 1e-12
    assert overlap_check(g, ref, w, c.dV) <= 1e-9


def test_one_band_gram_schmidt_and_subspace(gpu, cells):
    """A single band: Gram-Schmidt normalises it, the subspace step returns
    its Rayleigh quotient."""
    c, o = prepare(gpu, cells, "si64")
    psi = np.asfortranarray(c.psi0()[:, :1])
    u = dev(psi)
    gpu.gram_schmidt(1, 1, 1, 1, u)
    esp = torch.zeros(1, dtype=torch.float64, device="cuda")
    gpu.subspace_diag(1, 1, u, esp)
    torch.cuda.synchronize()
    ref = psi / np.sqrt((psi * psi).sum() * c.dV)
    g = host(u)
    assert rel(np.abs(g), np.abs(ref)) <= TOL
    e = float((ref[:, 0] @ o.hamiltonian(ref)[:, 0]) * c.dV)
    assert abs(float(host(esp)[0]) - e) <= TOL * abs(e)


def test_mixed_rayleigh_ritz_ragged(gpu, cells):
    c, o = prepare(gpu, cells, "si64")
    nb = 37
    q = o.gram_schmidt_t(np.asfortranarray(c.psi0()[:, :nb]))
    u0, _, _, _ = o.conjugate_gradient(q, 4, 3)
    _, w, _ = o.subspace_diag_la(o.gram_schmidt_t(u0))
    u = dev(u0)
    esp = torch.zeros(nb, dtype=torch.float64, device="cuda")
    gpu.orth_subspace_diag(1, 1, u, esp, mode=api.MODE_MIXED_BF16X3)
    torch.cuda.synchronize()
    assert np.abs(host(esp) - w).max() <= 3e-6 * max(1.0, np.abs(w).max())
