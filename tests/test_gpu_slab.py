"""The z-slab driver on the GPU backend (library entries op_local,
op_nonlocal_project / _add, gram, overlap_cholesky, rr_reduced, rotate).

One GPU cannot hold ranks that wait on one another, so the multi-rank cases
run the ranks one after the other in one process, with the exchanges done on
the host between them: each slab's halo planes are filled from the global
bands and the projector partials are summed before the scatter.  The halo
exchange and the all-reduces themselves run on gloo ranks in test_slab.py.
The one-rank case runs the whole driver, exchange included (the halo wraps
onto the rank's own planes)."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from rsdft_b200 import api
from rsdft_b200.slab import GpuSlabBackend, SlabDomain, SlabSolver

from test_gpu_parity import TOL, dev, host, rel

pytestmark = pytest.mark.gpu


def _ext(d, psi_g):
    return dev(d.ext_from_global(psi_g))


def test_one_rank_driver_si64(gpu, cells):
    c = cells("si64")
    nb = 16
    psi_g = np.asfortranarray(c.psi0(nb))
    d = SlabDomain(c.ngrid, c.md, 0, 1)
    sol = SlabSolver(d, GpuSlabBackend(gpu, d, c), None)
    psi = sol.empty_bands(nb)
    psi.fill_(float("nan"))
    d.own(psi).copy_(dev(psi_g))
    hpsi = sol.empty_bands(nb)
    sol.hamiltonian(psi, hpsi)
    torch.cuda.synchronize()
    assert bool(torch.isfinite(psi).all())
    o = O.Oracle(c)
    assert rel(host(d.own(hpsi)), o.hamiltonian(psi_g)) <= TOL
    esp = torch.zeros(nb, dtype=torch.float64, device="cuda")
    sol.rayleigh_ritz(psi, esp)
    torch.cuda.synchronize()
    q, w, _ = o.subspace_diag_la(o.gram_schmidt_t(psi_g))
    assert rel(host(esp), w) <= TOL
    g = host(d.own(psi))
    assert np.abs(g.T @ g * c.dV - np.eye(nb)).max() <= 1e-12
    assert np.abs(np.abs(np.diag(q.T @ g * c.dV)) - 1.0).max() <= 1e-9


def _virtual_ranks(gpu, c, nranks, psi_g):
    """H psi and the Gram sums of nranks slabs computed one after another."""
    nb = psi_g.shape[1]
    parts, hp, grams = [], [], []
    usum = api.fortran_empty(c.nzlma, nb)
    usum.zero_()
    for r in range(nranks):
        d = SlabDomain(c.ngrid, c.md, r, nranks)
        b = GpuSlabBackend(gpu, d, c)
        psi = _ext(d, psi_g)
        h = b.empty(d.ml_ext, nb)
        h.fill_(float("nan"))
        b.op_local(psi, h)
        u = api.fortran_empty(c.nzlma, nb)
        b.project(psi, u)
        usum += u
        parts.append((d, psi))
        hp.append(h)
    for (d, psi), h in zip(parts, hp):
        b = GpuSlabBackend(gpu, d, c)
        b.add(usum, h)
        s = api.fortran_empty(nb, nb)
        b.gram(d.own(psi), d.own(psi), s, c.dV, 0)
        hs = api.fortran_empty(nb, nb)
        b.gram(d.own(psi), d.own(h), hs, c.dV, 1)
        grams.append((host(s), host(hs)))
    torch.cuda.synchronize()
    got = np.concatenate([host(d.own(h)) for (d, _), h in zip(parts, hp)])
    return got, sum(g[0] for g in grams), sum(g[1] for g in grams), parts


@pytest.mark.parametrize("name,nranks,nb", [("si216", 2, 16), ("si216", 3, 8), ("si64", 8, 8)])
def test_virtual_slabs_match_single_domain(gpu, cells, name, nranks, nb):
    """Slabs of 36 / 24 planes (si216) and of 6 planes, thinner than the
    12 halo planes around them (si64 on 8): own-plane H psi 1e-12, Gram
    sums 1e-12, and the Rayleigh-Ritz step from the summed matrices."""
    c = cells(name)
    psi_g = np.asfortranarray(c.psi0(nb))
    got, s, hs, parts = _virtual_ranks(gpu, c, nranks, psi_g)
    o = O.Oracle(c)
    ref = o.hamiltonian(psi_g)
    assert rel(got, ref) <= TOL
    assert rel(s, psi_g.T @ psi_g * c.dV) <= TOL
    href = psi_g.T @ ref * c.dV
    assert rel(hs, 0.5 * (href + href.T)) <= TOL
    # the small steps on the summed matrices, then each slab's own rows
    rinv = api.fortran_empty(nb, nb)
    kappa = gpu.overlap_cholesky(dev(s), rinv)
    assert kappa < 1e3
    esp = torch.zeros(nb, dtype=torch.float64, device="cuda")
    w = api.fortran_empty(nb, nb)
    gpu.rr_reduced(rinv, dev(hs), esp, w)
    for d, psi in parts:
        gpu.rotate(d.own(psi), w)
    torch.cuda.synchronize()
    q, wref, _ = o.subspace_diag_la(o.gram_schmidt_t(psi_g))
    assert rel(host(esp), wref) <= TOL
    g = np.concatenate([host(d.own(psi)) for d, psi in parts])
    assert np.abs(g.T @ g * c.dV - np.eye(nb)).max() <= 1e-12
    assert np.abs(np.abs(np.diag(q.T @ g * c.dV)) - 1.0).max() <= 1e-9


def test_op_local_rejects_planes_outside_grid(gpu, cells):
    c = cells("si8")
    gpu.setup(c)
    psi = dev(np.asfortranarray(c.psi0(2)))
    out = api.fortran_empty(c.ML, 2)
    with pytest.raises(api.RsdftError):
        gpu.op_local(1, psi, out, z0=20, nz=10)
