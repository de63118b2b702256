"""The z-slab driver on the GPU backend (library entries op_local,
op_nonlocal_project / _add, gram, overlap_cholesky, rr_reduced, rotate), and
the split iteration (CG on each rank's bands, Rayleigh-Ritz on each rank's
planes) on the whole-grid backend.

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
from rsdft_b200.slab import (BandGridIteration, BandGridLayout, GpuBandBackend, GpuSlabBackend, SlabDomain,
                             SlabSolver)

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


def test_band_grid_iteration_one_rank_si64(gpu, cells):
    """The split iteration's driver on one rank (layout moves with no peer)
    against the library's one-call iteration on the same start: CG
    residuals 1e-12, Rayleigh-Ritz eigenvalues 1e-12, the same eigenvectors."""
    c = cells("si64")
    nb = 32
    q = np.asfortranarray(O.Oracle(c).gram_schmidt_t(np.asfortranarray(c.psi0(nb))))
    it = BandGridIteration(BandGridLayout(c.ngrid, nb, 0, 1), GpuBandBackend(gpu, c), None)
    u = dev(q)
    esp = torch.zeros(nb, dtype=torch.float64, device="cuda")
    res = torch.zeros_like(esp)
    it.iterate(u, esp, res, ncg=4, mloop=3)
    ref = dev(q)
    eref, rref = torch.zeros_like(esp), torch.zeros_like(esp)
    gpu.eigensolver_iteration(ref, eref, rref, ncg=4, mloop=3)
    torch.cuda.synchronize()
    assert rel(host(res), host(rref)) <= TOL
    assert rel(host(esp), host(eref)) <= TOL
    g, gr = host(u), host(ref)
    assert np.abs(g.T @ g * c.dV - np.eye(nb)).max() <= 1e-12
    assert np.abs(np.abs(np.diag(gr.T @ g * c.dV)) - 1.0).max() <= 1e-9


@pytest.mark.parametrize("nranks", [2, 3])
def test_band_grid_iteration_virtual_ranks_si64(gpu, cells, nranks):
    """The split iteration's per-rank steps for nranks ranks run one after
    another on the GPU (CG and H psi on each rank's bands, Gram partial sums
    on each rank's planes, summed here; the layout moves done by slicing on
    the host) against the library's one-call iteration on all bands."""
    c = cells("si64")
    nb = 48
    q = np.asfortranarray(O.Oracle(c).gram_schmidt_t(np.asfortranarray(c.psi0(nb))))
    b = GpuBandBackend(gpu, c)
    lay = [BandGridLayout(c.ngrid, nb, r, nranks) for r in range(nranks)]
    cg_out, h_out, res = [], [], np.zeros(nb)
    for L in lay:
        u = dev(q[:, L.b0:L.b0 + L.nb_own])
        e, r = b.vector(L.nb_own), b.vector(L.nb_own)
        b.cg(u, e, r, 4, 3, api.MODE_FP64)
        h = b.empty(c.ML, L.nb_own)
        b.hamiltonian(u, h)
        cg_out.append(host(u))
        h_out.append(host(h))
        res[L.b0:L.b0 + L.nb_own] = host(r)
    psi_all, h_all = np.concatenate(cg_out, axis=1), np.concatenate(h_out, axis=1)
    grids = [(dev(psi_all[L.rows[L.rank][0]:L.rows[L.rank][1]]), dev(h_all[L.rows[L.rank][0]:L.rows[L.rank][1]]))
             for L in lay]
    s = np.zeros((nb, nb))
    hs = np.zeros((nb, nb))
    for gp, gh in grids:
        t = b.empty(nb, nb)
        b.gram(gp, gp, t, c.dV, 0)
        s += host(t)
        b.gram(gp, gh, t, c.dV, 1)
        hs += host(t)
    rinv = b.empty(nb, nb)
    assert b.overlap_cholesky(dev(s), rinv) < 1e3
    esp = b.vector(nb)
    w = b.empty(nb, nb)
    b.rr_reduced(rinv, dev(hs), esp, w)
    for gp, _ in grids:
        b.rotate(gp, w)
    ref = dev(q)
    eref, rref = b.vector(nb), b.vector(nb)
    gpu.eigensolver_iteration(ref, eref, rref, ncg=4, mloop=3)
    torch.cuda.synchronize()
    assert rel(res, host(rref)) <= TOL
    assert rel(host(esp), host(eref)) <= TOL
    g = np.concatenate([host(gp) for gp, _ in grids])
    gr = host(ref)
    assert np.abs(g.T @ g * c.dV - np.eye(nb)).max() <= 1e-12
    assert np.abs(np.abs(np.diag(gr.T @ g * c.dV)) - 1.0).max() <= 1e-9


def test_band_grid_iteration_nccl_one_rank(gpu, cells):
    """The split iteration's driver over a real NCCL process group of one
    rank: its all-reduces of the Gram sums and the residuals run on the
    library's stream (the backend binds the library to torch's current
    stream), same result as without a process group."""
    import datetime
    import socket

    import torch.distributed as dist

    c = cells("si8")
    nb = 16
    q = np.asfortranarray(O.Oracle(c).gram_schmidt_t(np.asfortranarray(c.psi0(nb))))
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        out = []
        for group in (dist, None):
            it = BandGridIteration(BandGridLayout(c.ngrid, nb, 0, 1), GpuBandBackend(gpu, c), group)
            u = dev(q)
            esp = torch.zeros(nb, dtype=torch.float64, device="cuda")
            res = torch.zeros_like(esp)
            it.iterate(u, esp, res, ncg=4, mloop=3)
            torch.cuda.synchronize()
            out.append((host(u), host(esp), host(res)))
    finally:
        dist.destroy_process_group()
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a, b)
