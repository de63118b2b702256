"""z-slab decomposition on the host: plane split, halo index maps, projector
restriction, and world_size 2 / 3 gloo ranks computing H psi, the Gram sums
and the Rayleigh-Ritz step slab by slab, checked against the single-domain
oracle; the band split, the band <-> grid layout moves and whole iterations
with the CG band-parallel and the Rayleigh-Ritz step grid-parallel.  The per-slab compute here is the oracle (kinetic + local) and numpy
(projector partials and scatter, small dense steps); the GPU backend runs the
same driver in test_gpu_slab.py."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from oracle import oracle as O
from rsdft_b200 import api
from rsdft_b200.cell import build_cell
from rsdft_b200.slab import (BandGridIteration, BandGridLayout, SlabDomain, SlabSolver, halo_runs, split_bands,
                             split_planes)

TOL = 1e-12


def rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


class OracleSlabBackend:
    """The per-slab compute on the host: the oracle's H psi of the extended
    slab with no projectors (kinetic + local; the own planes read no
    wrapped plane), numpy projector partials and scatter
    (ps_nloc2_op_module.f90:161-175, 255-263) and numpy small dense steps."""

    def __init__(self, domain, cell):
        self.domain = domain
        self.cell = domain.slab_cell(cell)
        self.nzlma = self.cell.nzlma
        self.dV = self.cell.dV
        self.device = torch.device("cpu")
        bare = dict(vars(self.cell))
        bare.update(lma_ptr=np.zeros(1, np.int32), jjp=np.zeros(0, np.int32), uv=np.zeros(0),
                    iuv=np.zeros(0, np.int32), nzlma=0)
        import types

        self.oracle = O.Oracle(types.SimpleNamespace(**bare))
        ptr = self.cell.lma_ptr.astype(np.int64)
        self.lma_of = np.repeat(np.arange(self.nzlma), np.diff(ptr))
        self.jjp = self.cell.jjp.astype(np.int64)
        self.uv = self.cell.uv
        self.iuv = self.cell.iuv.astype(np.float64)

    def empty(self, rows, cols):
        return api.fortran_empty(rows, cols, device="cpu")

    def zeros(self, rows, cols):
        t = self.empty(rows, cols)
        t.zero_()
        return t

    def op_local(self, psi, hpsi):
        h = self.oracle.hamiltonian(psi.numpy())
        s = self.domain.own_slice()
        hpsi.numpy()[s] = h[s]

    def project(self, psi, u):
        acc = np.zeros((self.nzlma, psi.shape[1]))
        np.add.at(acc, self.lma_of, self.uv[:, None] * psi.numpy()[self.jjp])
        u.numpy()[:] = (self.iuv * self.dV)[:, None] * acc

    def add(self, u, hpsi):
        np.add.at(hpsi.numpy(), self.jjp, self.uv[:, None] * u.numpy()[self.lma_of])

    def gram(self, a, b, out, alpha, sym):
        c = alpha * (a.numpy().T @ b.numpy())
        out.numpy()[:] = 0.5 * (c + c.T) if sym else c

    def overlap_cholesky(self, s, rinv):
        r = np.linalg.cholesky(s.numpy()).T
        rinv.numpy()[:] = np.linalg.inv(r)
        d = np.abs(np.diag(r))
        return float((d.max() / d.min()) ** 2)

    def rr_reduced(self, rinv, hsub, esp, w):
        h = np.triu(hsub.numpy())
        h = h + np.triu(h, 1).T
        ri = rinv.numpy()
        e, v = np.linalg.eigh(ri.T @ h @ ri)
        esp.numpy()[:] = e
        w.numpy()[:] = ri @ v

    def rotate(self, psi_own, w):
        a = psi_own.numpy()
        a[:] = a @ w.numpy()


class OracleBandBackend(OracleSlabBackend):
    """The whole-grid compute of a rank on the host: the oracle's CG (band
    by band, cg_module.f90:97-430) and H psi on the rank's bands, numpy Gram
    sums and small dense steps."""

    def __init__(self, cell):
        self.oracle = O.Oracle(cell)
        self.ml = cell.ML
        self.dV = cell.dV
        self.device = torch.device("cpu")

    def vector(self, n):
        return torch.zeros(n, dtype=torch.float64)

    def cg(self, psi, esp, res, ncg, mloop, mode):
        u, e, r, _ = self.oracle.conjugate_gradient(np.asfortranarray(psi.numpy()), ncg, mloop)
        psi.numpy()[:] = u
        esp.numpy()[:] = e
        res.numpy()[:] = r

    def hamiltonian(self, psi, hpsi):
        hpsi.numpy()[:] = self.oracle.hamiltonian(np.asfortranarray(psi.numpy()))


# ------------------------------------------------------------ index maps
@pytest.mark.parametrize("n,parts", [(24, 1), (24, 2), (24, 5), (72, 8), (13, 4), (7, 7), (96, 3)])
def test_split_planes_reference_rule(n, parts):
    """InitParallel_RgridSol: part p holds as many points as there are i in
    [0, n) with mod(i, np) == p, after the parts before it."""
    ref = [sum(1 for i in range(n) if i % parts == p) for p in range(parts)]
    counts, offsets = split_planes(n, parts)
    assert counts == ref
    assert offsets == [sum(ref[:p]) for p in range(parts)]


def test_split_planes_rejects_empty_slabs():
    with pytest.raises(ValueError):
        split_planes(3, 4)


@pytest.mark.parametrize("n3,nranks,md", [(24, 1, 6), (24, 2, 6), (24, 3, 6), (12, 3, 6), (12, 5, 4),
                                          (72, 8, 6), (9, 4, 2), (8, 8, 3)])
def test_halo_runs_map_every_halo_plane(n3, nranks, md):
    sent = 0
    received = 0
    for r in range(nranks):
        d = SlabDomain((4, 4, n3), md, r, nranks)
        planes = d.global_planes()
        covered = []
        for run in d.recv:
            for k in range(run.n):
                assert 0 <= run.src + k < d.counts[run.peer]
                assert d.offsets[run.peer] + run.src + k == planes[run.dst + k]
                covered.append(run.dst + k)
        assert sorted(covered) == list(range(md)) + list(range(md + d.nz, 2 * md + d.nz))
        received += sum(run.n for run in d.recv)
        sent += sum(run.n for _, run in d.send)
        for q, run in d.send:
            assert run in halo_runs(n3, nranks, md, q) and run.peer == r
    assert sent == received == 2 * md * nranks


@pytest.mark.parametrize("nranks", [2, 3, 5])
def test_projector_restriction_partitions_entries(nranks):
    cell = build_cell("si8_g12")
    seen = []
    for r in range(nranks):
        d = SlabDomain(cell.ngrid, cell.md, r, nranks)
        ptr, jjp, uv = d.restrict_projectors(cell.lma_ptr, cell.jjp, cell.uv)
        assert ptr.shape[0] == cell.nzlma + 1
        g = jjp.astype(np.int64) + (d.z0 - d.md) * d.n12
        assert np.all((g >= d.z0 * d.n12) & (g < (d.z0 + d.nz) * d.n12))
        lma = np.repeat(np.arange(cell.nzlma), np.diff(ptr))
        seen.append(np.stack([lma, g, uv.view(np.int64)], axis=1))
    seen = np.concatenate(seen)
    glma = np.repeat(np.arange(cell.nzlma), np.diff(cell.lma_ptr))
    ref = np.stack([glma, cell.jjp.astype(np.int64), cell.uv.view(np.int64)], axis=1)
    order = lambda a: a[np.lexsort(a.T[::-1])]  # noqa: E731
    assert np.array_equal(order(seen), order(ref))


# ----------------------------------------------------------- gloo ranks
def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, name, nb, out):
    import datetime

    import torch.distributed as dist

    torch.set_num_threads(1)
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        cell = build_cell(name, with_duv=False)
        d = SlabDomain(cell.ngrid, cell.md, rank, world)
        sol = SlabSolver(d, OracleSlabBackend(d, cell), dist)
        psi_g = np.asfortranarray(cell.psi0(nb))
        psi = sol.empty_bands(nb)
        psi.numpy()[:] = d.ext_from_global(psi_g)
        # halo rows the exchange must overwrite
        psi.numpy()[: d.row0] = np.nan
        psi.numpy()[d.row0 + d.ml_own:] = np.nan
        hpsi = sol.empty_bands(nb)
        hpsi.zero_()
        sol.hamiltonian(psi, hpsi)
        halo_ok = bool(np.isfinite(psi.numpy()).all())
        s = sol.gram(psi, psi).numpy().copy()
        h = sol.gram(psi, hpsi, sym=1).numpy().copy()
        esp = torch.zeros(nb, dtype=torch.float64)
        sol.rayleigh_ritz(psi, esp)
        out[rank] = (d.own(hpsi).numpy().copy(), halo_ok, s, h, esp.numpy().copy(), d.own(psi).numpy().copy())
    finally:
        dist.destroy_process_group()


def _run(world, name, nb):
    O.lib()  # build the oracle library once, before the ranks load it
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.spawn(_rank, args=(world, port, name, nb, out), nprocs=world, join=True)
    return [out[r] for r in range(world)]


@pytest.mark.parametrize("world,name", [(2, "si8"), (3, "si8"), (3, "si8_g12")])
def test_slab_ranks_match_single_domain(world, name):
    """H psi, dV psi^T psi, dV sym(psi^T H psi) and the Rayleigh-Ritz step
    (eigenvalues, orthonormality, eigenspaces) from slab ranks against the
    single-domain oracle.  si8_g12 on 3 ranks has 4-plane slabs, thinner than
    the Md = 6 halo: halos come from two ranks and across the wrap."""
    nb = 8
    res = _run(world, name, nb)
    cell = build_cell(name, with_duv=False)
    o = O.Oracle(cell)
    psi = np.asfortranarray(cell.psi0(nb))
    ref = o.hamiltonian(psi)
    got = np.concatenate([r[0] for r in res])
    assert all(r[1] for r in res), "halo planes left unfilled"
    assert rel(got, ref) <= TOL
    s_ref = psi.T @ psi * cell.dV
    h_ref = psi.T @ ref * cell.dV
    h_ref = 0.5 * (h_ref + h_ref.T)
    for r in res:
        assert rel(r[2], s_ref) <= TOL
        assert rel(r[3], h_ref) <= TOL
    q, w, _ = o.subspace_diag_la(o.gram_schmidt_t(psi))
    for r in res:
        assert rel(r[4], w) <= TOL
    g = np.concatenate([r[5] for r in res])
    assert np.abs(g.T @ g * cell.dV - np.eye(nb)).max() <= 1e-12
    # same eigenvectors up to sign (the eigenvalues of random bands are apart)
    ov = np.abs(np.diag(q.T @ g * cell.dV))
    assert np.abs(ov - 1.0).max() <= 1e-9


def test_one_rank_is_its_own_neighbour():
    """One rank: the halo wraps onto the rank's own planes, no process group."""
    cell = build_cell("si8_g12", with_duv=False)
    d = SlabDomain(cell.ngrid, cell.md, 0, 1)
    sol = SlabSolver(d, OracleSlabBackend(d, cell), None)
    psi_g = np.asfortranarray(cell.psi0(4))
    psi = sol.empty_bands(4)
    psi.numpy()[:] = np.nan
    d.own(psi).numpy()[:] = psi_g
    hpsi = sol.empty_bands(4)
    sol.hamiltonian(psi, hpsi)
    assert rel(d.own(hpsi).numpy(), O.Oracle(cell).hamiltonian(psi_g)) <= TOL


@pytest.mark.parametrize("nb,parts", [(32, 2), (480, 8), (160, 3), (7, 7)])
def test_split_bands_reference_rule(nb, parts):
    """parallel_module.f90:366-377: rank j holds as many bands as there are
    i with mod(i, np_band) == j, the ranks' bands contiguous in order."""
    counts, offsets = split_bands(nb, parts)
    assert counts == [sum(1 for i in range(nb) if i % parts == j) for j in range(parts)]
    assert offsets == [sum(counts[:j]) for j in range(parts)]


def _layout_rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    torch.set_num_threads(1)
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        ngrid, nb = (6, 5, 7), 9
        L = BandGridLayout(ngrid, nb, rank, world)
        full = np.arange(L.ml * nb, dtype=np.float64).reshape(nb, L.ml).T  # (ML, nb) global
        band = api.fortran_empty(L.ml, L.nb_own, device="cpu")
        band.numpy()[:] = full[:, L.b0:L.b0 + L.nb_own]
        grid = api.fortran_empty(L.ml_own, nb, device="cpu")
        grid.fill_(float("nan"))
        L.to_grid(band, grid, dist)
        r0, r1 = L.rows[rank]
        grid_ok = np.array_equal(grid.numpy(), full[r0:r1])
        grid.mul_(-1.0)
        back = api.fortran_empty(L.ml, L.nb_own, device="cpu")
        back.fill_(float("nan"))
        L.to_band(grid, back, dist)
        out[rank] = (grid_ok, np.array_equal(back.numpy(), -full[:, L.b0:L.b0 + L.nb_own]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_band_grid_layout_moves(world):
    """to_grid gives each rank its planes of every band; to_band brings each
    rank's bands back on the whole grid (7 planes and 9 bands on 2 and 3
    ranks: uneven parts both ways)."""
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.spawn(_layout_rank, args=(world, port, out), nprocs=world, join=True)
    for r in range(world):
        assert out[r] == (True, True), (r, out[r])


def _iter_rank(rank, world, port, name, nb, out):
    import datetime

    import torch.distributed as dist

    torch.set_num_threads(1)
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        cell = build_cell(name, with_duv=False)
        o = O.Oracle(cell)
        start = o.gram_schmidt_t(np.asfortranarray(cell.psi0(nb)))
        L = BandGridLayout(cell.ngrid, nb, rank, world)
        it = BandGridIteration(L, OracleBandBackend(cell), dist)
        psi = api.fortran_empty(cell.ML, L.nb_own, device="cpu")
        psi.numpy()[:] = start[:, L.b0:L.b0 + L.nb_own]
        esp = torch.zeros(nb, dtype=torch.float64)
        res = torch.zeros(nb, dtype=torch.float64)
        it.iterate(psi, esp, res, ncg=4, mloop=3)
        out[rank] = (psi.numpy().copy(), esp.numpy().copy(), res.numpy().copy())
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,name", [(2, "si8"), (3, "si8_g12")])
def test_band_grid_iteration_matches_single_domain(world, name):
    """One iteration with the CG on each rank's bands and the Rayleigh-Ritz
    step on each rank's planes against the single-domain oracle iteration
    (conjugate_gradient -> gram_schmidt_t -> subspace_diag_la): CG residuals
    bitwise (the CG is band by band), eigenvalues 1e-12, orthonormal bands
    spanning the same eigenvectors."""
    nb = 16
    O.lib()
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.spawn(_iter_rank, args=(world, port, name, nb, out), nprocs=world, join=True)
    cell = build_cell(name, with_duv=False)
    o = O.Oracle(cell)
    start = o.gram_schmidt_t(np.asfortranarray(cell.psi0(nb)))
    u, _, rref, _ = o.conjugate_gradient(start, 4, 3)
    q, w, _ = o.subspace_diag_la(o.gram_schmidt_t(u))
    g = np.concatenate([out[r][0] for r in range(world)], axis=1)
    for r in range(world):
        assert np.array_equal(out[r][2], rref)
        assert rel(out[r][1], w) <= TOL
    assert np.abs(g.T @ g * cell.dV - np.eye(nb)).max() <= 1e-12
    assert np.abs(np.abs(np.diag(q.T @ g * cell.dV)) - 1.0).max() <= 1e-9
