"""z-slab decomposition of the real-space grid over ranks (one GPU each).

Split (rgrid_sol_module.f90:79-113, InitParallel_RgridSol): the N points of
an axis cut into np parts give part p as many points as there are i in
[0, N) with mod(i, np) == p, i.e. N // np + (1 if p < N % np else 0), placed
after the parts before it.  Only z is cut here (np = (1, 1, nranks)), so rank
r owns the whole planes [z0(r), z0(r) + nz(r)) of the (n1, n2, n3) grid, x
fastest (grid index i1 + n1 i2 + n1 n2 i3, as in the projector tables).

Layout in device memory: a rank keeps its bands in an extended slab,
column-major (n1 n2 (nz + 2 Md), nb): Md halo planes, its own nz planes, Md
halo planes.  Its own rows are the view ``own(t)`` (leading dimension the
extended row count), so the stencil, the projections, the Gram sums and the
rotations run on the slab in place, with no copy between the caller's bands
and a halo buffer.

One H psi (hamiltonian_module.f90:20-72 on a grid split over comm_grid):

1. halo exchange (bcset_3_module.f90:15-151): the Md planes either side come
   from the ranks that own them (from several ranks when slabs are thinner
   than Md, from the rank itself across the periodic boundary when it owns
   them), one point-to-point message per peer and direction holding every
   band's planes, packed (nb, planes, n1 n2); NCCL send/recv between GPUs,
   gloo on the host;
2. kinetic + local potential on the own planes (op_kinetic + op_localpot),
   the stencil reading the halo planes in place;
3. the nonlocal part: projections over the own points (partial sums), one
   all-reduce of the (nzlma, nb) block, the scatter-add at the own points
   (ps_nloc2_op_module.f90:161-263).  The reference sends each partial only
   to the ranks whose slabs its sphere touches (:179-250); one all-reduce of
   the block gives every rank the same sums.

The Gram sums of Gram-Schmidt and the subspace matrix (gram_schmidt_t_module
.f90:187-195, subspace_diag_la_module.f90:96-122) are each rank's own rows
followed by an all-reduce; the small problems are then solved redundantly on
every rank and each rank rotates its own rows (subspace_rotv_sl_module.f90:
92).

The per-slab compute goes through a backend: ``GpuSlabBackend`` calls the
library's entries on this rank's GPU.  Every rank takes the same collective
steps in the same order.

A whole iteration (``BandGridIteration``) uses both partitions the
reference has, each where it needs no exchange: the CG band-parallel (the
reference's comm_band split; the CG is band by band, so a rank's bands need
nothing from the others), the Rayleigh-Ritz step grid-parallel (MB x MB
partial sums), with all-to-all moves of the bands between the two layouts
(``BandGridLayout``).
"""
from __future__ import annotations

import dataclasses
import types

import numpy as np

# One CholeskyQR pass is kept for the fused Rayleigh-Ritz step while
# (max diag R / min diag R)^2 <= this; above it a second pass runs first
# (the FP64 bound of the single-GPU step).
KAPPA_MAX = 1e3


def _split(n: int, nparts: int, what: str):
    if nparts < 1 or n < nparts:
        raise ValueError(f"cannot cut {n} {what} into {nparts} parts of at least one")
    counts = [n // nparts + (1 if p < n % nparts else 0) for p in range(nparts)]
    offsets = [sum(counts[:p]) for p in range(nparts)]
    return counts, offsets


def split_planes(n: int, nparts: int):
    """(counts, offsets) of n points cut into nparts parts
    (rgrid_sol_module.f90:84-108)."""
    return _split(n, nparts, "planes")


def split_bands(nb: int, nparts: int):
    """(counts, offsets) of nb bands over nparts ranks: band i counts for rank
    mod(i, np), each rank's bands contiguous in rank order
    (parallel_module.f90:366-377, the same rule as the grid split)."""
    return _split(nb, nparts, "bands")


@dataclasses.dataclass(frozen=True)
class HaloRun:
    """n consecutive halo planes of one rank's extended slab, from one peer."""

    peer: int  # rank that owns the planes
    src: int  # first plane, in the peer's own-plane numbering (0 .. nz(peer) - 1)
    dst: int  # first plane of the receiving extended slab (0 .. nz + 2 Md - 1)
    n: int


def halo_runs(n3: int, nranks: int, md: int, rank: int):
    """The halo planes of ``rank``'s extended slab as runs of planes owned by
    one peer, lower halo first (the planes bcset_3 fills, periodic in z)."""
    counts, offsets = split_planes(n3, nranks)
    z0, nz = offsets[rank], counts[rank]
    owner = np.repeat(np.arange(nranks), counts)
    runs = []
    for e in list(range(md)) + list(range(md + nz, 2 * md + nz)):
        g = (z0 - md + e) % n3
        p = int(owner[g])
        src = g - offsets[p]
        last = runs[-1] if runs else None
        if last and last.peer == p and last.src + last.n == src and last.dst + last.n == e:
            runs[-1] = HaloRun(p, last.src, last.dst, last.n + 1)
        else:
            runs.append(HaloRun(p, src, e, 1))
    return runs


class SlabDomain:
    """One rank's slab: plane split, halo maps and the restriction of the
    grid data (local potential, projector tables) to the extended slab."""

    def __init__(self, ngrid, md: int, rank: int, nranks: int):
        self.n1, self.n2, self.n3 = (int(v) for v in ngrid)
        self.md, self.rank, self.nranks = int(md), int(rank), int(nranks)
        self.counts, self.offsets = split_planes(self.n3, self.nranks)
        self.z0, self.nz = self.offsets[rank], self.counts[rank]
        self.n12 = self.n1 * self.n2
        self.planes = self.nz + 2 * self.md
        self.ml_ext = self.n12 * self.planes
        self.ml_own = self.n12 * self.nz
        self.row0 = self.n12 * self.md  # first own row of the extended slab
        self.recv = halo_runs(self.n3, nranks, md, rank)
        # what this rank sends: every peer's runs that it owns, in the peer's order
        self.send = [(q, r) for q in range(nranks) for r in halo_runs(self.n3, nranks, md, q) if r.peer == rank]

    # -------------------------------------------------------- index maps
    def global_planes(self) -> np.ndarray:
        """Global z plane of each plane of the extended slab."""
        return (self.z0 - self.md + np.arange(self.planes)) % self.n3

    def ext_from_global(self, a: np.ndarray) -> np.ndarray:
        """The extended slab's rows of a global (ML, ...) array, halo planes
        included (set-up and checks; the halo of the bands is exchanged)."""
        rows = (self.global_planes()[:, None] * self.n12 + np.arange(self.n12)[None, :]).reshape(-1)
        out = np.asarray(a)[rows]
        return out if out.ndim == 1 else np.asfortranarray(out)

    def own_slice(self) -> slice:
        return slice(self.row0, self.row0 + self.ml_own)

    def own(self, t):
        """The own rows of an extended-slab array (a view)."""
        return t[self.own_slice()]

    def restrict_projectors(self, lma_ptr, jjp, uv):
        """Projector tables over the own points, in extended-slab indices,
        every projector kept (those whose sphere misses the slab with no
        entries), so the partial sums of all ranks line up row by row."""
        lma_ptr = np.asarray(lma_ptr, dtype=np.int64)
        jjp = np.asarray(jjp, dtype=np.int64)
        nzlma = lma_ptr.shape[0] - 1
        lma_of = np.repeat(np.arange(nzlma), np.diff(lma_ptr))
        z = jjp // self.n12
        keep = (z >= self.z0) & (z < self.z0 + self.nz)
        cnt = np.bincount(lma_of[keep], minlength=nzlma)
        ptr = np.concatenate([[0], np.cumsum(cnt)]).astype(np.int32)
        local = (jjp[keep] - (self.z0 - self.md) * self.n12).astype(np.int32)
        return ptr, local, np.asarray(uv, dtype=np.float64)[keep]

    def slab_cell(self, cell):
        """The extended slab as a cell: grid (n1, n2, nz + 2 Md), the local
        potential on its planes and the projector entries of its own points."""
        ptr, jjp, uv = self.restrict_projectors(cell.lma_ptr, cell.jjp, cell.uv)
        ns = types.SimpleNamespace(
            name=f"{getattr(cell, 'name', 'cell')}[slab {self.rank}/{self.nranks}]",
            ngrid=(self.n1, self.n2, self.planes), md=self.md, h=np.asarray(cell.h), dV=float(cell.dV),
            coef_lap0=float(cell.coef_lap0), coef_lap=np.asarray(cell.coef_lap),
            vloc=self.ext_from_global(np.asarray(cell.vloc)), lma_ptr=ptr, jjp=jjp, uv=uv,
            iuv=np.asarray(cell.iuv, dtype=np.int32), amap=np.asarray(cell.amap, dtype=np.int32),
            duv=np.zeros((0, 3)), nzlma=int(cell.nzlma), natom=int(cell.natom), ML=self.ml_ext)
        return ns

    # ------------------------------------------------------ halo exchange
    def exchange(self, psi, dist=None) -> None:
        """Fill the halo planes of the extended-slab bands psi (ml_ext, nb),
        column-major with leading dimension ml_ext, from the ranks that own
        them (bcset_3_module.f90:15-151).  dist: torch.distributed (None for
        one rank)."""
        if psi.shape[0] != self.ml_ext or psi.stride(0) != 1 or psi.stride(1) != self.ml_ext:
            raise ValueError("exchange: psi must be a column-major (ml_ext, nb) extended-slab array")
        import torch

        nb = psi.shape[1]
        v = psi.t().view(nb, self.planes, self.n12)
        md = self.md
        # the rank's own planes that its own halo needs (one rank, or the
        # periodic wrap when a rank owns both sides)
        for r in self.recv:
            if r.peer == self.rank:
                v[:, r.dst:r.dst + r.n].copy_(v[:, md + r.src:md + r.src + r.n])
        peers_in = sorted({r.peer for r in self.recv if r.peer != self.rank})
        peers_out = sorted({q for q, _ in self.send if q != self.rank})
        if not peers_in and not peers_out:
            return
        if dist is None:
            raise ValueError("exchange: more than one rank needs a process group")
        ops, bufs = [], []
        for q in peers_out:
            parts = [v[:, md + r.src:md + r.src + r.n] for qq, r in self.send if qq == q]
            buf = torch.cat(parts, dim=1).contiguous()
            ops.append(dist.P2POp(dist.isend, buf, q))
        for p in peers_in:
            runs = [r for r in self.recv if r.peer == p]
            buf = torch.empty((nb, sum(r.n for r in runs), self.n12), dtype=psi.dtype, device=psi.device)
            bufs.append((runs, buf))
            ops.append(dist.P2POp(dist.irecv, buf, p))
        for req in dist.batch_isend_irecv(ops):
            req.wait()
        for runs, buf in bufs:
            k = 0
            for r in runs:
                v[:, r.dst:r.dst + r.n].copy_(buf[:, k:k + r.n])
                k += r.n


def _all_reduce(dist, t):
    """Sum t over the ranks in place (no process group: t as it is).  NCCL
    takes contiguous tensors only, so a column-major matrix is reduced
    through its storage (the row-major transpose view)."""
    if dist is None:
        return t
    if t.is_contiguous():
        dist.all_reduce(t)
    elif t.dim() == 2 and t.t().is_contiguous():
        dist.all_reduce(t.t())
    else:
        buf = t.contiguous()
        dist.all_reduce(buf)
        t.copy_(buf)
    return t


def _share_stream(gpu, device) -> None:
    """Bind the library to torch's current stream on ``device``: the layout
    moves and the collectives are torch work (NCCL waits on the current
    stream), so the library's kernels must be ordered on that stream too."""
    import torch

    gpu.set_stream(torch.cuda.current_stream(device).cuda_stream)


class GpuSlabBackend:
    """The per-slab compute on this rank's GPU through the library's entries:
    op_local on the own planes, projection partials and scatter, Gram sums,
    the small dense steps, own-row rotations."""

    def __init__(self, gpu, domain: SlabDomain, cell):
        import torch

        self.gpu, self.domain = gpu, domain
        self.device = torch.device("cuda", gpu.device)
        _share_stream(gpu, self.device)
        self.cell = domain.slab_cell(cell)
        gpu.setup(self.cell, with_forces=False)
        self.nzlma = self.cell.nzlma
        self.dV = self.cell.dV

    def empty(self, rows, cols):
        from . import api

        return api.fortran_empty(rows, cols, device=self.device)

    def zeros(self, rows, cols):
        t = self.empty(rows, cols)
        t.zero_()
        return t

    def op_local(self, psi, hpsi):
        self.gpu.op_local(1, psi, hpsi, z0=self.domain.md, nz=self.domain.nz)

    def project(self, psi, uvunk):
        self.gpu.op_nonlocal_project(psi, uvunk)

    def add(self, uvunk, hpsi):
        self.gpu.op_nonlocal_add(uvunk, hpsi)

    def gram(self, a, b, out, alpha, sym):
        self.gpu.gram(a, b, out, alpha=alpha, sym=sym)

    def overlap_cholesky(self, s, rinv) -> float:
        return self.gpu.overlap_cholesky(s, rinv)

    def rr_reduced(self, rinv, hsub, esp, w):
        self.gpu.rr_reduced(rinv, hsub, esp, w)

    def rotate(self, psi_own, w):
        self.gpu.rotate(psi_own, w)


class SlabSolver:
    """H psi, Gram sums and the Rayleigh-Ritz step of the bands of one slab,
    the ranks exchanging halos and partial sums over ``dist`` (None: one
    rank, which then is its own neighbour in z)."""

    def __init__(self, domain: SlabDomain, backend, dist=None):
        self.d, self.b, self.dist = domain, backend, dist
        if dist is None and domain.nranks != 1:
            raise ValueError("SlabSolver: more than one rank needs a process group")

    def _allreduce(self, t):
        return _all_reduce(self.dist, t)

    def empty_bands(self, nb):
        """Extended-slab bands (ml_ext, nb), column-major."""
        return self.b.empty(self.d.ml_ext, nb)

    def hamiltonian(self, psi, hpsi) -> None:
        """hpsi = H psi on the own rows (the halo rows of hpsi are not
        written); psi's halo planes are exchanged first."""
        self.d.exchange(psi, self.dist)
        self.b.op_local(psi, hpsi)
        if self.b.nzlma > 0:
            u = self.b.zeros(self.b.nzlma, psi.shape[1])
            self.b.project(psi, u)
            self._allreduce(u)
            self.b.add(u, hpsi)

    def gram(self, a, b, alpha=None, sym=0):
        """alpha a^T b over the whole grid (default alpha = dV): own-row
        partial sums, then the all-reduce."""
        d = self.d
        out = self.b.empty(a.shape[1], b.shape[1])
        self.b.gram(d.own(a), d.own(b), out, self.b.dV if alpha is None else alpha, sym)
        return self._allreduce(out)

    def rayleigh_ritz(self, psi, esp):
        """Gram-Schmidt followed by subspace_diag on the distributed bands
        (the pair calc_sweep calls, sweep_module.f90:152-155) as one
        Rayleigh-Ritz step: S = dV psi^T psi = R^T R, H = dV sym(psi^T H psi),
        R^-T H R^-1 = V diag(esp) V^T, psi <- psi R^-1 V on the own rows.
        A second CholeskyQR pass runs first when the overlap's Cholesky
        factor is spread beyond KAPPA_MAX.  Returns H psi's work array."""
        d, b = self.d, self.b
        nb = psi.shape[1]
        rinv = b.empty(nb, nb)
        kappa = b.overlap_cholesky(self.gram(psi, psi), rinv)
        if not kappa <= KAPPA_MAX:
            b.rotate(d.own(psi), rinv)
            kappa = b.overlap_cholesky(self.gram(psi, psi), rinv)
        hpsi = self.empty_bands(nb)
        self.hamiltonian(psi, hpsi)
        hsub = self.gram(psi, hpsi, sym=1)
        w = b.empty(nb, nb)
        b.rr_reduced(rinv, hsub, esp, w)
        b.rotate(d.own(psi), w)
        return hpsi


# ------------------------------------------------- band / grid layouts
class BandGridLayout:
    """One band set over N ranks in two layouts.

    band layout  rank r holds bands [b0(r), b0(r) + nb(r)) (split_bands) on
                 the whole grid, column-major (ML, nb(r));
    grid layout  rank r holds every band on its own planes [z0(r), z0(r) +
                 nz(r)) (split_planes), column-major (n1 n2 nz(r), nb).

    to_grid / to_band move the bands between them: rank r sends rank q the
    rows of q's planes of its own bands as one packed (nb(r), rows(q))
    message (an all-to-all: NCCL send/recv between GPUs, gloo on the host)."""

    def __init__(self, ngrid, nb: int, rank: int, nranks: int):
        self.n1, self.n2, self.n3 = (int(v) for v in ngrid)
        self.nb, self.rank, self.nranks = int(nb), int(rank), int(nranks)
        self.n12 = self.n1 * self.n2
        self.ml = self.n12 * self.n3
        self.pcounts, self.poffsets = split_planes(self.n3, self.nranks)
        self.bcounts, self.boffsets = split_bands(self.nb, self.nranks)
        self.rows = [(o * self.n12, (o + c) * self.n12) for c, o in zip(self.pcounts, self.poffsets)]
        self.b0, self.nb_own = self.boffsets[rank], self.bcounts[rank]
        self.ml_own = self.pcounts[rank] * self.n12

    @staticmethod
    def _rows_major(t, rows, cols, what):
        """The (cols, rows) row-major view of a column-major (rows, cols) array."""
        if tuple(t.shape) != (rows, cols) or (cols > 1 and t.stride(1) != rows) or t.stride(0) != 1:
            raise ValueError(f"{what} must be a column-major ({rows}, {cols}) array with leading dimension {rows}")
        return t.t()

    def _exchange(self, sends, recvs, dist):
        if not sends and not recvs:
            return
        if dist is None:
            raise ValueError("more than one rank needs a process group")
        ops = [dist.P2POp(dist.isend, buf, q) for q, buf in sends]
        ops += [dist.P2POp(dist.irecv, buf, q) for q, buf in recvs]
        for req in dist.batch_isend_irecv(ops):
            req.wait()

    def to_grid(self, band, grid, dist=None) -> None:
        """grid (ml_own, nb) <- the rank's planes of every band, from the band
        layouts of all ranks."""
        import torch

        bt = self._rows_major(band, self.ml, self.nb_own, "band-layout array")
        gt = self._rows_major(grid, self.ml_own, self.nb, "grid-layout array")
        r0, r1 = self.rows[self.rank]
        gt[self.b0:self.b0 + self.nb_own].copy_(bt[:, r0:r1])
        sends, recvs = [], []
        for q in range(self.nranks):
            if q == self.rank:
                continue
            q0, q1 = self.rows[q]
            sends.append((q, bt[:, q0:q1].contiguous()))
            recvs.append((q, torch.empty((self.bcounts[q], r1 - r0), dtype=band.dtype, device=band.device)))
        self._exchange(sends, recvs, dist)
        for q, buf in recvs:
            gt[self.boffsets[q]:self.boffsets[q] + self.bcounts[q]].copy_(buf)

    def to_band(self, grid, band, dist=None) -> None:
        """band (ML, nb_own) <- the rank's bands on the whole grid, from the
        grid layouts of all ranks."""
        import torch

        bt = self._rows_major(band, self.ml, self.nb_own, "band-layout array")
        gt = self._rows_major(grid, self.ml_own, self.nb, "grid-layout array")
        r0, r1 = self.rows[self.rank]
        bt[:, r0:r1].copy_(gt[self.b0:self.b0 + self.nb_own])
        sends, recvs = [], []
        for q in range(self.nranks):
            if q == self.rank:
                continue
            q0, q1 = self.rows[q]
            sends.append((q, gt[self.boffsets[q]:self.boffsets[q] + self.bcounts[q]].contiguous()))
            recvs.append((q, torch.empty((self.nb_own, q1 - q0), dtype=grid.dtype, device=grid.device)))
        self._exchange(sends, recvs, dist)
        for q, buf in recvs:
            q0, q1 = self.rows[q]
            bt[:, q0:q1].copy_(buf)


class GpuBandBackend:
    """The whole-grid compute of one rank on its GPU: the library set up on
    the full cell, CG and H psi on the rank's bands, Gram sums over any rows,
    the small dense steps, row-block rotations."""

    def __init__(self, gpu, cell):
        import torch

        self.gpu = gpu
        self.device = torch.device("cuda", gpu.device)
        _share_stream(gpu, self.device)
        gpu.setup(cell, with_forces=False)
        self.ml = int(cell.ML)
        self.dV = float(cell.dV)

    def empty(self, rows, cols):
        from . import api

        return api.fortran_empty(rows, cols, device=self.device)

    def vector(self, n):
        import torch

        return torch.zeros(n, dtype=torch.float64, device=self.device)

    def cg(self, psi, esp, res, ncg, mloop, mode):
        self.gpu.conjugate_gradient(1, self.ml, psi.shape[1], 1, 1, psi, esp, res, ncg=ncg, mloop=mloop, mode=mode)

    def hamiltonian(self, psi, hpsi):
        self.gpu.hamiltonian(1, 1, psi, hpsi, 1, self.ml, 1, psi.shape[1])

    def gram(self, a, b, out, alpha, sym):
        self.gpu.gram(a, b, out, alpha=alpha, sym=sym)

    def overlap_cholesky(self, s, rinv) -> float:
        return self.gpu.overlap_cholesky(s, rinv)

    def rr_reduced(self, rinv, hsub, esp, w):
        self.gpu.rr_reduced(rinv, hsub, esp, w)

    def rotate(self, psi, w):
        self.gpu.rotate(psi, w)


class BandGridIteration:
    """One eigensolver iteration as calc_sweep runs it (sweep_module.f90:
    150-155) over the ranks of ``layout``:

    1. conjugate_gradient on the rank's own bands on the whole grid (band
       parallel: cg_module.f90:97-430 treats each band alone at SWGS = 0),
       then H psi of those bands;
    2. psi and H psi moved to the grid layout;
    3. gram_schmidt + subspace_diag as one Rayleigh-Ritz step on the grid
       layout: S = dV psi^T psi and H = dV sym(psi^T H psi) summed over the
       ranks' planes (the MB x MB all-reduces of gram_schmidt_t_module.f90:
       194 and subspace_diag_la_module.f90:122), S = R^T R, R^-T H R^-1 =
       V diag(esp) V^T solved on every rank, the own rows rotated by R^-1 V
       (a second CholeskyQR pass first when diag(R) spreads beyond
       KAPPA_MAX, applied to H psi as well since H (psi R^-1) = (H psi) R^-1);
    4. the bands moved back to the band layout.

    esp (MB) ends up the Rayleigh-Ritz eigenvalues and res (MB) the CG
    residuals, on every rank."""

    def __init__(self, layout: BandGridLayout, backend, dist=None):
        self.L, self.b, self.dist = layout, backend, dist
        if dist is None and layout.nranks != 1:
            raise ValueError("BandGridIteration: more than one rank needs a process group")

    def _allreduce(self, t):
        return _all_reduce(self.dist, t)

    def _gram(self, a, c, sym):
        out = self.b.empty(self.L.nb, self.L.nb)
        self.b.gram(a, c, out, self.b.dV, sym)
        return self._allreduce(out)

    def iterate(self, psi, esp, res, ncg=4, mloop=3, mode=0) -> None:
        L, b = self.L, self.b
        e_own, r_own = b.vector(L.nb_own), b.vector(L.nb_own)
        b.cg(psi, e_own, r_own, ncg, mloop, mode)
        hpsi = b.empty(L.ml, L.nb_own)
        b.hamiltonian(psi, hpsi)
        gpsi, ghpsi = b.empty(L.ml_own, L.nb), b.empty(L.ml_own, L.nb)
        L.to_grid(psi, gpsi, self.dist)
        L.to_grid(hpsi, ghpsi, self.dist)
        del hpsi
        rinv = b.empty(L.nb, L.nb)
        kappa = b.overlap_cholesky(self._gram(gpsi, gpsi, 0), rinv)
        if not kappa <= KAPPA_MAX:
            b.rotate(gpsi, rinv)
            b.rotate(ghpsi, rinv)
            kappa = b.overlap_cholesky(self._gram(gpsi, gpsi, 0), rinv)
        hsub = self._gram(gpsi, ghpsi, 1)
        w = b.empty(L.nb, L.nb)
        b.rr_reduced(rinv, hsub, esp, w)
        b.rotate(gpsi, w)
        L.to_band(gpsi, psi, self.dist)
        full = b.vector(L.nb)
        full[L.b0:L.b0 + L.nb_own] = r_own
        res.copy_(self._allreduce(full))
