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
"""
from __future__ import annotations

import dataclasses
import types

import numpy as np

# One CholeskyQR pass is kept for the fused Rayleigh-Ritz step while
# (max diag R / min diag R)^2 <= this; above it a second pass runs first
# (the FP64 bound of the single-GPU step).
KAPPA_MAX = 1e3


def split_planes(n: int, nparts: int):
    """(counts, offsets) of n points cut into nparts parts
    (rgrid_sol_module.f90:84-108)."""
    if nparts < 1 or n < nparts:
        raise ValueError(f"cannot cut {n} planes into {nparts} slabs of at least one plane")
    counts = [n // nparts + (1 if p < n % nparts else 0) for p in range(nparts)]
    offsets = [sum(counts[:p]) for p in range(nparts)]
    return counts, offsets


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


class GpuSlabBackend:
    """The per-slab compute on this rank's GPU through the library's entries:
    op_local on the own planes, projection partials and scatter, Gram sums,
    the small dense steps, own-row rotations."""

    def __init__(self, gpu, domain: SlabDomain, cell):
        import torch

        self.gpu, self.domain = gpu, domain
        self.device = torch.device("cuda", gpu.device)
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
        if self.dist is not None:
            self.dist.all_reduce(t)
        return t

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
