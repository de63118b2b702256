"""Synthetic seeded silicon cells: grid, local potential, KB projectors, start bands.

This is the host-side set-up that produces the inputs of the eigensolver inner
loop.  In RSDFT the same inputs come from ``init_rgrid``/``init_kinetic``
(grid and FD weights), ``Vloc`` (localpot_module.f90:18-25), ``prep_ps_nloc2``
(ps_nloc2_module.f90:56-939: sphere point lists ``JJP``/``MJJ`` and the
projector values ``uV``), ``prep_uvk_ps_nloc2`` (:1128-1190: merging of
duplicate periodic images) and ``init_wf`` (random start bands).

Recipe (identical for every cell):

* diamond Si conventional cubic cell, a = 10.26 bohr, 8 atoms at the standard
  fractional sites, replicated ``ncell**3`` times, optional seeded Gaussian
  displacements;
* periodic grid with spacing h = a_super / N on each axis, point ``(i1,i2,i3)``
  at ``(i1*h, i2*h, i3*h)``, flat index ``i1 + N1*(i2 + N2*i3)`` (x fastest,
  kinetic_sol_module.f90:85);
* ``Vloc(r) = sum_atoms sum_images d_a exp(-(|r-R|/1.2)^2)`` (d_a ~ U[-2,-1] Ha,
  images within 8 bohr) plus 8 seeded low-k cosine modes scaled to a maximum
  of 1e-3 Ha;
* per atom l = 0 and l = 1 projectors (4 per atom), ``uV = sqrt(D_al) r^l
  exp(-r^2/0.8) Ylm(r_hat)`` on the grid points with ``r^2 <= rc^2 + 1e-10``
  (the inclusion test of ps_nloc2_module.f90:300), rc = 2.0 bohr, ``D_al ~
  U[0.5, 3]`` Ha folded in as ``sqrt(D)`` and ``iuV = sign(D) = +1`` (the KB
  normalisation of ps_read_psv.f90:239-240,275-279);
* real spherical harmonics in the convention of ``Ylm`` (ylm_module.f90:10-72):
  ``Y00 = 1/sqrt(4 pi)``, ``r Y1,-1 = -c y``, ``r Y1,0 = c z``, ``r Y1,1 = -c x``
  with ``c = sqrt(3/(4 pi))``;
* start bands uniform in [-0.5, 0.5].

All random numbers come from SplitMix64 streams so the same cell is produced
on every machine.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from . import fd

A_SI = 10.26
DIAMOND_FRAC = np.array(
    [
        [0.0, 0.0, 0.0],
        [0.0, 0.5, 0.5],
        [0.5, 0.0, 0.5],
        [0.5, 0.5, 0.0],
        [0.25, 0.25, 0.25],
        [0.25, 0.75, 0.75],
        [0.75, 0.25, 0.75],
        [0.75, 0.75, 0.25],
    ]
)
GAUSS_WIDTH = 1.2
VLOC_CUTOFF = 8.0
PROJ_ALPHA = 0.8
PROJ_RC = 2.0
C_Y1 = math.sqrt(3.0 / (4.0 * math.pi))
C_Y0 = 1.0 / math.sqrt(4.0 * math.pi)

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed: int, n: int, offset: int = 0) -> np.ndarray:
    """``n`` consecutive SplitMix64 outputs of stream ``seed`` starting at ``offset``."""
    with np.errstate(over="ignore"):
        idx = np.arange(offset + 1, offset + n + 1, dtype=np.uint64)
        z = np.uint64(seed & 0xFFFFFFFFFFFFFFFF) + idx * _GOLDEN
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        z = z ^ (z >> np.uint64(31))
    return z


def uniform(seed: int, n: int, lo=0.0, hi=1.0, offset: int = 0) -> np.ndarray:
    u = (splitmix64(seed, n, offset) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    return lo + (hi - lo) * u


def normal(seed: int, n: int, sigma=1.0) -> np.ndarray:
    """Box-Muller normals from one SplitMix64 stream."""
    u = uniform(seed, 2 * n)
    u1 = 1.0 - u[0::2]  # (0, 1]
    u2 = u[1::2]
    return sigma * np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * math.pi * u2)


def substream(seed: int, tag: int) -> int:
    """Independent stream id for quantity ``tag`` of cell ``seed``."""
    return int(splitmix64(seed * 1000003 + tag, 1)[0])


@dataclasses.dataclass
class Workload:
    name: str
    ncell: int
    ngrid: int
    nband: int
    nocc: int
    disp_sigma: float
    seed: int
    md: int = 6


WORKLOADS = {
    # 8-atom cell, 24^3, 32 bands: hpsi, one CG sweep, GS, subspace.
    "si8": Workload("si8", 1, 24, 32, 16, 0.0, 1001),
    # 64-atom cell, 48^3, 160 bands, displacements N(0, 0.02).
    "si64": Workload("si64", 2, 48, 160, 128, 0.02, 1002),
    # 216-atom cell, 72^3, 480 bands (432 occupied), displacements N(0, 0.02).
    "si216": Workload("si216", 3, 72, 480, 432, 0.02, 1003),
    # 64-atom cell for the force/adjoint checks, displacements N(0, 0.05).
    "si64_adjoint": Workload("si64_adjoint", 2, 48, 160, 128, 0.05, 1004),
    # 512-atom cell, 96^3, 1088 bands (1024 occupied).
    "si512": Workload("si512", 4, 96, 1088, 1024, 0.02, 1005),
    # small cells for dense-matrix and finite-difference checks
    "si8_g12": Workload("si8_g12", 1, 12, 16, 8, 0.03, 1006),
    "si8_g16": Workload("si8_g16", 1, 16, 24, 12, 0.03, 1007),
    # ML = 18^3 = 5832 (a multiple of 8, not of 32) and 36 bands (not a
    # multiple of 8): the general-shape paths of the mixed contractions
    "si8_g18": Workload("si8_g18", 1, 18, 36, 16, 0.03, 1008),
}


@dataclasses.dataclass
class Cell:
    """Everything the hot path reads, in the reference's layout (0-based)."""

    name: str
    ngrid: tuple
    a: float
    h: np.ndarray  # (3,)
    dV: float
    md: int
    coef_lap0: float
    coef_lap: np.ndarray  # (3, Md)
    atoms: np.ndarray  # (Natom, 3) cartesian bohr
    depth: np.ndarray  # (Natom,)
    dvals: np.ndarray  # (Natom, 2) D for l=0, 1
    vloc: np.ndarray  # (ML,)
    # nonlocal projectors in CSR by projector lma
    lma_ptr: np.ndarray  # int32 (nzlma+1,)
    jjp: np.ndarray  # int32 (nnz,) grid index, sorted ascending per lma
    uv: np.ndarray  # float64 (nnz,)
    duv: np.ndarray  # float64 (nnz, 3) dUV/dR_atom (analytic)
    iuv: np.ndarray  # int32 (nzlma,) = +-1
    amap: np.ndarray  # int32 (nzlma,) atom of lma
    lmap: np.ndarray  # int32 (nzlma,)
    mmap: np.ndarray  # int32 (nzlma,)
    nband: int
    nocc: int
    seed: int

    @property
    def ML(self) -> int:
        return int(self.ngrid[0] * self.ngrid[1] * self.ngrid[2])

    @property
    def nzlma(self) -> int:
        return int(self.iuv.shape[0])

    @property
    def natom(self) -> int:
        return int(self.atoms.shape[0])

    def occupations(self) -> np.ndarray:
        occ = np.zeros(self.nband)
        occ[: self.nocc] = 2.0
        return occ

    def psi0(self, nband: int | None = None) -> np.ndarray:
        """Start bands, uniform in [-0.5, 0.5], Fortran order ``(ML, MB)``."""
        nb = self.nband if nband is None else nband
        flat = uniform(substream(self.seed, 7), self.ML * nb, -0.5, 0.5)
        return flat.reshape((nb, self.ML)).T  # column-major view: column n contiguous

    def grid_coords(self) -> np.ndarray:
        n1, n2, n3 = self.ngrid
        i = np.arange(self.ML)
        i1 = i % n1
        i2 = (i // n1) % n2
        i3 = i // (n1 * n2)
        return np.stack([i1 * self.h[0], i2 * self.h[1], i3 * self.h[2]], axis=1)


def _box_offsets(k: int):
    r = np.arange(-k, k + 1)
    o1, o2, o3 = np.meshgrid(r, r, r, indexing="ij")
    return o1.ravel(), o2.ravel(), o3.ravel()


def _atoms(w: Workload) -> np.ndarray:
    a = A_SI
    frac = []
    for c3 in range(w.ncell):
        for c2 in range(w.ncell):
            for c1 in range(w.ncell):
                frac.append(DIAMOND_FRAC + np.array([c1, c2, c3], dtype=float))
    pos = np.concatenate(frac, axis=0) * a
    if w.disp_sigma > 0.0:
        pos = pos + normal(substream(w.seed, 1), pos.size, w.disp_sigma).reshape(pos.shape)
    return pos


def build_cell(name_or_workload, *, with_duv: bool = True) -> Cell:
    w = WORKLOADS[name_or_workload] if isinstance(name_or_workload, str) else name_or_workload
    a_sup = A_SI * w.ncell
    n = w.ngrid
    ngrid = (n, n, n)
    h = np.array([a_sup / n] * 3)
    dV = float(h[0] * h[1] * h[2])
    coef_lap0, coef_lap = fd.kinetic_coefficients(w.md, h)
    atoms = _atoms(w)
    natom = atoms.shape[0]
    depth = uniform(substream(w.seed, 2), natom, -2.0, -1.0)
    dvals = uniform(substream(w.seed, 3), natom * 2, 0.5, 3.0).reshape(natom, 2)
    ML = n * n * n

    # ---- local potential: Gaussian wells over periodic images + smooth noise
    vloc = np.zeros(ML)
    k = int(math.ceil(VLOC_CUTOFF / h.min()))
    o1, o2, o3 = _box_offsets(k)
    for ia in range(natom):
        R = atoms[ia]
        c = np.floor(R / h).astype(int)
        u1, u2, u3 = c[0] + o1, c[1] + o2, c[2] + o3
        d = np.stack([u1 * h[0] - R[0], u2 * h[1] - R[1], u3 * h[2] - R[2]], axis=1)
        r2 = np.einsum("ij,ij->i", d, d)
        sel = r2 <= VLOC_CUTOFF ** 2
        idx = np.mod(u1[sel], n) + n * (np.mod(u2[sel], n) + n * np.mod(u3[sel], n))
        vloc += np.bincount(idx, weights=depth[ia] * np.exp(-r2[sel] / GAUSS_WIDTH ** 2), minlength=ML)
    # noise: 8 low-k cosine modes with integer wave vectors in [-2, 2]
    ns = substream(w.seed, 4)
    kv = (np.floor(uniform(ns, 24) * 5.0) - 2.0).reshape(8, 3)
    ph = uniform(ns, 8, 0.0, 2.0 * math.pi, offset=24)
    amp = uniform(ns, 8, 0.5, 1.0, offset=32)
    i = np.arange(ML)
    frac = np.stack([(i % n) / n, ((i // n) % n) / n, (i // (n * n)) / n], axis=1)
    noise = np.zeros(ML)
    for m in range(8):
        noise += amp[m] * np.cos(2.0 * math.pi * (frac @ kv[m]) + ph[m])
    noise *= 1e-3 / np.abs(noise).max()
    vloc += noise

    # ---- nonlocal projectors
    kp = int(math.ceil(PROJ_RC / h.min())) + 1
    p1, p2, p3 = _box_offsets(kp)
    lma_ptr = [0]
    jjp_l, uv_l, duv_l, iuv_l, amap_l, lmap_l, mmap_l = [], [], [], [], [], [], []
    for ia in range(natom):
        R = atoms[ia]
        c = np.floor(R / h).astype(int)
        u1, u2, u3 = c[0] + p1, c[1] + p2, c[2] + p3
        d = np.stack([u1 * h[0] - R[0], u2 * h[1] - R[1], u3 * h[2] - R[2]], axis=1)
        r2 = np.einsum("ij,ij->i", d, d)
        sel = r2 <= PROJ_RC ** 2 + 1e-10
        d = d[sel]
        r2 = r2[sel]
        idx = np.mod(u1[sel], n) + n * (np.mod(u2[sel], n) + n * np.mod(u3[sel], n))
        g = np.exp(-r2 / PROJ_ALPHA)
        x, y, z = d[:, 0], d[:, 1], d[:, 2]
        s0 = math.sqrt(dvals[ia, 0])
        s1 = math.sqrt(dvals[ia, 1])
        # (value, d/dR) per projector; d/dR_atom = -grad_r
        t = 2.0 / PROJ_ALPHA
        val0 = s0 * C_Y0 * g
        dR0 = (s0 * C_Y0 * t * g)[:, None] * d
        comps = []
        comps.append((0, 0, val0, dR0))
        for m, (sign, axis) in zip((-1, 0, 1), ((-1.0, 1), (1.0, 2), (-1.0, 0))):
            xk = d[:, axis]
            val = s1 * sign * C_Y1 * xk * g
            grad = (-t * xk * g)[:, None] * d
            grad[:, axis] += g
            dR = -(s1 * sign * C_Y1) * grad
            comps.append((1, m, val, dR))
        order = np.argsort(idx, kind="stable")
        idx_s = idx[order]
        uniq, start = np.unique(idx_s, return_index=True)
        for (l, m, val, dR) in comps:
            # merge duplicate periodic images of one point (prep_uvk_ps_nloc2)
            v = np.add.reduceat(val[order], start) if len(order) else val
            dd = np.add.reduceat(dR[order], start, axis=0) if len(order) else dR
            jjp_l.append(uniq.astype(np.int32))
            uv_l.append(v)
            duv_l.append(dd)
            iuv_l.append(1)
            amap_l.append(ia)
            lmap_l.append(l)
            mmap_l.append(m)
            lma_ptr.append(lma_ptr[-1] + len(uniq))
    cell = Cell(
        name=w.name,
        ngrid=ngrid,
        a=a_sup,
        h=h,
        dV=dV,
        md=w.md,
        coef_lap0=float(coef_lap0),
        coef_lap=coef_lap,
        atoms=atoms,
        depth=depth,
        dvals=dvals,
        vloc=vloc,
        lma_ptr=np.asarray(lma_ptr, dtype=np.int32),
        jjp=np.concatenate(jjp_l).astype(np.int32),
        uv=np.concatenate(uv_l),
        duv=np.concatenate(duv_l, axis=0) if with_duv else np.zeros((0, 3)),
        iuv=np.asarray(iuv_l, dtype=np.int32),
        amap=np.asarray(amap_l, dtype=np.int32),
        lmap=np.asarray(lmap_l, dtype=np.int32),
        mmap=np.asarray(mmap_l, dtype=np.int32),
        nband=w.nband,
        nocc=w.nocc,
        seed=w.seed,
    )
    return cell


def projector_values(cell: Cell, atoms: np.ndarray):
    """Recompute ``uV`` on the fixed point lists of ``cell`` for moved ``atoms``.

    Used by finite-difference checks: the support (which grid points belong to
    each sphere) is held fixed, the projector values follow the atoms.  Points
    are matched to the nearest periodic image of the displaced atom.
    """
    n1, n2, n3 = cell.ngrid
    out = np.empty_like(cell.uv)
    L = np.array([cell.a, cell.a, cell.a])
    for lma in range(cell.nzlma):
        s, e = cell.lma_ptr[lma], cell.lma_ptr[lma + 1]
        ia = cell.amap[lma]
        j = cell.jjp[s:e].astype(np.int64)
        pos = np.stack([(j % n1) * cell.h[0], ((j // n1) % n2) * cell.h[1], (j // (n1 * n2)) * cell.h[2]], axis=1)
        d = pos - atoms[ia]
        d -= L * np.round(d / L)
        r2 = np.einsum("ij,ij->i", d, d)
        g = np.exp(-r2 / PROJ_ALPHA)
        l, m = cell.lmap[lma], cell.mmap[lma]
        if l == 0:
            out[s:e] = math.sqrt(cell.dvals[ia, 0]) * C_Y0 * g
        else:
            sign, axis = {-1: (-1.0, 1), 0: (1.0, 2), 1: (-1.0, 0)}[int(m)]
            out[s:e] = math.sqrt(cell.dvals[ia, 1]) * sign * C_Y1 * d[:, axis] * g
    return out
