"""Oracle: CPU restatement of RSDFT's eigensolver inner loop (test infrastructure).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg import this module.  The product never does.

Point-wise and per-band loops (hpsi, preconditioner, CG, nonlocal force) live
in ``oracle.c`` (C + OpenMP, built by ``build()`` below).  The BLAS/LAPACK
level routines are restated here with numpy (``@`` = dgemm/dgemv) and
scipy.linalg.lapack (``dsyev``, ``dsyevd``, ``dsygv``), the same library calls
the reference makes:

* ``gram_schmidt_t``   gram_schmidt_t_module.f90:84-157 and the recursive
  ``gram_schmidt_sub`` :161-316, reproduced literally (one band rank);
* ``subspace_diag_la`` subspace_diag_la_module.f90:18-232 (hpsi per band,
  dsyr2k with alpha = dV/2, DSYEV('V','U'), rotation dgemm);
* ``subspace_mate_sl`` subspace_mate_sl_module.f90:27-366 and the recursive
  ``mate_sub`` :369-414 (lower triangle of dV psi^T H psi, 1x1 process grid);
* ``subspace_solv_sl`` subspace_solv_sl_module.f90:96 (pdsyevd('V','L') on a
  1x1 grid = dsyevd('V','L'));
* ``subspace_rotv_sl`` subspace_rotv_sl_module.f90:24-135 (psi <- psi V);
* ``dense_hamiltonian`` the explicit matrix of construct_hamiltonian_matrix
  (hamiltonian_matrix_module.f90:31-145), an independent check of hpsi;
* ``reference_duvdr`` the reference's tabulated, interpolated derivative
  table of the nonlocal force (calc_force_ps_nloc2, ps_nloc2_module.f90:
  1489-1586, on the radial tables of ps_nloc2_init_derivative,
  ps_nloc2_init_module.f90:219-301, polint_module.f90, ylm_module.f90), with
  ``gaunt_l1`` the coupling coefficients of get_gaunt_coefficient_L1
  (force_sub_sub_module.f90:64-387) computed from their definition.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np
import scipy.linalg.lapack as lapack

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
SRC = os.path.join(HERE, "oracle.c")

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def build(force: bool = False) -> str:
    """Compile oracle.c into liboracle.so (gcc, OpenMP, no fast-math)."""
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    cmd = ["gcc", "-O2", "-fopenmp", "-fno-fast-math", "-ffp-contract=off", "-shared", "-fPIC",
           "-o", LIB, SRC, "-lm"]
    subprocess.run(cmd, check=True)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB)
        L.oracle_set_hamiltonian.argtypes = [ctypes.c_int] * 4 + [ctypes.c_double, _dp, ctypes.c_double, _dp,
                                             ctypes.c_int, _ip, _ip, _dp, _ip] + [ctypes.c_double] * 4
        L.oracle_hamiltonian.argtypes = [_dp, _dp, ctypes.c_long, ctypes.c_int, _dp]
        L.oracle_dot.argtypes = [_dp, _dp, ctypes.c_long, ctypes.c_double]
        L.oracle_dot.restype = ctypes.c_double
        L.oracle_precond.argtypes = [_dp, _dp, ctypes.c_int, _dp]
        L.oracle_dsygv2.argtypes = [_dp, _dp, _dp]
        L.oracle_cg.argtypes = [_dp, ctypes.c_long, ctypes.c_int, _dp, _dp, ctypes.c_int, ctypes.c_int, _ip]
        L.oracle_force_nloc.argtypes = [_dp, ctypes.c_long, ctypes.c_int, _dp, _dp, _ip, ctypes.c_int, _dp]
        L.oracle_num_threads.restype = ctypes.c_int
        L.oracle_ylm.argtypes = [ctypes.c_double] * 3 + [ctypes.c_int, ctypes.c_int]
        L.oracle_ylm.restype = ctypes.c_double
        L.oracle_dviod.argtypes = [_dp, _dp, ctypes.c_int, ctypes.c_int, _dp]
        L.oracle_duvdr_ref.argtypes = [ctypes.c_int, _dp, ctypes.c_int, _dp, ctypes.c_int, _dp, _dp, _dp]
        _lib = L
    return _lib


def _p(a, t=_dp):
    return a.ctypes.data_as(t)


class Oracle:
    """Holds one cell's operator tables and exposes the restated routines."""

    def __init__(self, cell, spin_vloc=None):
        from rsdft_b200 import fd  # FD/preconditioner weights are set-up, shared with the product

        self.cell = cell
        self.ML = cell.ML
        self.dV = cell.dV
        self._keep = []
        coef = np.ascontiguousarray(cell.coef_lap, dtype=np.float64)
        vloc = np.ascontiguousarray(cell.vloc if spin_vloc is None else spin_vloc, dtype=np.float64)
        lma_ptr = np.ascontiguousarray(cell.lma_ptr, dtype=np.int32)
        jjp = np.ascontiguousarray(cell.jjp, dtype=np.int32)
        uv = np.ascontiguousarray(cell.uv, dtype=np.float64)
        iuv = np.ascontiguousarray(cell.iuv, dtype=np.int32)
        self._keep += [coef, vloc, lma_ptr, jjp, uv, iuv]
        c, c1, c2, c3 = fd.precond_coefficients(cell.h)
        n1, n2, n3 = cell.ngrid
        rc = lib().oracle_set_hamiltonian(n1, n2, n3, cell.md, cell.coef_lap0, _p(coef), cell.dV, _p(vloc),
                                          cell.nzlma, _p(lma_ptr, _ip), _p(jjp, _ip), _p(uv), _p(iuv, _ip),
                                          c, c1, c2, c3)
        if rc != 0:
            raise RuntimeError("oracle_set_hamiltonian failed")

    # ------------------------------------------------------------------ hpsi
    def hamiltonian(self, psi: np.ndarray, want_uvunk: bool = False):
        """H psi for psi of shape (ML, nb) (Fortran order) or (ML,)."""
        psi = np.asarray(psi, dtype=np.float64)
        one = psi.ndim == 1
        p = np.asfortranarray(psi.reshape(self.ML, -1))
        nb = p.shape[1]
        h = np.zeros_like(p, order="F")
        uvunk = np.zeros((self.cell.nzlma, nb), order="F") if want_uvunk else None
        lib().oracle_hamiltonian(_p(p), _p(h), self.ML, nb, _p(uvunk) if want_uvunk else None)
        h = h[:, 0] if one else h
        return (h, uvunk) if want_uvunk else h

    def dot(self, a, b):
        a = np.ascontiguousarray(a, dtype=np.float64)
        b = np.ascontiguousarray(b, dtype=np.float64)
        return lib().oracle_dot(_p(a), _p(b), a.size, self.dV)

    def precond(self, gk, mloop=3):
        gk = np.ascontiguousarray(gk, dtype=np.float64)
        pg = gk.copy()
        work = np.zeros(3 * self.ML)
        lib().oracle_precond(_p(gk), _p(pg), mloop, _p(work))
        return pg

    # --------------------------------------------------------------------- CG
    def conjugate_gradient(self, unk, ncg=4, mloop=3):
        """conjugate_gradient_1 on a copy of unk (ML, MB); returns (unk, esp, res, stats)."""
        u = np.array(unk, dtype=np.float64, order="F", copy=True)
        MB = u.shape[1]
        esp = np.zeros(MB)
        res = np.zeros(MB)
        stats = np.zeros(2, dtype=np.int32)
        rc = lib().oracle_cg(_p(u), self.ML, MB, _p(esp), _p(res), ncg, mloop, _p(stats, _ip))
        if rc != 0:
            raise RuntimeError(f"oracle_cg failed ({rc})")
        return u, esp, res, stats

    # ---------------------------------------------------------- Gram-Schmidt
    def gram_schmidt_t(self, unk, nblk=0, nblk1=4):
        u = np.array(unk, dtype=np.float64, order="F", copy=True)
        gram_schmidt_t(u, self.dV, nblk, nblk1)
        return u

    # ------------------------------------------------------------- subspace
    def subspace_diag_la(self, unk):
        u = np.array(unk, dtype=np.float64, order="F", copy=True)
        psit = self.hamiltonian(u)
        hsub = 0.5 * self.dV * (u.T @ psit + psit.T @ u)  # dsyr2k('U','T', alpha = dV/2)
        w, v, info = lapack.dsyev(np.triu(hsub), compute_v=1, lower=0)
        if info != 0:
            raise RuntimeError(f"dsyev info={info}")
        return np.asfortranarray(u @ v), w, v

    def subspace_mate_sl(self, unk, mblk=None):
        u = np.asarray(unk, dtype=np.float64, order="F")
        hpsi = self.hamiltonian(u)
        return subspace_mate(u, hpsi, self.dV, mblk)

    # ----------------------------------------------------------------- force
    def force_nloc_with(self, unk, occ, duv):
        """force_nloc with the derivative table ``duv`` (nnz, 3) in place of
        the cell's analytic one (e.g. ``reference_duvdr(cell)``)."""
        u = np.asfortranarray(unk, dtype=np.float64)
        occ = np.ascontiguousarray(occ, dtype=np.float64)
        d = np.ascontiguousarray(duv, dtype=np.float64)
        am = np.ascontiguousarray(self.cell.amap, dtype=np.int32)
        f = np.zeros((self.cell.natom, 3))
        lib().oracle_force_nloc(_p(u), self.ML, u.shape[1], _p(occ), _p(d), _p(am, _ip), self.cell.natom, _p(f))
        return f

    def force_nloc(self, unk, occ):
        c = self.cell
        u = np.asfortranarray(unk, dtype=np.float64)
        occ = np.ascontiguousarray(occ, dtype=np.float64)
        duv = np.ascontiguousarray(c.duv, dtype=np.float64)
        amap = np.ascontiguousarray(c.amap, dtype=np.int32)
        f = np.zeros((c.natom, 3))
        lib().oracle_force_nloc(_p(u), self.ML, u.shape[1], _p(occ), _p(duv), _p(amap, _ip), c.natom, _p(f))
        return f

    def energy(self, unk, occ):
        """E = sum_n f_n <psi_n|H|psi_n> dV."""
        u = np.asfortranarray(unk, dtype=np.float64)
        h = self.hamiltonian(u)
        return float(np.sum(occ * np.einsum("ij,ij->j", u, h)) * self.dV)

    def dense_hamiltonian(self):
        return dense_hamiltonian(self.cell)


# -------------------------------------------------------------------------
def dsygv2(A, B):
    """oracle.c's restatement of dsygv(1,'V','U',2): returns (W, vectors)."""
    a = np.array(A, dtype=np.float64, order="F", copy=True)
    b = np.array(B, dtype=np.float64, order="F", copy=True)
    w = np.zeros(2)
    info = lib().oracle_dsygv2(_p(a), _p(b), _p(w))
    if info != 0:
        raise RuntimeError(f"dsygv2 info={info}")
    return w, a


def _normalise(u, col, dV):
    c = float(np.sum(np.abs(u[:, col]) ** 2))
    c = 1.0 / np.sqrt(c * dV)
    u[:, col] *= c


def _gs_sub(u, mm1, mm2, nn1, nn2, mblk, dV, nblk1):
    """gram_schmidt_sub (gram_schmidt_t_module.f90:161-316), 1-based bounds."""
    for ms in range(mm1, mm2 + 1, mblk):
        me = min(ms + mblk - 1, mm2)
        mm = me - ms + 1
        for ns in range(nn1, nn2 + 1, mblk):
            ne = min(ns + mblk - 1, nn2)
            ne = min(ne, me - 1)
            nn = ne - ns + 1
            if nn <= 0:
                continue
            if ms >= ne + 1:
                utmp2 = (-dV) * (u[:, ns - 1:ne].T @ u[:, ms - 1:me])  # dgemm('T','N')
                u[:, ms - 1:me] += u[:, ns - 1:ne] @ utmp2           # dgemm('N','N')
                if ms == ne + 1:
                    _normalise(u, ms - 1, dV)
            elif mm <= nblk1:
                for m in range(ms, me + 1):
                    n = min(m - 1, ne)
                    if n - ns + 1 > 0:
                        utmp = (-dV) * (u[:, ns - 1:n].T @ u[:, m - 1])  # dgemv('T')
                        u[:, m - 1] += u[:, ns - 1:n] @ utmp               # dgemv('N')
                    if m == 1 or (n == m - 1 and m != ns):
                        _normalise(u, m - 1, dV)
            else:
                mblkh = max(mblk // 2, nblk1)
                _gs_sub(u, ms, me, ns, ne, mblkh, dV, nblk1)


def gram_schmidt_t(u, dV, nblk=0, nblk1=4):
    """gram_schmidt_t (gram_schmidt_t_module.f90:84-157), np_band = 1, in place."""
    MB = u.shape[1]
    if nblk == 0:
        nblk = MB
    if nblk1 == 0:
        nblk1 = 4
    ncycle = (MB - 1) // nblk + 1
    for k1 in range(1, ncycle + 1):
        ns = nblk * (k1 - 1) + 1
        ne = min(ns + nblk - 1, MB)
        _gs_sub(u, ns, ne, ns, ne, nblk, dV, nblk1)
        if ns <= MB - nblk:
            for ib in range(1, (ncycle - 1) + 2):
                nbss = ib
                if k1 + 1 <= nbss <= ncycle:
                    ms = nblk * (nbss - 1) + 1
                    me = min(ms + nblk - 1, MB)
                    if ms <= me:
                        _gs_sub(u, ms, me, ns, ne, nblk, dV, nblk1)
    return u


def _mate_sub(u, hpsi, vt, mm1, mm2, nn1, nn2, mblk, ns0, dV, nblk1=4):
    """mate_sub (subspace_mate_sl_module.f90:369-414); vt indexed by 1-based band."""
    for ns in range(nn1, nn2 + 1, mblk):
        ne = min(ns + mblk - 1, nn2)
        nn = ne - ns + 1
        if nn <= 0:
            continue
        for mms in range(mm1, mm2 + 1, mblk):
            ms = max(ns, mms)
            me = min(mms + mblk - 1, mm2)
            mm = me - ms + 1
            if mm <= 0:
                continue
            if ms >= ne:
                vt[ms - 1:me, ns - 1:ne] = dV * (u[:, ms - 1:me].T @ hpsi[:, ns - ns0:ne - ns0 + 1])
            elif mm <= nblk1:
                for n in range(ns, ne + 1):
                    vt[n - 1:ne, n - 1] = dV * (u[:, n - 1:ne].T @ hpsi[:, n - ns0])
            else:
                _mate_sub(u, hpsi, vt, ms, me, ns, ne, max(mblk // 2, nblk1), ns0, dV, nblk1)


def subspace_mate(u, hpsi, dV, mblk=None):
    """Lower triangle of dV psi^T (H psi) by the reference's block recursion.

    subspace_mate_sl (subspace_mate_sl_module.f90:71-366) on a 1x1 process
    grid: column blocks of MBLK, diagonal blocks through mate_sub, the blocks
    below them through one dgemm each.
    """
    MB = u.shape[1]
    if mblk is None:
        mblk = MB
    hsub = np.zeros((MB, MB))
    for ns in range(1, MB + 1, mblk):
        ne = min(ns + mblk - 1, MB)
        hp = hpsi[:, ns - 1:ne]
        for ms in range(ns, ne + 1, mblk):
            me = min(ms + mblk - 1, ne)
            _mate_sub(u, hp, hsub, ms, me, ns, ne, max(mblk // 2, 4), ns, dV)
        if ne + 1 <= MB:
            for ms in range(ne + 1, MB + 1, mblk):
                me = min(ms + mblk - 1, MB)
                hsub[ms - 1:me, ns - 1:ne] = dV * (u[:, ms - 1:me].T @ hp)
    return np.tril(hsub)


def subspace_solv(hsub_lower):
    """pdsyevd('V','L') on one process = dsyevd('V','L')."""
    w, v, info = lapack.dsyevd(hsub_lower, compute_v=1, lower=1)
    if info != 0:
        raise RuntimeError(f"dsyevd info={info}")
    return w, v


def subspace_rotv(u, vsub):
    return np.asfortranarray(u @ vsub)


def dense_hamiltonian(cell):
    """Explicit H (ML x ML) as construct_hamiltonian_matrix builds it."""
    n1, n2, n3 = cell.ngrid
    ML = cell.ML
    Hm = np.zeros((ML, ML))
    idx = np.arange(ML)
    i1, i2, i3 = idx % n1, (idx // n1) % n2, idx // (n1 * n2)
    Hm[idx, idx] += cell.coef_lap0 + cell.vloc
    for m in range(1, cell.md + 1):
        for sgn in (-1, 1):
            jx = (i1 + sgn * m) % n1 + n1 * (i2 + n2 * i3)
            jy = i1 + n1 * ((i2 + sgn * m) % n2 + n2 * i3)
            jz = i1 + n1 * (i2 + n2 * ((i3 + sgn * m) % n3))
            np.add.at(Hm, (idx, jx), cell.coef_lap[0, m - 1])
            np.add.at(Hm, (idx, jy), cell.coef_lap[1, m - 1])
            np.add.at(Hm, (idx, jz), cell.coef_lap[2, m - 1])
    for lma in range(cell.nzlma):
        s, e = cell.lma_ptr[lma], cell.lma_ptr[lma + 1]
        j = cell.jjp[s:e]
        v = cell.uv[s:e]
        Hm[np.ix_(j, j)] += cell.iuv[lma] * cell.dV * np.outer(v, v)
    return Hm


def vloc_adjoint(unk, occ, dV):
    """dE/dV(r) = sum_n f_n psi_n(r)^2 dV for E = sum f_n <psi|H|psi> dV."""
    return (np.asarray(unk) ** 2) @ np.asarray(occ) * dV


# ---------------------------------------------------------------------------
# Reference path of the nonlocal force's derivative table
RAD_DR = 2e-3  # radial grid of the synthetic projector tables (rad1)


def gaunt_l1(lmax: int):
    """G[k][L][m + lmax][L1][L1z + lmax + 1] = integral over the unit sphere
    of Ylm(L, m) * Ylm(1, q_k) * Ylm(L1, L1z), q = (1, -1, 0) for k = x, y,
    z, with the reference's real harmonics (ylm_module.f90): the tables Y1,
    Y2, Y3 of get_gaunt_coefficient_L1 (force_sub_sub_module.f90:64-387) for
    L <= lmax, L1 <= lmax + 1.  Gauss-Legendre in cos(theta) x uniform phi,
    exact for these polynomial degrees."""
    L = lib()
    mu, wmu = np.polynomial.legendre.leggauss(12)
    nphi = 24
    phi = 2.0 * np.pi * np.arange(nphi) / nphi
    pts = []
    for a, wa in zip(mu, wmu):
        st = np.sqrt(1.0 - a * a)
        for p in phi:
            pts.append((st * np.cos(p), st * np.sin(p), a, wa * 2.0 * np.pi / nphi))
    lm_all = [(l, m) for l in range(lmax + 3) for m in range(-l, l + 1)]
    Y = {lm: np.array([L.oracle_ylm(x, y, z, lm[0], lm[1]) for x, y, z, _ in pts]) for lm in lm_all}
    w = np.array([p[3] for p in pts])
    G = np.zeros((3, lmax + 1, 2 * lmax + 1, lmax + 2, 2 * lmax + 3))
    for k, q in enumerate((1, -1, 0)):
        for l in range(lmax + 1):
            for m in range(-l, l + 1):
                for l1 in range(lmax + 2):
                    for m1 in range(-l1, l1 + 1):
                        G[k, l, m + lmax, l1, m1 + lmax + 1] = np.sum(w * Y[(l, m)] * Y[(1, q)] * Y[(l1, m1)])
    return G


def reference_duvdr(cell):
    """duVdR (nnz, 3) of the cell's projectors by the reference's tabulated
    path, aligned with ``cell.jjp``: per atom and l the radial function
    viod(r) = sqrt(D) r^l exp(-r^2 / alpha) on rad1 = 0, dr, .., rc;
    ps_nloc2_init_derivative's dviod tables (dpolint derivatives); per
    periodic image of each sphere point the polint-interpolated
    dviod(r) / r^2 contracted with Ylm and the coupling coefficients
    (ps_nloc2_module.f90:1507-1586); images of one grid point summed, as
    the force's JJ_MAP loop does (:1634-1645)."""
    from rsdft_b200 import cell as C

    Lb = lib()
    n = cell.ngrid[0]
    h = cell.h
    nrc = int(round(C.PROJ_RC / RAD_DR)) + 1
    rad = np.ascontiguousarray(np.arange(nrc) * RAD_DR)
    G = gaunt_l1(1)
    kp = int(np.ceil(C.PROJ_RC / h.min())) + 1
    p1, p2, p3 = C._box_offsets(kp)
    out = np.zeros((int(cell.lma_ptr[-1]), 3))
    lma = 0
    for ia in range(cell.natom):
        R = cell.atoms[ia]
        c0 = np.floor(R / h).astype(int)
        u1, u2, u3 = c0[0] + p1, c0[1] + p2, c0[2] + p3
        d = np.stack([u1 * h[0] - R[0], u2 * h[1] - R[1], u3 * h[2] - R[2]], axis=1)
        r2 = np.einsum("ij,ij->i", d, d)
        sel = r2 <= C.PROJ_RC ** 2 + 1e-10
        d = np.ascontiguousarray(d[sel])
        idx = np.mod(u1[sel], n) + n * (np.mod(u2[sel], n) + n * np.mod(u3[sel], n))
        order = np.argsort(idx, kind="stable")
        _, start = np.unique(idx[order], return_index=True)
        for l in (0, 1):
            viod = np.ascontiguousarray(np.sqrt(cell.dvals[ia, l]) * rad ** l * np.exp(-rad ** 2 / C.PROJ_ALPHA))
            nj = 3 if l == 1 else 1
            dv = np.zeros(nj * nrc)
            if Lb.oracle_dviod(_p(rad), _p(viod), nrc, l, _p(dv)) != 0:
                raise RuntimeError("oracle_dviod failed")
            for m in (range(-1, 2) if l == 1 else (0,)):
                while not (cell.amap[lma] == ia and cell.lmap[lma] == l and cell.mmap[lma] == m):
                    raise RuntimeError(f"projector order differs at lma {lma}")
                g = np.ascontiguousarray(G[:, l, m + 1, : l + 2, 1 - l: 1 - l + 2 * l + 3])
                dd = np.zeros((len(d), 3))
                if Lb.oracle_duvdr_ref(l, _p(d), len(d), _p(rad), nrc, _p(dv), _p(g), _p(dd)) != 0:
                    raise RuntimeError("oracle_duvdr_ref: point below the radial grid")
                merged = np.add.reduceat(dd[order], start, axis=0)
                s0, e0 = cell.lma_ptr[lma], cell.lma_ptr[lma + 1]
                if e0 - s0 != len(merged):
                    raise RuntimeError(f"sphere of projector {lma} differs from the cell's")
                out[s0:e0] = merged
                lma += 1
    return out


# ---------------------------------------------------------------------------
# calc_sweep's scalar steps
def mp_ff0(n: int, x: np.ndarray) -> np.ndarray:
    """ff0 (fermi_mp_module.f90:287-306): Methfessel-Paxton occupation of
    order n (0.5 (1 - erf x) plus the Hermite series with factor(1) =
    -1/(4 sqrt(pi)), factor(i) = -factor(i-1)/(4 i), :147-153); erf is
    scipy's in place of the reference's bberf."""
    from scipy.special import erf

    x = np.asarray(x, dtype=np.float64)
    ff0 = 0.5 * (1.0 - erf(x))
    if n <= 0:
        return ff0
    fac = -1.0 / (4.0 * np.sqrt(np.pi))
    hp0 = np.ones_like(x)
    hp1 = 2.0 * x
    ff = fac * hp1
    for i in range(2, n + 1):
        fac = -fac / (4.0 * i)
        hp2 = 2.0 * x * hp1 - 2.0 * (2 * i - 3) * hp0
        hp3 = 2.0 * x * hp2 - 2.0 * (2 * i - 2) * hp1
        ff = ff + fac * hp3
        hp0, hp1 = hp2, hp3
    return ff0 + ff * np.exp(-x * x)


def calc_fermi(esp: np.ndarray, nelectron: float, ekbt: float = 1e-5, kinteg: int = 5, nfixed: int = 0,
               dspn: float = 0.0, it: int = 1):
    """calc_fermi (fermi_mp_module.f90:95-284) for one Gamma point (wbz = 1),
    all bands: esp (MB, MSP).  Bisection in the reference's loop order
    (sequential sums over s, n).  Returns (occ (MB, MSP), efermi)."""
    esp = np.asarray(esp, dtype=np.float64).reshape(esp.shape[0], -1)
    mb, msp = esp.shape
    occ = np.zeros_like(esp)

    def bisect(cols, zne, w):
        e = esp[:, cols]
        ef1, ef2 = e.min(), e.max()
        if ef1 == ef2:
            ef1, ef2 = ef1 - 0.01, ef2 + 0.01
        ef2 += min(ekbt * 1e2, 0.1)
        ef0, ef, octmp = 1e10, 0.0, 0.0
        for _ in range(1000):
            ef = 0.5 * (ef1 + ef2)
            if ef == ef0:
                return ef, True
            ff = mp_ff0(kinteg, (e - ef) / ekbt)
            occ[:, cols] = ff
            octmp = 0.0
            for s in range(e.shape[1]):
                for n in range(mb):
                    octmp = octmp + ff[n, s] * w
            if octmp - zne > 0.0:
                ef2 = ef
            elif octmp - zne < 0.0:
                ef1 = ef
            else:
                return ef, True
            ef0 = ef
        return ef, abs(octmp - zne) <= 1e-10

    if msp == 1 or it > nfixed:
        ef, ok = bisect(list(range(msp)), nelectron, 2.0 / msp)
    else:
        ok = True
        for s in range(msp):
            ef, o = bisect([s], 0.5 * nelectron + (1 - 2 * s) * 0.5 * dspn, 1.0)
            ok = ok and o
    if not ok:
        raise RuntimeError("EF IS NOT CONVERGED")
    return 2.0 * occ / msp, ef


def conv_check(esp, esp0, mb_ref: int, tol_esp: float):
    """conv_check_2 (sweep_module.f90:255-266): max |esp - esp0| over bands
    1..mb_ref of every spin, and whether it is below tol_esp."""
    d = np.abs(np.asarray(esp) - np.asarray(esp0)).reshape(len(esp0) if np.ndim(esp0) == 1 else esp0.shape[0], -1)
    m = float(d[:mb_ref].max())
    return m, m < tol_esp
