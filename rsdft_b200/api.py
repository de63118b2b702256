"""Host-side mirror of RSDFT's eigensolver call surfaces on the B200 library.

Method names, argument order and meaning follow the Fortran routines they
replace (j-iwata/RSDFT v1.3.0, src/):

====================================  ==========================================
``RsdftGpu`` method                   reference routine
====================================  ==========================================
``hamiltonian(k,s,tpsi,htpsi,...)``   hamiltonian_module.f90:20
``conjugate_gradient(n1,n2,MB,...)``  cg_module.f90:54
``gram_schmidt(n0,n1,k,s,unk)``       gram_schmidt_module.f90:28 -> gram_schmidt_t
``subspace_diag(k,s,unk,esp)``        subspace_diag_module.f90:17 -> subspace_diag_la
``subspace_mate_sl(k,s,unk,hsub)``    subspace_mate_sl_module.f90:27
``subspace_solv_sl(hsub,esp,vsub)``   subspace_solv_sl_module.f90:15
``subspace_rotv_sl(k,s,unk,vsub)``    subspace_rotv_sl_module.f90:24
``calc_force_ps_nloc2(MI,force2,..)`` ps_nloc2_module.f90:1281
``hpsi_adjoint(psi, ...)``            (adjoint of op_localpot + op_ps_nloc2_hp)
``calc_density(unk, occ, rho)``      density_module.f90:115 (calc_density, NCPP)
``calc_sweep(unk, esp, res, occ,..)``  sweep_module.f90:60 (calc_sweep's loop)
``write_wf(path, unk, ngrid, ...)``   io_write_module.f90:19 (simple_wf_io_write)
``read_wf(path, unk, ngrid, ...)``    io_read_module.f90:15 (simple_wf_io_read)
``write_vrho(path, ngrid, ...)``      io_module.f90:97 (write_data, density/potentials)
``read_vrho(path, ngrid, ...)``       io_module.f90:283 (read_data, VRHO branch)
====================================  ==========================================

The reference routines read module state (``unk``, ``Vloc``, the projector
tables, ``occ``); here that state is set once with ``setup(cell)`` and the
arrays are passed explicitly.  Wavefunction arrays are Fortran-ordered
``(ML, nb)`` float64: numpy arrays (host) or torch tensors (device or host)
with strides ``(1, ML)`` (``fortran_empty`` makes one).  Every call raises
``RsdftError`` on a non-zero status; nothing falls back to the CPU.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _lib
from ._lib import RsdftError  # noqa: F401  (re-export)

MODE_FP64 = 0
MODE_MIXED_BF16X3 = 1  # 3-term split-BF16 contractions (6 products)
MODE_MIXED_TF32 = 2    # 2-term split-TF32 contractions (3 products)
MODE_MIXED_BF16X2 = 3  # 2-term split-BF16 contractions (3 products)


def _is_torch(a) -> bool:
    return type(a).__module__.startswith("torch")


def _ptr(a, *, name="array", shape=None, dtype="float64"):
    """Address of a numpy array or torch tensor, checking dtype and layout."""
    if a is None:
        return None
    if _is_torch(a):
        import torch

        want = {"float64": torch.float64, "int32": torch.int32}[dtype]
        if a.dtype != want:
            raise TypeError(f"{name}: dtype {a.dtype}, expected {want}")
        if a.dim() == 2:
            if not (a.stride(0) == 1 and a.stride(1) >= a.shape[0]):
                raise ValueError(f"{name}: torch tensor must be Fortran-ordered (ML, nb)")
        elif not a.is_contiguous():
            raise ValueError(f"{name}: tensor must be contiguous")
        return a.data_ptr()
    if not isinstance(a, np.ndarray):
        raise TypeError(f"{name}: expected numpy array or torch tensor, got {type(a)}")
    if a.dtype != np.dtype(dtype):
        raise TypeError(f"{name}: dtype {a.dtype}, expected {dtype}")
    if not a.flags.f_contiguous:
        raise ValueError(f"{name}: array must be Fortran-contiguous")
    return a.ctypes.data


def fortran_empty(ml: int, nb: int, device="cuda", dtype=None):
    """torch tensor of shape (ml, nb) with column-major strides."""
    import torch

    return torch.empty((nb, ml), dtype=dtype or torch.float64, device=device).t()


def fortran_copy(t):
    """A new (ML, nb) column-major tensor holding the values of the
    column-major tensor t.  (t.t().contiguous().t() is not a copy: t.t() is
    already contiguous, so it returns t's own storage.)"""
    return t.t().clone().t()


def _ld(a) -> int:
    if _is_torch(a):
        return int(a.stride(1)) if a.dim() == 2 else int(a.shape[0])
    return int(a.strides[1] // a.itemsize) if a.ndim == 2 else int(a.shape[0])


HEADER_FIELDS = ("ML", "ML1", "ML2", "ML3", "MB", "MB1", "MB2", "MK", "MS", "MMBZ", "IO_ctrl", "OC", "TYPE_WF")


def _wf_dims(unk, mk, ms):
    """(ld, mb, mk, ms) of a Fortran-ordered unk(ML, MB) or unk(ML, MB, MK, MS)."""
    if unk.ndim == 4:
        return int(unk.shape[0]), int(unk.shape[1]), int(unk.shape[2]), int(unk.shape[3])
    if unk.ndim == 2:
        nb = int(unk.shape[1])
        if nb % (mk * ms) != 0:
            raise ValueError(f"unk has {nb} columns, not a multiple of mk * ms = {mk * ms}")
        return _ld(unk), nb // (mk * ms), mk, ms
    raise ValueError("unk must be (ML, MB) or (ML, MB, MK, MS)")


def _f64(a, shape, name):
    if a is None:
        return None
    a = np.asfortranarray(a, dtype=np.float64)
    if a.size != int(np.prod(shape)):
        raise ValueError(f"{name}: {a.size} values, expected {shape}")
    return a


def write_wf(path, unk, ngrid, *, mk=1, ms=1, mbwr1=1, mbwr2=None, oc=0, io_ctrl=0, occ=None, aa=None, bb=None,
             kbb=None) -> None:
    """simple_wf_io_write (io_write_module.f90:19-264) for one process.

    unk is Fortran-ordered (ML, MB) -- columns band-major over (k, spin) when
    mk * ms > 1 -- or (ML, MB, MK, MS); a host array, a registered one, or a
    device tensor.  oc = 4 or 5 writes FP32 bands, oc >= 10 the old format;
    io_ctrl 3 writes the bands to path + ".00000".  Needs no device for host
    arrays."""
    ld, mb, mk, ms = _wf_dims(unk, mk, ms)
    ng = np.ascontiguousarray(ngrid, dtype=np.int32)
    occ = _f64(occ, (mb, mk, ms), "occ")
    aa = _f64(aa, (3, 3), "aa")
    bb = _f64(bb, (3, 3), "bb")
    kbb = None if kbb is None else np.asfortranarray(np.asarray(kbb, dtype=np.float64).reshape(3, -1))
    mmbz = 0 if kbb is None else kbb.shape[1]
    _lib.call("rsdft_gpu_write_wf", os.fsencode(path), _ptr(unk, name="unk"), ld, mb, mk, ms, mbwr1,
              mb if mbwr2 is None else mbwr2, oc, io_ctrl, ng.ctypes.data,
              None if occ is None else occ.ctypes.data, None if aa is None else aa.ctypes.data,
              None if bb is None else bb.ctypes.data, mmbz, None if kbb is None else kbb.ctypes.data)


def read_wf(path, unk, ngrid, *, mk=1, ms=1, io_ctrl=0, occ=None) -> dict:
    """simple_wf_io_read (io_read_module.f90:15-521) for one process: fills
    unk (as for write_wf) and occ(MB, MK, MS) if given; returns the file's
    header fields."""
    ld, mb, mk, ms = _wf_dims(unk, mk, ms)
    ng = np.ascontiguousarray(ngrid, dtype=np.int32)
    if occ is not None and (not isinstance(occ, np.ndarray) or occ.dtype != np.float64 or not occ.flags.f_contiguous
                            or occ.size != mb * mk * ms):
        raise ValueError("occ must be a Fortran-ordered float64 array of MB * MK * MS values")
    info = np.zeros(13, dtype=np.int32)
    _lib.call("rsdft_gpu_read_wf", os.fsencode(path), _ptr(unk, name="unk"), ld, mb, mk, ms, io_ctrl, ng.ctypes.data,
              None if occ is None else occ.ctypes.data, info.ctypes.data)
    return dict(zip(HEADER_FIELDS, (int(v) for v in info)))


def _field(a, n, name):
    """Address of an ML * nspin field stored without gaps (host or device)."""
    if a is None:
        return None
    size = a.numel() if _is_torch(a) else a.size
    if size != n:
        raise ValueError(f"{name}: {size} values, expected {n}")
    if _is_torch(a) and a.dim() == 2 and a.shape[1] > 1 and a.stride(1) != a.shape[0]:
        raise ValueError(f"{name}: columns must be stored without gaps")
    return _ptr(a, name=name)


def write_vrho(path, ngrid, rho, vloc, vh, vxc, *, aa=None, aa_atom=None, ki_atom=None, zn_atom=None,
               efermi=0.0) -> None:
    """The density/potential branch of write_data (io_module.f90:97-226) for
    one process.  rho, vloc, vxc are (ML, nspin) Fortran-ordered (or (ML,) for
    one spin), vh is (ML,); each a host array, a registered one or a device
    tensor.  aa(3, 3) is the lattice, aa_atom(3, Natom) the fractional atom
    positions, ki_atom(Natom) the element index of each atom (1-based, as in
    the reference) and zn_atom(Nelement) the atomic numbers."""
    ng = np.ascontiguousarray(ngrid, dtype=np.int32)
    ml = int(np.prod(ng))
    nspin = (rho.numel() if _is_torch(rho) else rho.size) // ml
    aa = np.zeros((3, 3), order="F") if aa is None else _f64(aa, (3, 3), "aa")
    aa_atom = np.zeros((3, 0), order="F") if aa_atom is None else np.asfortranarray(
        np.asarray(aa_atom, dtype=np.float64).reshape(3, -1, order="F"))
    natom = aa_atom.shape[1]
    ki_atom = np.ones(natom, dtype=np.int32) if ki_atom is None else np.ascontiguousarray(ki_atom, dtype=np.int32)
    zn_atom = np.zeros(0, dtype=np.int32) if zn_atom is None else np.ascontiguousarray(zn_atom, dtype=np.int32)
    if ki_atom.size != natom:
        raise ValueError(f"ki_atom: {ki_atom.size} values for {natom} atoms")
    _lib.call("rsdft_gpu_write_vrho", os.fsencode(path), ng.ctypes.data, aa.ctypes.data, zn_atom.size, natom,
              aa_atom.ctypes.data, ki_atom.ctypes.data, zn_atom.ctypes.data, float(efermi), nspin,
              _field(rho, ml * nspin, "rho"), _field(vloc, ml * nspin, "vloc"), _field(vh, ml, "vh"),
              _field(vxc, ml * nspin, "vxc"))


def read_vrho(path, ngrid, *, rho=None, vloc=None, vh=None, vxc=None, nspin=1):
    """The VRHO branch of read_data (io_module.f90:283-432) for one process:
    fills the fields given (shapes as for write_vrho) by the file's LL2 map;
    returns the file's Fermi energy (None for an unversioned file, which
    holds none)."""
    ng = np.ascontiguousarray(ngrid, dtype=np.int32)
    ml = int(np.prod(ng))
    ef = ctypes.c_double(np.nan)
    _lib.call("rsdft_gpu_read_vrho", os.fsencode(path), ng.ctypes.data, nspin, _field(rho, ml * nspin, "rho"),
              _field(vloc, ml * nspin, "vloc"), _field(vh, ml, "vh"), _field(vxc, ml * nspin, "vxc"),
              ctypes.addressof(ef))
    return None if np.isnan(ef.value) else ef.value


class RsdftGpu:
    """One device context of the B200 eigensolver library."""

    def __init__(self, device: int = 0):
        _lib.call("rsdft_gpu_init", device)
        self.device = device
        self.cell = None
        self._keep = []

    # ----------------------------------------------------------- set-up
    def setup(self, cell, *, with_forces: bool = True) -> None:
        """Upload grid, FD weights, Vloc and the projector tables of ``cell``."""
        ng = np.asarray(cell.ngrid, dtype=np.int32)
        coef = np.asfortranarray(np.ascontiguousarray(cell.coef_lap).ravel(), dtype=np.float64)
        h = np.asarray(cell.h, dtype=np.float64)
        ggg = np.ones(3)
        _lib.call("rsdft_gpu_set_grid", ng.ctypes.data, cell.md, cell.coef_lap0, coef.ctypes.data, h.ctypes.data,
                  ggg.ctypes.data, cell.dV)
        v = np.ascontiguousarray(cell.vloc, dtype=np.float64)
        _lib.call("rsdft_gpu_set_vloc", v.ctypes.data, cell.ML, 1)
        lp = np.ascontiguousarray(cell.lma_ptr, dtype=np.int32)
        jj = np.ascontiguousarray(cell.jjp, dtype=np.int32)
        uv = np.ascontiguousarray(cell.uv, dtype=np.float64)
        iu = np.ascontiguousarray(cell.iuv, dtype=np.int32)
        am = np.ascontiguousarray(cell.amap, dtype=np.int32)
        duv = np.ascontiguousarray(cell.duv, dtype=np.float64) if with_forces and cell.duv.size else None
        _lib.call("rsdft_gpu_set_nonlocal", cell.nzlma, lp.ctypes.data, jj.ctypes.data, uv.ctypes.data,
                  iu.ctypes.data, am.ctypes.data, cell.natom, duv.ctypes.data if duv is not None else None)
        self.cell = cell

    def set_stream(self, stream) -> None:
        """Launch on a cudaStream_t (e.g. ``torch.cuda.current_stream().cuda_stream``)."""
        _lib.call("rsdft_gpu_set_stream", stream)

    def synchronize(self) -> None:
        _lib.call("rsdft_gpu_synchronize")

    def register_wf(self, unk: np.ndarray) -> None:
        _lib.call("rsdft_gpu_register_wf", _ptr(unk, name="unk"), unk.shape[0], unk.shape[1])
        self._keep.append(unk)

    def unregister_wf(self, unk: np.ndarray) -> None:
        _lib.call("rsdft_gpu_unregister_wf", _ptr(unk, name="unk"))

    def sync_to_host(self, unk: np.ndarray) -> None:
        _lib.call("rsdft_gpu_sync_to_host", _ptr(unk, name="unk"))

    def sync_to_device(self, unk: np.ndarray) -> None:
        _lib.call("rsdft_gpu_sync_to_device", _ptr(unk, name="unk"))

    # ---------------------------------------------------------- hot path
    def hamiltonian(self, k, s, tpsi, htpsi, n1, n2, ib1, ib2) -> None:
        _lib.call("rsdft_gpu_hamiltonian", k, s, _ptr(tpsi, name="tpsi"), _ptr(htpsi, name="htpsi"), n1, n2, ib1,
                  ib2)

    def op_local(self, s, tpsi, htpsi, z0=0, nz=None) -> None:
        """(T + Vloc) tpsi on z planes [z0, z0 + nz): op_kinetic + op_localpot
        (hamiltonian_module.f90:42,50)."""
        if nz is None:
            nz = int(self.cell.ngrid[2]) - z0
        _lib.call("rsdft_gpu_op_local", s, _ptr(tpsi, name="tpsi"), _ptr(htpsi, name="htpsi"), _ld(tpsi),
                  tpsi.shape[1], z0, nz)

    def op_nonlocal_project(self, tpsi, uvunk) -> None:
        """uvunk (nzlma, nb) = iuV dV <uV|tpsi> over this context's projector
        entries (ps_nloc2_op_module.f90:161-175)."""
        _lib.call("rsdft_gpu_op_nonlocal_project", _ptr(tpsi, name="tpsi"), _ld(tpsi), tpsi.shape[1],
                  _ptr(uvunk, name="uvunk"))

    def op_nonlocal_add(self, uvunk, htpsi) -> None:
        """htpsi += uV uvunk at this context's projector points
        (ps_nloc2_op_module.f90:255-263)."""
        _lib.call("rsdft_gpu_op_nonlocal_add", _ptr(uvunk, name="uvunk"), _ptr(htpsi, name="htpsi"), _ld(htpsi),
                  htpsi.shape[1])

    def gram(self, a, b, cmat, *, alpha=1.0, sym=0) -> None:
        """cmat(m, n) = alpha a^T b over a's rows (the partial sum of one grid
        slab; gram_schmidt_t_module.f90:187, subspace_diag_la_module.f90:96)."""
        if a.shape[0] != b.shape[0] or _ld(a) != _ld(b):
            raise ValueError("gram: a and b need the same rows and leading dimension")
        _lib.call("rsdft_gpu_gram", _ptr(a, name="a"), _ptr(b, name="b"), _ld(a), a.shape[0], a.shape[1],
                  b.shape[1], float(alpha), int(sym), _ptr(cmat, name="c"), _ld(cmat))

    def overlap_cholesky(self, smat, rinv) -> float:
        """rinv = R^-1 for smat = R^T R; returns (max diag R / min diag R)^2."""
        kappa = ctypes.c_double(0.0)
        _lib.call("rsdft_gpu_overlap_cholesky", smat.shape[0], _ptr(smat, name="s"), _ld(smat),
                  _ptr(rinv, name="rinv"), _ld(rinv), ctypes.addressof(kappa))
        return float(kappa.value)

    def rr_reduced(self, rinv, hsub, esp, w) -> None:
        """R^-T Hsub R^-1 = V diag(esp) V^T and w = R^-1 V."""
        _lib.call("rsdft_gpu_rr_reduced", hsub.shape[0], _ptr(rinv, name="rinv"), _ld(rinv),
                  _ptr(hsub, name="hsub"), _ld(hsub), _ptr(esp, name="esp"), _ptr(w, name="w"), _ld(w))

    def rotate(self, unk, v) -> None:
        """unk <- unk v on unk's rows (device tensor, any leading dimension)."""
        _lib.call("rsdft_gpu_rotate", _ptr(unk, name="unk"), _ld(unk), unk.shape[0], unk.shape[1],
                  _ptr(v, name="v"), _ld(v))

    def hamiltonian_noalloc(self, k, s, tpsi, htpsi, n1, n2, ib1, ib2) -> None:
        """H psi without any device allocation (static 4 MiB scratch; see the
        header).  tpsi/htpsi must be device tensors or registered arrays."""
        _lib.call("rsdft_gpu_hamiltonian_noalloc", k, s, _ptr(tpsi, name="tpsi"), _ptr(htpsi, name="htpsi"), n1, n2,
                  ib1, ib2)

    def conjugate_gradient(self, n1, n2, MB, k, s, unk, esp, res, *, ncg=3, mloop=3, ipc=4,
                           mode=MODE_FP64) -> None:
        """Reference defaults: Ncg = 3 (cg_module.f90:23), mloop = 3, IPC = 4."""
        _lib.call("rsdft_gpu_conjugate_gradient", n1, n2, MB, k, s, _ptr(unk, name="unk"), _ptr(esp, name="esp"),
                  _ptr(res, name="res"), ncg, mloop, ipc, mode)

    def gram_schmidt(self, n0, n1, k, s, unk, *, nblk=0, nblk1=4, mode=MODE_FP64) -> None:
        _lib.call("rsdft_gpu_gram_schmidt", n0, n1, k, s, _ptr(unk, name="unk"), _ld(unk), nblk, nblk1, mode)

    def subspace_diag(self, k, s, unk, esp, *, mode=MODE_FP64) -> None:
        _lib.call("rsdft_gpu_subspace_diag", k, s, _ptr(unk, name="unk"), _ld(unk), unk.shape[1],
                  _ptr(esp, name="esp"), mode)

    def orth_subspace_diag(self, k, s, unk, esp, *, mode=MODE_FP64) -> None:
        """gram_schmidt + subspace_diag as one Rayleigh-Ritz step."""
        _lib.call("rsdft_gpu_orth_subspace_diag", k, s, _ptr(unk, name="unk"), _ld(unk), unk.shape[1],
                  _ptr(esp, name="esp"), mode)

    def subspace_mate_sl(self, k, s, unk, hsub) -> None:
        _lib.call("rsdft_gpu_subspace_mate", k, s, _ptr(unk, name="unk"), _ld(unk), unk.shape[1],
                  _ptr(hsub, name="hsub"), _ld(hsub))

    def subspace_solv_sl(self, hsub, esp, vsub) -> None:
        _lib.call("rsdft_gpu_subspace_solv", hsub.shape[0], _ptr(hsub, name="hsub"), _ld(hsub),
                  _ptr(esp, name="esp"), _ptr(vsub, name="vsub"), _ld(vsub))

    def subspace_rotv_sl(self, k, s, unk, vsub) -> None:
        _lib.call("rsdft_gpu_subspace_rotv", k, s, _ptr(unk, name="unk"), _ld(unk), unk.shape[1],
                  _ptr(vsub, name="vsub"), _ld(vsub))

    def calc_sweep(self, unk, esp, res, occ, *, diter, nelectron, nspin=1, iconv_check=2, tol_esp=1e-7,
                   mb_ref=None, nfixed=0, dspn=0.0, ekbt=1e-5, kinteg=5, ncg=4, mloop=3, ipc=4,
                   mode=MODE_FP64) -> dict:
        """calc_sweep (sweep_module.f90:60-226) on device-resident bands:
        CG + GS + subspace per spin, calc_fermi, conv_check, up to diter
        iterations.  unk is (ML, MB * nspin); esp / res / occ hold MB * nspin
        values (esp: esp0 on entry).  Returns the iteration count, whether
        conv_check passed and the Fermi level."""
        import ctypes

        mb = unk.shape[1] // nspin
        it = ctypes.c_int(0)
        cv = ctypes.c_int(0)
        ef = ctypes.c_double(0.0)
        _lib.call("rsdft_gpu_calc_sweep", _ptr(unk, name="unk"), _ld(unk), mb, nspin, _ptr(esp, name="esp"),
                  _ptr(res, name="res"), _ptr(occ, name="occ"), diter, iconv_check, tol_esp,
                  mb if mb_ref is None else mb_ref, float(nelectron), nfixed, dspn, ekbt, kinteg, ncg, mloop, ipc,
                  mode, ctypes.addressof(it), ctypes.addressof(cv), ctypes.addressof(ef))
        return {"iter": it.value, "converged": bool(cv.value), "efermi": ef.value}

    def esp_calc(self, k, s, wf, n1, n2, ns, ne, e) -> None:
        _lib.call("rsdft_gpu_esp_calc", k, s, _ptr(wf, name="wf"), n1, n2, ns, ne, _ptr(e, name="e"))

    def residual(self, k, s, wf, e, res) -> None:
        """FP64 Rayleigh quotients e and residual norms res of all columns of wf."""
        _lib.call("rsdft_gpu_residual", k, s, _ptr(wf, name="wf"), _ld(wf), wf.shape[1], _ptr(e, name="e"),
                  _ptr(res, name="res"))

    def calc_force_ps_nloc2(self, MI, force2, unk, occ) -> None:
        """force2 is (3, MI) Fortran-ordered (xyz of atom 1 first)."""
        _lib.call("rsdft_gpu_force_nloc", MI, _ptr(unk, name="unk"), _ld(unk), unk.shape[1],
                  _ptr(occ, name="occ"), _ptr(force2, name="force2"))

    def hpsi_adjoint(self, psi, *, chi=None, occ=None, dl_dv=None, dl_dr=None) -> None:
        _lib.call("rsdft_gpu_hpsi_adjoint", _ptr(psi, name="psi"), _ptr(chi, name="chi"), _ld(psi), psi.shape[1],
                  _ptr(occ, name="occ"), _ptr(dl_dv, name="dl_dv"), _ptr(dl_dr, name="dl_dr"))

    def calc_density(self, unk, occ, rho) -> None:
        """rho(ML) = sum_n occ(n) unk(:, n)^2 (calc_density's NCPP branch,
        density_module.f90:129-136, for one k / spin block)."""
        _lib.call("rsdft_gpu_calc_density", _ptr(unk, name="unk"), _ld(unk), unk.shape[1], _ptr(occ, name="occ"),
                  _ptr(rho, name="rho"))

    # ------------------------------------------------ wavefunction file
    def write_wf(self, path, unk, *, mbwr1=1, mbwr2=None, oc=0, io_ctrl=0, occ=None, aa=None, bb=None,
                 kbb=None, mk=1, ms=1) -> None:
        """write_wf on this context's grid (see the module function)."""
        write_wf(path, unk, self.cell.ngrid, mk=mk, ms=ms, mbwr1=mbwr1, mbwr2=mbwr2, oc=oc, io_ctrl=io_ctrl, occ=occ,
                 aa=aa, bb=bb, kbb=kbb)

    def read_wf(self, path, unk, *, io_ctrl=0, occ=None, mk=1, ms=1) -> dict:
        """read_wf on this context's grid (see the module function)."""
        return read_wf(path, unk, self.cell.ngrid, mk=mk, ms=ms, io_ctrl=io_ctrl, occ=occ)

    def write_vrho(self, path, rho, vloc, vh, vxc, **kw) -> None:
        """write_vrho on this context's grid (see the module function)."""
        write_vrho(path, self.cell.ngrid, rho, vloc, vh, vxc, **kw)

    def read_vrho(self, path, **kw):
        """read_vrho on this context's grid (see the module function)."""
        return read_vrho(path, self.cell.ngrid, **kw)

    # --------------------------------------------------------- composite
    def finalize_fp64(self, unk, esp, res) -> None:
        """The FP64 closing pass of the mixed forms: CholeskyQR2 in FP64, then
        FP64 Rayleigh quotients and residual norms."""
        ml, mb = unk.shape
        self.gram_schmidt(1, mb, 1, 1, unk, mode=MODE_FP64)
        self.residual(1, 1, unk, esp, res)

    def eigensolver_sweep(self, k, s, unk, esp, res, *, ncg=4, mloop=3, ipc=4, mode=MODE_FP64) -> None:
        """conjugate_gradient + gram_schmidt + subspace_diag in one call."""
        _lib.call("rsdft_gpu_eigensolver_sweep", k, s, _ptr(unk, name="unk"), _ld(unk), unk.shape[1],
                  _ptr(esp, name="esp"), _ptr(res, name="res"), ncg, mloop, ipc, mode)

    def eigensolver_iteration(self, unk, esp, res, *, ncg=4, mloop=3, mode=MODE_FP64, fused=True) -> None:
        """One sweep iteration as calc_sweep runs it (sweep_module.f90:150-155):
        conjugate_gradient -> gram_schmidt -> subspace_diag.  fused=True runs it
        as one eigensolver_sweep call (Gram-Schmidt and Rayleigh-Ritz as one
        step); fused=False makes the three reference calls."""
        ml, mb = unk.shape
        if fused:
            self.eigensolver_sweep(1, 1, unk, esp, res, ncg=ncg, mloop=mloop, mode=mode)
            return
        self.conjugate_gradient(1, ml, mb, 1, 1, unk, esp, res, ncg=ncg, mloop=mloop, mode=mode)
        self.gram_schmidt(1, mb, 1, 1, unk, mode=mode)
        self.subspace_diag(1, 1, unk, esp, mode=mode)
