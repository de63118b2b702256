"""Parity of the CUDA path (through the C ABI) with the oracle on seeded cells.

FP64 tolerance: 1e-12 relative (max-norm), the bar the plain form must meet.
Eigenvectors are compared through subspace overlaps, never raw columns.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from rsdft_b200 import api
from rsdft_b200.cell import Workload, build_cell, projector_values

pytestmark = pytest.mark.gpu
TOL = 1e-12


def dev(a):
    """numpy (ML, nb) -> Fortran-ordered cuda tensor."""
    a = np.asarray(a, dtype=np.float64)
    if a.ndim == 1:
        return torch.from_numpy(a.copy()).cuda()
    return torch.from_numpy(np.ascontiguousarray(a.T)).cuda().t()


def host(t):
    if t.dim() == 1:
        return t.cpu().numpy()
    return np.asfortranarray(t.t().cpu().numpy().T)


def rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


def prepare(gpu, cells, name):
    """Upload the cell to the library and bind the oracle to the same tables."""
    c = cells(name)
    gpu.setup(c)
    return c, O.Oracle(c)


@pytest.mark.parametrize("name,nb", [("si8", 32), ("si64", 12), ("si8_g12", 16)])
def test_hpsi(gpu, cells, name, nb):
    c, o = prepare(gpu, cells, name)
    psi = np.asfortranarray(c.psi0()[:, :nb])
    ref = o.hamiltonian(psi)
    t = dev(psi)
    out = api.fortran_empty(c.ML, nb)
    gpu.hamiltonian(1, 1, t, out, 1, c.ML, 1, nb)
    torch.cuda.synchronize()
    assert rel(host(out), ref) <= TOL
    # host arrays through the same entry (staged copies)
    hout = np.zeros((c.ML, nb), order="F")
    gpu.hamiltonian(1, 1, psi, hout, 1, c.ML, 1, nb)
    assert rel(hout, ref) <= TOL


@pytest.mark.parametrize("md", [1, 2, 4, 8])
def test_hpsi_fd_orders(gpu, md):
    c = build_cell(Workload(f"si8_md{md}", 1, 20, 6, 3, 0.03, 77, md=md))
    gpu.setup(c)
    o = O.Oracle(c)
    psi = np.asfortranarray(c.psi0())
    ref = o.hamiltonian(psi)
    out = np.zeros_like(psi, order="F")
    gpu.hamiltonian(1, 1, psi, out, 1, c.ML, 1, psi.shape[1])
    assert rel(out, ref) <= TOL


@pytest.mark.parametrize("ngrid", [16, 24])
@pytest.mark.parametrize("md", [1, 2, 3, 4, 5, 6, 7, 8])
def test_hpsi_fd_orders_tma_stencil(gpu, ngrid, md):
    """Grids with 16-byte-aligned rows take the TMA z-march stencil
    (k_stencil_tma): every Md with the periodic wrap of 16- and 24-row grids
    (y halo boxes on both sides, a tile as high as the grid)."""
    c = build_cell(Workload(f"si8_md{md}_g{ngrid}", 1, ngrid, 6, 3, 0.03, 79, md=md))
    gpu.setup(c)
    o = O.Oracle(c)
    psi = np.asfortranarray(c.psi0())
    ref = o.hamiltonian(psi)
    out = np.zeros_like(psi, order="F")
    gpu.hamiltonian(1, 1, psi, out, 1, c.ML, 1, psi.shape[1])
    assert rel(out, ref) <= TOL


def test_hpsi_symmetric(gpu, cells):
    c, o = prepare(gpu, cells, "si8")
    psi = np.asfortranarray(c.psi0()[:, :8])
    t = dev(psi)
    out = api.fortran_empty(c.ML, 8)
    gpu.hamiltonian(1, 1, t, out, 1, c.ML, 1, 8)
    m = psi.T @ host(out)
    assert np.abs(m - m.T).max() <= 1e-12 * np.abs(m).max()


def test_cg_sweep(gpu, cells):
    c, o = prepare(gpu, cells, "si8")
    q = o.gram_schmidt_t(c.psi0())
    ru, resp, rres, _ = o.conjugate_gradient(q, 4, 3)
    u = dev(q)
    esp = torch.zeros(c.nband, dtype=torch.float64, device="cuda")
    res = torch.zeros_like(esp)
    gpu.conjugate_gradient(1, c.ML, c.nband, 1, 1, u, esp, res, ncg=4, mloop=3)
    torch.cuda.synchronize()
    assert rel(host(esp), resp) <= TOL
    assert rel(host(res), rres) <= TOL
    assert rel(host(u), ru) <= TOL


def test_cg_reference_defaults_and_no_preconditioner(gpu, cells):
    c, o = prepare(gpu, cells, "si8_g12")
    q = o.gram_schmidt_t(c.psi0())
    for ncg, mloop, ipc in ((3, 3, 4), (2, 1, 4)):
        ru, resp, rres, _ = o.conjugate_gradient(q, ncg, mloop)
        u = dev(q)
        esp = torch.zeros(c.nband, dtype=torch.float64, device="cuda")
        res = torch.zeros_like(esp)
        gpu.conjugate_gradient(1, c.ML, c.nband, 1, 1, u, esp, res, ncg=ncg, mloop=mloop, ipc=ipc)
        torch.cuda.synchronize()
        assert rel(host(esp), resp) <= TOL
        assert rel(host(res), rres) <= TOL
        assert rel(host(u), ru) <= TOL


@pytest.mark.parametrize("name,nb", [("si8", 32), ("si64", 160)])
def test_gram_schmidt(gpu, cells, name, nb):
    c, o = prepare(gpu, cells, name)
    psi = np.asfortranarray(c.psi0()[:, :nb])
    ref = o.gram_schmidt_t(psi)
    u = dev(psi)
    gpu.gram_schmidt(1, nb, 1, 1, u)
    torch.cuda.synchronize()
    g = host(u)
    assert rel(g, ref) <= TOL
    assert np.abs(g.T @ g * c.dV - np.eye(nb)).max() <= 1e-13


def test_gram_schmidt_band_range(gpu, cells):
    """gram_schmidt(n0, n1): only columns n0..n1 are orthonormalised."""
    c, o = prepare(gpu, cells, "si8")
    psi = np.asfortranarray(c.psi0())
    u = dev(psi)
    gpu.gram_schmidt(5, 20, 1, 1, u)
    g = host(u)
    assert np.array_equal(g[:, :4], psi[:, :4]) and np.array_equal(g[:, 20:], psi[:, 20:])
    assert rel(g[:, 4:20], o.gram_schmidt_t(psi[:, 4:20])) <= TOL


def overlap_check(g, ref, w, dV, gap_tol=1e-6):
    """Columns of g and ref span the same eigenspaces, cluster by cluster."""
    R = ref.T @ g * dV
    n = len(w)
    cl = np.zeros(n, dtype=int)
    for i in range(1, n):
        cl[i] = cl[i - 1] + (1 if w[i] - w[i - 1] > gap_tol * max(1.0, abs(w[i])) else 0)
    worst = 0.0
    for i in range(n):
        for j in range(n):
            if cl[i] != cl[j]:
                worst = max(worst, abs(R[i, j]))
    for k in range(cl[-1] + 1):
        idx = np.where(cl == k)[0]
        blk = R[np.ix_(idx, idx)]
        worst = max(worst, np.abs(blk.T @ blk - np.eye(len(idx))).max())
    return worst


def test_subspace_diag(gpu, cells):
    c, o = prepare(gpu, cells, "si8")
    q = o.gram_schmidt_t(c.psi0())
    u1, _, _, _ = o.conjugate_gradient(q, 4, 3)
    u1 = o.gram_schmidt_t(u1)
    ref, w, _ = o.subspace_diag_la(u1)
    u = dev(u1)
    esp = torch.zeros(c.nband, dtype=torch.float64, device="cuda")
    gpu.subspace_diag(1, 1, u, esp)
    torch.cuda.synchronize()
    assert rel(host(esp), w) <= TOL
    assert overlap_check(host(u), ref, w, c.dV) <= 1e-10


def test_subspace_mate_solv_rotv(gpu, cells):
    c, o = prepare(gpu, cells, "si8")
    u0 = o.gram_schmidt_t(c.psi0())
    hs_ref = o.subspace_mate_sl(u0)
    w_ref, v_ref = O.subspace_solv(hs_ref)
    rot_ref = O.subspace_rotv(u0, v_ref)
    u = dev(u0)
    hsub = np.zeros((c.nband, c.nband), order="F")
    gpu.subspace_mate_sl(1, 1, u, hsub)
    assert rel(hsub, hs_ref) <= TOL
    assert np.all(np.triu(hsub, 1) == 0.0)
    esp = np.zeros(c.nband)
    vsub = np.zeros((c.nband, c.nband), order="F")
    gpu.subspace_solv_sl(hsub, esp, vsub)
    assert rel(esp, w_ref) <= TOL
    gpu.subspace_rotv_sl(1, 1, u, vsub)
    torch.cuda.synchronize()
    assert overlap_check(host(u), rot_ref, w_ref, c.dV) <= 1e-10


@pytest.mark.parametrize("name,nb", [("si8", 32), ("si64", 160)])
def test_orth_subspace_diag_matches_gs_then_subspace(gpu, cells, name, nb):
    """One Rayleigh-Ritz step on non-orthonormal bands (a CG sweep's output)
    equals gram_schmidt followed by subspace_diag."""
    c, o = prepare(gpu, cells, name)
    q = o.gram_schmidt_t(np.asfortranarray(c.psi0()[:, :nb]))
    u0, _, _, _ = o.conjugate_gradient(q, 4, 3)
    ref, w, _ = o.subspace_diag_la(o.gram_schmidt_t(u0))
    u = dev(u0)
    esp = torch.zeros(nb, dtype=torch.float64, device="cuda")
    gpu.orth_subspace_diag(1, 1, u, esp)
    torch.cuda.synchronize()
    g = host(u)
    assert rel(host(esp), w) <= 1e-12
    assert np.abs(g.T @ g * c.dV - np.eye(nb)).max() <= 1e-12
    assert overlap_check(g, ref, w, c.dV) <= 1e-9


def test_orth_subspace_diag_ill_conditioned_overlap(gpu, cells):
    """Two nearly parallel bands: the explicit CholeskyQR2 path is taken and
    the result still equals gram_schmidt followed by subspace_diag."""
    c, o = prepare(gpu, cells, "si8")
    nb = 32
    u0 = np.asfortranarray(c.psi0()[:, :nb]).copy()
    u0[:, 1] = u0[:, 0] + 1e-4 * u0[:, 1]
    ref, w, _ = o.subspace_diag_la(o.gram_schmidt_t(u0))
    u = dev(u0)
    esp = torch.zeros(nb, dtype=torch.float64, device="cuda")
    gpu.orth_subspace_diag(1, 1, u, esp)
    torch.cuda.synchronize()
    g = host(u)
    assert rel(host(esp), w) <= 1e-10
    assert np.abs(g.T @ g * c.dV - np.eye(nb)).max() <= 1e-12


def test_sweep_fp64_equals_separate_calls(gpu, cells):
    """eigensolver_sweep (FP64) runs CG then orth_subspace_diag, handing the
    CG's H x (kept through its updates) to the Rayleigh-Ritz step instead of
    forming H psi again: the same CG (residuals bitwise), eigenvalues and
    eigenvectors of the separate calls to 1e-12."""
    c, o = prepare(gpu, cells, "si8")
    q = o.gram_schmidt_t(c.psi0())
    ua, ub = dev(q), dev(q)
    ea = torch.zeros(c.nband, dtype=torch.float64, device="cuda")
    eb, ra, rb = torch.zeros_like(ea), torch.zeros_like(ea), torch.zeros_like(ea)
    gpu.conjugate_gradient(1, c.ML, c.nband, 1, 1, ua, ea, ra, ncg=4, mloop=3)
    gpu.orth_subspace_diag(1, 1, ua, ea)
    gpu.eigensolver_sweep(1, 1, ub, eb, rb, ncg=4, mloop=3)
    torch.cuda.synchronize()
    assert np.array_equal(host(ra), host(rb))
    assert rel(host(eb), host(ea)) <= TOL
    g, ga = host(ub), host(ua)
    assert np.abs(g.T @ g * c.dV - np.eye(c.nband)).max() <= 1e-12
    assert np.abs(np.abs(np.diag(ga.T @ g * c.dV)) - 1.0).max() <= 1e-9


def test_eigensolver_iteration_sequence(gpu, cells):
    """CG -> GS -> subspace, two iterations, as calc_sweep calls them."""
    c, o = prepare(gpu, cells, "si8")
    u_ref = o.gram_schmidt_t(c.psi0())
    u = dev(u_ref)
    esp = torch.zeros(c.nband, dtype=torch.float64, device="cuda")
    res = torch.zeros_like(esp)
    for it in range(2):
        u_ref, _, _, _ = o.conjugate_gradient(u_ref, 4, 3)
        u_ref = o.gram_schmidt_t(u_ref)
        u_ref, w, _ = o.subspace_diag_la(u_ref)
        gpu.eigensolver_iteration(u, esp, res, ncg=4, mloop=3)
    torch.cuda.synchronize()
    assert rel(host(esp), w) <= 1e-11
    assert overlap_check(host(u), u_ref, w, c.dV) <= 1e-9


@pytest.mark.parametrize("name", ["si8", "si64_adjoint"])
def test_force(gpu, cells, name):
    c, o = prepare(gpu, cells, name)
    nb = 32 if name == "si8" else 40
    psi = np.asfortranarray(c.psi0()[:, :nb])
    occ = np.zeros(nb)
    occ[: nb // 2] = 2.0
    occ[3] = 0.0
    ref = o.force_nloc(psi, occ)  # (natom, 3)
    f = np.zeros((3, c.natom), order="F")
    gpu.calc_force_ps_nloc2(c.natom, f, dev(psi), occ)
    assert rel(f.T, ref) <= TOL


def test_hpsi_adjoint(gpu, cells):
    c, o = prepare(gpu, cells, "si8_g12")
    nb = 8
    psi = np.asfortranarray(o.gram_schmidt_t(c.psi0())[:, :nb])
    occ = np.linspace(2.0, 0.5, nb)
    dv = torch.zeros(c.ML, dtype=torch.float64, device="cuda")
    dr = torch.zeros(3 * c.natom, dtype=torch.float64, device="cuda")
    gpu.hpsi_adjoint(dev(psi), occ=occ, dl_dv=dv, dl_dr=dr)
    torch.cuda.synchronize()
    assert rel(host(dv), O.vloc_adjoint(psi, occ, c.dV)) <= TOL
    F = o.force_nloc(psi, occ)
    assert rel(host(dr).reshape(c.natom, 3), -F) <= TOL
    # general cotangent: L = sum_n chi_n . (H psi_n)
    rng = np.random.default_rng(3)
    chi = np.asfortranarray(rng.standard_normal(psi.shape))
    gpu.hpsi_adjoint(dev(psi), chi=dev(chi), dl_dv=dv, dl_dr=dr)
    torch.cuda.synchronize()
    assert rel(host(dv), np.sum(chi * psi, axis=1)) <= TOL
    h = 1e-5
    ia, k = 1, 2
    uv0 = c.uv.copy()
    L = []
    for s in (1, -1):
        at = c.atoms.copy()
        at[ia, k] += s * h
        c.uv[:] = projector_values(c, at)
        L.append(float(np.sum(chi * O.Oracle(c).hamiltonian(psi))))
    c.uv[:] = uv0
    O.Oracle(c)
    fd_ = (L[0] - L[1]) / (2 * h)
    g = host(dr).reshape(c.natom, 3)[ia, k]
    assert abs(g - fd_) <= 1e-6 * max(1.0, abs(fd_))


def test_registered_host_wavefunction(gpu, cells):
    """The Fortran residency protocol: register host unk, call with element
    addresses, sync back."""
    c, o = prepare(gpu, cells, "si8")
    q = np.asfortranarray(o.gram_schmidt_t(c.psi0()))
    ru, resp, _, _ = o.conjugate_gradient(q, 4, 3)
    unk = np.array(q, order="F", copy=True)
    gpu.register_wf(unk)
    try:
        esp = np.zeros(c.nband)
        res = np.zeros(c.nband)
        gpu.conjugate_gradient(1, c.ML, c.nband, 1, 1, unk, esp, res, ncg=4, mloop=3)
        assert rel(esp, resp) <= TOL
        assert np.array_equal(unk, q)  # host copy untouched until sync
        gpu.sync_to_host(unk)
        assert rel(unk, ru) <= TOL
        # hpsi on a band slice addressed inside the registered array
        out = np.zeros((c.ML, 3), order="F")
        gpu.hamiltonian(1, 1, unk[:, 5:8], out, 1, c.ML, 6, 8)
        assert rel(out, o.hamiltonian(ru[:, 5:8])) <= TOL
    finally:
        gpu.unregister_wf(unk)


def test_span_past_registration_rejected(gpu, cells):
    """A block that starts inside a registered array but runs past its end
    is refused (EINVAL) before any kernel runs, by the staging and the
    no-allocation entries alike; the same block within range works."""
    c, o = prepare(gpu, cells, "si8")
    unk = np.array(c.psi0(), order="F", copy=True)
    gpu.register_wf(unk)
    try:
        nb = c.nband - 4 + 1  # from column 5: one band more than is left
        out = api.fortran_empty(c.ML, nb)
        for call in (gpu.hamiltonian, gpu.hamiltonian_noalloc):
            with pytest.raises(api.RsdftError) as e:
                call(1, 1, unk[:, 4:], out, 1, c.ML, 5, 4 + nb)
            assert e.value.code == -1 and "registered" in str(e.value)
        ok = api.fortran_empty(c.ML, c.nband - 4)
        gpu.hamiltonian(1, 1, unk[:, 4:], ok, 1, c.ML, 5, c.nband)
        torch.cuda.synchronize()
        assert rel(host(ok), o.hamiltonian(unk[:, 4:])) <= TOL
    finally:
        gpu.unregister_wf(unk)


def test_error_statuses(gpu, cells):
    c, o = prepare(gpu, cells, "si8_g12")
    psi = np.asfortranarray(c.psi0())
    out = np.zeros_like(psi, order="F")
    with pytest.raises(api.RsdftError) as e:
        gpu.hamiltonian(2, 1, psi, out, 1, c.ML, 1, 2)
    assert e.value.code == -6
    with pytest.raises(api.RsdftError) as e:
        gpu.hamiltonian(1, 1, psi, out, 1, c.ML - 1, 1, 2)
    assert e.value.code == -1
    with pytest.raises(api.RsdftError) as e:
        gpu.hamiltonian(1, 2, psi, out, 1, c.ML, 1, 2)
    assert e.value.code == -1
    bad = np.array(psi, order="F", copy=True)
    bad[:, 3] = 0.0  # zero band: the overlap matrix is not positive definite
    with pytest.raises(api.RsdftError) as e:
        gpu.gram_schmidt(1, c.nband, 1, 1, bad)
    assert e.value.code == -4
    # the context stays usable after the error
    gpu.hamiltonian(1, 1, psi, out, 1, c.ML, 1, psi.shape[1])
    assert rel(out, o.hamiltonian(psi)) <= TOL


def test_esp_calc_and_residual(gpu, cells):
    c, o = prepare(gpu, cells, "si8")
    psi = np.asfortranarray(o.gram_schmidt_t(c.psi0()))
    h = o.hamiltonian(psi)
    e_ref = np.einsum("ij,ij->j", psi, h) * c.dV  # esp_calc_module.f90:41
    r_ref = np.einsum("ij,ij->j", h - psi * e_ref, h - psi * e_ref) * c.dV
    e = np.zeros(c.nband)
    gpu.esp_calc(1, 1, psi, 1, c.ML, 1, c.nband, e)
    assert rel(e, e_ref) <= TOL
    e2 = np.zeros(c.nband)
    r = np.zeros(c.nband)
    gpu.residual(1, 1, dev(psi), e2, r)
    assert rel(e2, e_ref) <= TOL
    assert rel(r, r_ref) <= 1e-10
