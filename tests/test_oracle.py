"""The oracle itself, pinned against the reference's known answers (CPU).

* FD weights: the table the reference prints (examples/Si216/a.log:249-273).
* dsygv(2x2) restatement: LAPACK's own dsygv (scipy.linalg.lapack).
* hpsi: the explicit matrix of construct_hamiltonian_matrix.
* Gram-Schmidt: the unique positive-R QR factor.
* CG / GS / subspace: convergence to the dense-matrix eigenvalues.
* Nonlocal force: central finite differences of E with the sphere support fixed.
* Golden fixture: regression of the oracle's own outputs.
"""
import json
import os

import numpy as np
import pytest
import scipy.linalg.lapack as lapack

from oracle import oracle as O
from rsdft_b200 import cell as C
from rsdft_b200 import fd

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_fd_weights_match_reference_table():
    kat = json.load(open(os.path.join(GOLD, "fd_kat_si216.json")))
    # printed with f20.15: agreement to half a unit in the 15th decimal plus
    # one ulp of the value
    tol = lambda v: 5e-16 + 2.3e-16 * abs(v)  # noqa: E731
    lap = fd.lapla_coefficients(6)
    nab = fd.nabla_coefficients(6)
    for n in range(7):
        assert abs(lap[n] - kat["lap"][n]) <= tol(lap[n]) + 1e-15
    for n in range(1, 7):
        assert abs(nab[n] - kat["nab"][n - 1]) <= tol(nab[n]) + 1e-15
    c0, cl = fd.kinetic_coefficients(6, [kat["Hgrid"]] * 3)
    assert abs(c0 - kat["coef_lap0"]) <= 1e-15 * abs(c0)
    for n in range(6):
        assert abs(cl[0, n] - kat["coef_lap"][n]) <= tol(cl[0, n]) + 1e-15
    h = kat["Hgrid"]
    for n in range(6):
        assert abs(nab[n + 1] / h - kat["coef_nab"][n]) <= 2e-15


@pytest.mark.parametrize("md", [1, 2, 4, 6, 8])
def test_fd_laplacian_exact_on_polynomials(md):
    lap = fd.lapla_coefficients(md)
    # the 2Md+1 point formula differentiates x^k exactly for k <= 2Md
    for k in range(0, 2 * md + 1, 2):
        x = np.arange(-md, md + 1, dtype=float)
        f = x ** k
        d2 = lap[0] * f[md] + sum(lap[m] * (f[md + m] + f[md - m]) for m in range(1, md + 1))
        exact = k * (k - 1) * 0.0 ** (k - 2) if k >= 2 else 0.0
        scale = max(abs(lap[m]) * f[md + m] for m in range(0, md + 1))
        assert abs(d2 - exact) < 1e-13 * scale + 1e-12


def test_dsygv2_matches_lapack():
    rng = np.random.default_rng(0)
    for _ in range(3000):
        X = rng.standard_normal((2, 2))
        B = X @ X.T + 1e-2 * np.eye(2)
        A = rng.standard_normal((2, 2))
        A = A + A.T
        w, v = O.dsygv2(A, B)
        r = lapack.dsygv(A, B, itype=1, jobz="V", uplo="U")
        w2, v2 = r[0], r[1].copy()
        assert r[-1] == 0
        for k in range(2):
            if v2[0, k] < 0:
                v2[:, k] *= -1
            if v[0, k] < 0:
                v[:, k] *= -1
        assert np.allclose(w, w2, rtol=1e-12, atol=1e-13 * np.abs(w2).max())
        assert np.abs(v - v2).max() <= 1e-11 * np.abs(v2).max()


def test_hpsi_matches_dense_matrix():
    c = C.build_cell("si8_g12")
    o = O.Oracle(c)
    Hd = o.dense_hamiltonian()
    assert np.abs(Hd - Hd.T).max() == 0.0
    psi = c.psi0()
    h = o.hamiltonian(psi)
    assert np.abs(h - Hd @ psi).max() <= 1e-14 * np.abs(h).max()


def test_gram_schmidt_is_positive_r_qr():
    c = C.build_cell("si8_g12")
    o = O.Oracle(c)
    psi = c.psi0()
    for nblk in (0, 5):
        u = o.gram_schmidt_t(psi, nblk=nblk)
        q, r = np.linalg.qr(psi)
        q = q * np.sign(np.diag(r)) / np.sqrt(c.dV)
        assert np.abs(u - q).max() <= 1e-13 * np.abs(q).max()
        assert np.abs(u.T @ u * c.dV - np.eye(u.shape[1])).max() <= 1e-14


def test_eigensolver_converges_to_dense_eigenvalues():
    c = C.build_cell("si8_g12")
    o = O.Oracle(c)
    exact = np.linalg.eigvalsh(o.dense_hamiltonian())[: c.nband]
    u = o.gram_schmidt_t(c.psi0())
    e_prev = None
    for it in range(40):
        u, esp, res, _ = o.conjugate_gradient(u, 4, 3)
        u = o.gram_schmidt_t(u)
        u, w, _ = o.subspace_diag_la(u)
        if e_prev is not None:
            # Ritz values bound the exact eigenvalues from above
            assert np.all(w >= exact - 1e-10)
        e_prev = w
    nconv = c.nband // 2
    assert np.abs(w[:nconv] - exact[:nconv]).max() < 1e-6


def test_subspace_mate_lower_triangle():
    c = C.build_cell("si8_g12")
    o = O.Oracle(c)
    u = o.gram_schmidt_t(c.psi0())
    for mblk in (None, 5, 8):
        hs = o.subspace_mate_sl(u, mblk)
        full = c.dV * (u.T @ o.hamiltonian(u))
        assert np.abs(hs - np.tril(full)).max() <= 1e-13 * np.abs(full).max()
    w, v = O.subspace_solv(hs)
    u3, w2, _ = o.subspace_diag_la(u)
    assert np.abs(w - w2).max() <= 1e-12 * np.abs(w2).max()


def test_force_matches_finite_difference_of_energy():
    c = C.build_cell("si8_g12")
    o = O.Oracle(c)
    psi = o.gram_schmidt_t(c.psi0())
    occ = c.occupations()
    F = o.force_nloc(psi, occ)
    h = 1e-4
    uv0 = c.uv.copy()
    for (ia, k) in [(0, 0), (3, 1), (5, 2)]:
        e = []
        for s in (+1, -1):
            at = c.atoms.copy()
            at[ia, k] += s * h
            c.uv[:] = C.projector_values(c, at)
            oo = O.Oracle(c)
            e.append(oo.energy(psi, occ))
        c.uv[:] = uv0
        dE = (e[0] - e[1]) / (2 * h)
        assert abs(-dE - F[ia, k]) < 1e-7 + 1e-5 * abs(F[ia, k])
    O.Oracle(c)  # restore tables


def test_golden_oracle_regression():
    g = np.load(os.path.join(GOLD, "oracle_si8_g12.npz"))
    c = C.build_cell("si8_g12")
    o = O.Oracle(c)
    psi = np.asfortranarray(c.psi0())
    idx = g["idx"]
    h = o.hamiltonian(psi[:, :4])
    assert np.allclose(h[idx], g["hpsi"], rtol=1e-13, atol=1e-13)
    q = o.gram_schmidt_t(psi)
    assert np.allclose(q[idx, :4], g["gs"], rtol=1e-12, atol=1e-12)
    u, esp, res, _ = o.conjugate_gradient(q, 4, 3)
    assert np.allclose(esp, g["cg_esp"], rtol=1e-11, atol=1e-12)
    assert np.allclose(res, g["cg_res"], rtol=1e-9, atol=1e-12)
    u3, w, _ = o.subspace_diag_la(o.gram_schmidt_t(u))
    assert np.allclose(w, g["sub_esp"], rtol=1e-11, atol=1e-12)
    f = o.force_nloc(u3, c.occupations())
    assert np.allclose(f, g["force"], rtol=1e-8, atol=1e-10)


def test_calc_fermi_restatement():
    """calc_fermi (fermi_mp_module.f90:95-284): the electron count is matched,
    occupations lie in [0, 2] (up to the Methfessel-Paxton overshoot, which
    vanishes for well separated levels), degenerate levels share equally,
    and the fixed-moment branch fills each spin to its own count."""
    rng = np.random.default_rng(7)
    e = np.sort(rng.uniform(-0.5, 0.8, 40))
    e[19] = e[20]  # a degenerate pair at the Fermi level: 19 + 1 of 2 levels filled
    occ, ef = O.calc_fermi(e, 40.0)
    assert abs(occ.sum() - 40.0) <= 1e-10
    assert occ[19, 0] == occ[20, 0] and abs(occ[19, 0] - 1.0) <= 1e-12
    assert np.all(occ[:19] > 2.0 - 1e-12) and np.all(occ[21:] < 1e-12)
    assert e[18] < ef < e[21]
    e2 = np.stack([e, e + 0.05], axis=1)
    occ2, _ = O.calc_fermi(e2, 40.0, nfixed=5, dspn=2.0, it=1)
    assert abs(occ2[:, 0].sum() - 21.0) <= 1e-10 and abs(occ2[:, 1].sum() - 19.0) <= 1e-10
    occ3, _ = O.calc_fermi(e2, 40.0, nfixed=5, dspn=2.0, it=6)  # past nfixed: one common level
    assert abs(occ3.sum() - 40.0) <= 1e-10
