"""The s-step form of the CG preconditioner, restated in numpy, against the
oracle's literal recurrences.

precond_hprsdft with IPC = 4 (cgpc_hprsdft_module.f90:126-263) runs mloop CG
steps on A z = g from z = g, A the 7-point operator d + offdiag
(precond_cg_mat2_omp, :281-348).  The device code (csrc/precond.cu) does
not run those recurrences on vectors: it builds the Chebyshev basis
w_0 = g - A g, w_1 = B w_0, w_{k+1} = 2 B w_k - w_{k-1} (B = offdiag / d)
in z-march passes, forms the Gram entries <w_i, w_j> and <w_j, g>, runs the
same recurrences on coefficient vectors with A's tridiagonal image in that
basis (s_sstep), and assembles Pg = g + sum_j c_j w_j and
rb = <g|g> + sum_j c_j <w_j|g> (k_ss_p, cg_module.f90:232-250).  This test
restates that scheme step by step in FP64 and checks it against
oracle_precond on the 12^3 cell for mloop = 1..4: the two are the same
algorithm up to rounding, including the early exit at |r0|^2 < 1e-24
(:186).
"""
import numpy as np
import pytest

from oracle.oracle import Oracle
from rsdft_b200 import fd
from rsdft_b200.cell import build_cell


@pytest.fixture(scope="module")
def setup():
    cell = build_cell("si8_g12", with_duv=False)
    return cell, Oracle(cell), fd.precond_coefficients(cell.h)


def offdiag(f, ngrid, c1, c2, c3):
    """The 7-point operator without its diagonal, on an x-fastest vector."""
    n1, n2, n3 = ngrid
    v = f.reshape(n3, n2, n1)
    o = (c1 * (np.roll(v, 1, 2) + np.roll(v, -1, 2)) + c2 * (np.roll(v, 1, 1) + np.roll(v, -1, 1))
         + c3 * (np.roll(v, 1, 0) + np.roll(v, -1, 0)))
    return o.ravel()


def sstep_precond(g, m, ngrid, coef):
    """Pg and <Pg|g> through the Chebyshev basis and coefficient recurrences."""
    d, c1, c2, c3 = coef
    w = [g - (d * g + offdiag(g, ngrid, c1, c2, c3))]
    for k in range(1, m + 1):
        b = offdiag(w[k - 1], ngrid, c1, c2, c3) / d
        w.append(b if k == 1 else 2.0 * b - w[k - 2])
    # the Gram entries the basis passes form: <w_k, w_j> for j <= k < m,
    # <w_m, w_j> for j < m (never <w_m, w_m>), and <w_j, g> for j < m
    G = np.zeros((m + 1, m + 1))
    for k in range(m + 1):
        for j in range(min(k + 1, m)):
            G[k, j] = G[j, k] = w[k] @ w[j]
    gd = np.array([w[j] @ g for j in range(m)])
    # A in the basis: A w_0 = d (w_0 + w_1), A w_j = d w_j + d/2 (w_{j+1} + w_{j-1})
    T = np.zeros((m + 1, m + 1))
    T[0, 0] = T[1, 0] = d
    for j in range(1, m):
        T[j, j] = d
        T[j + 1, j] = T[j - 1, j] = 0.5 * d
    cz = np.zeros(m + 1)
    rr = G[0, 0]
    if not rr < 1e-24:
        r = np.zeros(m + 1)
        r[0] = 1.0
        q = r.copy()
        for il in range(1, m + 1):
            ft = T @ q
            a = rr / (q @ G @ ft)
            cz += a * q
            if il == m:
                break
            r -= a * ft
            rn = r @ G @ r
            q = r + (rn / rr) * q
            rr = rn
    assert cz[m] == 0.0  # the last basis vector only ever enters the dot products
    pg = g + sum(cz[j] * w[j] for j in range(m))
    return pg, g @ g + cz[:m] @ gd


def inputs(cell, coef, rng):
    n1, n2, n3 = cell.ngrid
    i = np.arange(cell.ML)
    x, y, z = i % n1, (i // n1) % n2, i // (n1 * n2)
    rough = rng.standard_normal(cell.ML)
    d, c1, c2, c3 = coef
    a = lambda f: d * f + offdiag(f, cell.ngrid, c1, c2, c3)  # noqa: E731
    return {
        "random": rough,
        "smooth": np.cos(2 * np.pi * x / n1) * np.sin(4 * np.pi * y / n2) + 0.3 * np.cos(2 * np.pi * z / n3),
        "high_frequency": a(a(rough)),
        "gradient_like": rough * np.exp(-((x - n1 / 2) ** 2 + (y - n2 / 2) ** 2 + (z - n3 / 2) ** 2) / 8.0),
    }


@pytest.mark.parametrize("mloop", [1, 2, 3, 4])
def test_sstep_form_matches_literal_recurrences(setup, mloop):
    cell, orc, coef = setup
    rng = np.random.default_rng(40 + mloop)
    for name, g in inputs(cell, coef, rng).items():
        ref = orc.precond(g, mloop)
        pg, rb = sstep_precond(g, mloop, cell.ngrid, coef)
        scale = np.abs(ref).max()
        assert np.abs(pg - ref).max() <= 1e-12 * scale, (name, np.abs(pg - ref).max() / scale)
        rb_ref = ref @ g
        assert abs(rb - rb_ref) <= 1e-12 * abs(rb_ref), (name, rb, rb_ref)


def test_sstep_form_early_exit(setup):
    """|r0|^2 < 1e-24: both forms return g unchanged."""
    cell, orc, coef = setup
    g = 1e-15 * np.random.default_rng(3).standard_normal(cell.ML)
    ref = orc.precond(g, 3)
    pg, _ = sstep_precond(g, 3, cell.ngrid, coef)
    assert np.array_equal(ref, g) and np.array_equal(pg, g)
