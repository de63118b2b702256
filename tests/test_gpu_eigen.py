"""The small dense symmetric eigensolver behind the subspace steps, through
rsdft_gpu_subspace_solv (the reference's subspace_solv_sl: eigen-decomposition
of Hsub from its lower triangle), against numpy's LAPACK eigh.

Sizes up to ~590 take the cluster-resident tridiagonalisation with bisection
and inverse iteration; larger ones (and n < 3) take cuSOLVER's syevd.  The
spectra cover the shapes the Rayleigh-Ritz step meets: random, nearly
diagonal (converged bands), exactly degenerate triples (a symmetric crystal),
a tight cluster, and widely scaled values.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def spectrum_matrix(n, kind, rng):
    if kind == "random":
        b = rng.standard_normal((n, n))
        return b + b.T
    if kind == "near_diagonal":
        b = rng.standard_normal((n, n))
        return np.diag(np.linspace(-0.5, 1.0, n)) + 1e-3 * (b + b.T)
    q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    if kind == "degenerate":
        lam = np.repeat(np.linspace(-1.0, 1.0, (n + 2) // 3), 3)[:n]
    elif kind == "tight_cluster":
        lam = np.linspace(-1.0, 1.0, n)
        lam[n // 2: n // 2 + 8] = 0.25 + 1e-12 * np.arange(8)
    else:  # scaled
        lam = np.sign(rng.standard_normal(n)) * np.logspace(-6, 2, n)
    a = q @ np.diag(np.sort(lam)) @ q.T
    return 0.5 * (a + a.T)


def solve(gpu, a):
    n = a.shape[0]
    h = np.asfortranarray(np.tril(a))  # only the lower triangle is read
    h += np.triu(np.full((n, n), np.nan), 1)
    w = np.zeros(n)
    v = np.zeros((n, n), order="F")
    gpu.subspace_solv_sl(h, w, v)
    return w, v


@pytest.mark.parametrize("n,kind", [
    (480, "random"), (480, "near_diagonal"), (480, "degenerate"), (480, "tight_cluster"),
    (480, "scaled"), (3, "random"), (4, "degenerate"), (17, "near_diagonal"), (160, "random"),
    (592, "near_diagonal"), (700, "random"), (2, "random"), (1, "random"),
])
def test_subspace_solv_matches_lapack(gpu, n, kind):
    rng = np.random.default_rng(1000 + n)
    a = spectrum_matrix(n, kind, rng)
    w, v = solve(gpu, a)
    wr = np.linalg.eigvalsh(a)
    scale = np.abs(wr).max()
    assert np.all(np.diff(w) >= 0.0)
    assert np.abs(w - wr).max() <= 1e-13 * n * scale
    assert np.abs(v.T @ v - np.eye(n)).max() <= 1e-12
    assert np.abs(a @ v - v * w).max() <= 1e-13 * n * scale


def test_subspace_solv_repeatable(gpu):
    """Same input, same bits (fixed reduction orders, seeded start vectors)."""
    a = spectrum_matrix(480, "near_diagonal", np.random.default_rng(7))
    w1, v1 = solve(gpu, a)
    w2, v2 = solve(gpu, a)
    assert np.array_equal(w1, w2) and np.array_equal(v1, v2)


@pytest.mark.parametrize("n,spread", [(1, 1.0), (31, 1.0), (32, 3.0), (33, 1.0), (37, 1.0), (64, 10.0), (97, 1.0),
                                      (480, 30.0), (600, 300.0), (1088, 30.0)])
def test_overlap_cholesky_inverse(gpu, n, spread):
    """rsdft_gpu_overlap_cholesky: S = R^T R and rinv = R^-1 (upper, the
    lower triangle zero) against LAPACK's Cholesky and an explicit inverse,
    and kappa = (max diag R / min diag R)^2, for overlaps of the shapes a CG
    sweep leaves (near the identity, columns of spread norms)."""
    rng = np.random.default_rng(n)
    b = rng.standard_normal((4 * n + 8, n)) * np.linspace(1.0, np.sqrt(spread), n)
    s = np.asfortranarray(b.T @ b / (4 * n + 8))
    rinv = np.zeros((n, n), order="F")
    kappa = gpu.overlap_cholesky(s, rinv)
    r = np.linalg.cholesky(s).T
    ref = np.linalg.inv(r)
    assert np.abs(rinv - ref).max() <= 1e-12 * np.abs(ref).max() * max(1.0, np.linalg.cond(r))
    assert np.abs(np.tril(rinv, -1)).max() == 0.0
    assert np.abs(rinv @ r - np.eye(n)).max() <= 1e-12 * max(1.0, np.linalg.cond(r))
    d = np.diag(r)
    assert abs(kappa - (d.max() / d.min()) ** 2) <= 1e-12 * kappa


@pytest.mark.parametrize("n,bad", [(8, 1), (100, 41), (480, 480), (130, 97)])
def test_overlap_cholesky_reports_the_failing_pivot(gpu, n, bad):
    """A matrix whose leading minor of order `bad` is the first not positive
    definite: the Cholesky stops with dpotrf's info = bad, and the context
    factors the next matrix normally."""
    from rsdft_b200._lib import RsdftError

    rng = np.random.default_rng(n + bad)
    b = rng.standard_normal((2 * n, n))
    s = b.T @ b / (2 * n)
    r = np.linalg.cholesky(s).T  # s = r^T r; make pivot `bad` negative
    r[bad - 1, bad - 1] = 0.0
    s_bad = r.T @ r
    s_bad[bad - 1, bad - 1] -= 0.5
    rinv = np.zeros((n, n), order="F")
    with pytest.raises(RsdftError, match=f"info={bad}"):
        gpu.overlap_cholesky(np.asfortranarray(s_bad), rinv)
    gpu.overlap_cholesky(np.asfortranarray(s), rinv)
    assert np.abs(rinv @ np.linalg.cholesky(s).T - np.eye(n)).max() <= 1e-11
