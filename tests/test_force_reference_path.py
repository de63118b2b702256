"""The reference's tabulated nonlocal-force derivative, restated in the
oracle, against the analytic derivative the product uses (CPU).

calc_force_ps_nloc2 (ps_nloc2_module.f90:1489-1586) does not differentiate
the projectors analytically: ps_nloc2_init_derivative
(ps_nloc2_init_module.f90:219-301) tabulates radial derivatives with dpolint
on the radial grid, and every sphere point interpolates them with polint and
couples them to Ylm through the Gaunt tables of get_gaunt_coefficient_L1
(force_sub_sub_module.f90:64-387).  The oracle restates that path
(``oracle.reference_duvdr``); these tests pin its pieces and bound its
distance from the exact derivative:

* the coupling coefficients computed from their definition equal the
  reference's hard-coded table (fixture read from the reference source by
  tests/golden/make_golden.py) to 1e-14;
* uV = viod(r) * Ylm with the restated Ylm reproduces the cell's projector
  values (the reference's real-harmonic signs, Condon-Shortley phase);
* the dpolint derivative, the interpolated duVdR and the forces built on it
  stay within the truncation error of the reference's 3-point windows on the
  2e-3 bohr radial grid: 1.5e-5 relative for the derivative at r < rc - dr,
  3e-5 for duVdR, 2e-5 for the forces of the displaced 12^3 cell.
"""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from rsdft_b200 import cell as C

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_gaunt_coefficients_equal_reference_table():
    G = O.gaunt_l1(1)
    fx = json.load(open(os.path.join(GOLD, "gaunt_l1.json")))
    for k, name in enumerate(("Y1", "Y2", "Y3")):
        tab = np.zeros_like(G[k])
        for L, m, L1, L1z, v in fx[name]:
            tab[L, m + 1, L1, L1z + 2] = v
        assert len(fx[name]) >= 5
        assert np.abs(G[k] - tab).max() <= 1e-14, name


def test_ylm_restatement_reproduces_projector_values():
    c = C.build_cell("si8_g12")
    n = c.ngrid[0]
    L = O.lib()
    for lma in range(c.nzlma):
        s, e = c.lma_ptr[lma], c.lma_ptr[lma + 1]
        ia, l, m = c.amap[lma], c.lmap[lma], c.mmap[lma]
        j = c.jjp[s:e].astype(np.int64)
        d = np.stack([(j % n) * c.h[0], ((j // n) % n) * c.h[1], (j // (n * n)) * c.h[2]], axis=1) - c.atoms[ia]
        d -= c.a * np.round(d / c.a)
        r = np.sqrt((d * d).sum(1))
        viod = np.sqrt(c.dvals[ia, l]) * r ** l * np.exp(-r * r / C.PROJ_ALPHA)
        y = np.array([L.oracle_ylm(x[0], x[1], x[2], int(l), int(m)) for x in d])
        assert np.allclose(viod * y, c.uv[s:e], rtol=1e-13, atol=1e-15)


def test_dpolint_derivative_table():
    L = O.lib()
    nrc = int(round(C.PROJ_RC / O.RAD_DR)) + 1
    rad = np.arange(nrc) * O.RAD_DR
    v = np.ascontiguousarray(np.exp(-rad ** 2 / C.PROJ_ALPHA))
    out = np.zeros(nrc)
    assert L.oracle_dviod(O._p(rad), O._p(v), nrc, 0, O._p(out)) == 0
    dv = out[1:] / (np.sqrt(4 * np.pi / 3) * rad[1:] ** 2)
    exact = -2.0 * rad[1:] / C.PROJ_ALPHA * v[1:]
    rel = np.abs(dv - exact) / np.abs(exact)
    assert rel[:-1].max() <= 1.5e-5  # the last point has one-sided windows only


@pytest.mark.parametrize("name", ["si8", "si8_g12"])
def test_reference_duvdr_close_to_analytic(name):
    c = C.build_cell(name)
    d = O.reference_duvdr(c)
    assert d.shape == c.duv.shape
    assert np.abs(d - c.duv).max() <= 3e-5 * np.abs(c.duv).max()


def test_reference_path_force_close_to_analytic():
    c = C.build_cell("si8_g12")
    o = O.Oracle(c)
    psi = o.gram_schmidt_t(np.asfortranarray(c.psi0()))
    occ = c.occupations()
    f_an = o.force_nloc(psi, occ)
    f_ref = o.force_nloc_with(psi, occ, O.reference_duvdr(c))
    assert np.abs(f_ref - f_an).max() <= 2e-5 * np.abs(f_an).max()
