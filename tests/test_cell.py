"""Synthetic cell set-up (CPU): the recipe's shapes and the projector algebra."""
import math

import numpy as np
import pytest

from rsdft_b200 import cell as C


def test_splitmix_reproducible():
    a = C.uniform(5, 1000)
    b = C.uniform(5, 1000)
    assert np.array_equal(a, b)
    assert a.min() >= 0.0 and a.max() < 1.0
    assert abs(a.mean() - 0.5) < 0.05
    n = C.normal(9, 20000)
    assert abs(n.mean()) < 0.03 and abs(n.std() - 1.0) < 0.03


@pytest.mark.parametrize("name,ml,natom", [("si8", 13824, 8), ("si64", 110592, 64)])
def test_cell_shapes(name, ml, natom):
    c = C.build_cell(name)
    assert c.ML == ml and c.natom == natom and c.nzlma == 4 * natom
    mjj = np.diff(c.lma_ptr)
    assert 400 < mjj.mean() < 470  # ~437 points in a sphere of 2 bohr at h = 0.4275
    for l in range(c.nzlma):
        s, e = c.lma_ptr[l], c.lma_ptr[l + 1]
        assert np.all(np.diff(c.jjp[s:e]) > 0)  # JJP ascending per projector
    assert abs(c.h[0] - 0.4275) < 1e-12
    assert -2.5 < c.vloc.min() < -0.9 and c.vloc.max() < 2e-3
    assert np.all(c.iuv == 1)


def test_projector_ylm_convention():
    # Ylm of ylm_module.f90: Y1,1 = -c x/r, Y1,-1 = -c y/r, Y1,0 = c z/r
    c = C.build_cell("si8_g12")
    l0 = 0
    base = c.lma_ptr
    for q, (sign, axis) in zip((1, 2, 3), ((-1, 1), (1, 2), (-1, 0))):
        s, e = base[l0 + q], base[l0 + q + 1]
        j = c.jjp[s:e]
        pos = c.grid_coords()[j]
        d = pos - c.atoms[0]
        d -= c.a * np.round(d / c.a)
        r2 = (d ** 2).sum(1)
        ref = math.sqrt(c.dvals[0, 1]) * sign * C.C_Y1 * d[:, axis] * np.exp(-r2 / C.PROJ_ALPHA)
        assert np.allclose(c.uv[s:e], ref, rtol=1e-13, atol=1e-15)


def test_projector_derivative_is_d_dR():
    c = C.build_cell("si8_g12")
    h = 1e-6
    for k in range(3):
        at = c.atoms.copy()
        at[2, k] += h
        up = C.projector_values(c, at)
        at[2, k] -= 2 * h
        dn = C.projector_values(c, at)
        fdv = (up - dn) / (2 * h)
        sel = c.amap[np.searchsorted(c.lma_ptr, np.arange(len(c.uv)), side="right") - 1] == 2
        assert np.allclose(c.duv[sel, k], fdv[sel], rtol=1e-6, atol=1e-8)
