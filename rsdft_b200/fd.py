"""Finite-difference coefficients of the Md-order central Laplacian and gradient.

Host-side set-up for the kinetic operator.  The weights are the closed-form
Lagrange-derivative formulas RSDFT uses:

* ``lapla_coefficients`` follows ``get_coef_lapla_fd`` (fd_module.f90:18-54);
* ``nabla_coefficients`` follows ``get_coef_nabla_fd`` (fd_module.f90:56-78);
* ``kinetic_coefficients`` follows ``init_kinetic`` (kinetic_module.f90:77-89):
  ``coef_lap0 = lap(0)*(c1+c2+c3)``, ``coef_lap(axis,n) = lap(n)*c_axis`` with
  ``c_axis = -0.5*ggg(axis)/H_axis**2``.

The loops keep the reference's summation order so that the weights agree to
the last bit with the table the reference prints (examples/Si216/a.log:249-273).
"""
from __future__ import annotations

import numpy as np


def lapla_coefficients(md: int) -> np.ndarray:
    """Return ``lap(0..Md)`` (second-derivative weights, symmetric)."""
    if md < 1:
        raise ValueError("Md must be >= 1")
    s = 0.0
    for i in range(-md, md + 1):
        if i == 0:
            continue
        for j in range(-md, md + 1):
            if j == i or j == 0:
                continue
            s += 1.0 / float(i * j)
    lap = np.zeros(md + 1)
    lap[0] = s
    for j in range(1, md + 1):
        t = 1.0
        for i in range(-md, md + 1):
            if i == j:
                continue
            t *= float(j - i)
        s = 0.0
        for k in range(-md, md + 1):
            if k == j or k == 0:
                continue
            s0 = 1.0
            for i in range(-md, md + 1):
                if i == k or i == j or i == 0:
                    continue
                s0 *= float(-i)
            s += s0
        lap[j] = 2.0 * s / t
    return lap


def nabla_coefficients(md: int) -> np.ndarray:
    """Return ``nab(0..Md)`` (first-derivative weights; nab(0) = 0)."""
    nab = np.zeros(md + 1)
    for j in range(1, md + 1):
        t = 1.0
        for i in range(-md, md + 1):
            if i == j:
                continue
            t *= float(j - i)
        s = 1.0
        for i in range(-md, md + 1):
            if i == j or i == 0:
                continue
            s *= float(-i)
        nab[j] = s / t
    return nab


def kinetic_coefficients(md: int, hgrid, ggg=(1.0, 1.0, 1.0)):
    """Return ``(coef_lap0, coef_lap[3, Md])`` for an orthorhombic grid.

    ``hgrid`` is the spacing per axis; ``ggg`` the diagonal metric factors
    (1 for an orthogonal cell, get_ggg_kinetic).  k = Gamma, so ``const_k2 = 0``.
    """
    lap = lapla_coefficients(md)
    h1, h2, h3 = (float(h) for h in hgrid)
    c1 = -0.5 * ggg[0] / h1 ** 2
    c2 = -0.5 * ggg[1] / h2 ** 2
    c3 = -0.5 * ggg[2] / h3 ** 2
    coef_lap0 = lap[0] * (c1 + c2 + c3)
    coef_lap = np.zeros((3, md))
    for n in range(1, md + 1):
        coef_lap[0, n - 1] = lap[n] * c1
        coef_lap[1, n - 1] = lap[n] * c2
        coef_lap[2, n - 1] = lap[n] * c3
    return coef_lap0, coef_lap


def precond_coefficients(hgrid, ggg=(1.0, 1.0, 1.0)):
    """Return ``(c, c1, c2, c3)`` of the 7-point preconditioner operator.

    Follows ``precond_cg_mat2_omp`` (cgpc_hprsdft_module.f90:290-293):
    ``c = ggg1/H1^2 + ggg2/H2^2 + ggg3/H3^2``, ``c_axis = -0.5/H_axis^2*ggg_axis``.
    """
    h1, h2, h3 = (float(h) for h in hgrid)
    c = ggg[0] / h1 ** 2 + ggg[1] / h2 ** 2 + ggg[2] / h3 ** 2
    c1 = -0.5 / h1 ** 2 * ggg[0]
    c2 = -0.5 / h2 ** 2 * ggg[1]
    c3 = -0.5 / h3 ** 2 * ggg[2]
    return c, c1, c2, c3
