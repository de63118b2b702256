"""calc_sweep's loop on device-resident bands (rsdft_gpu_calc_sweep), through
the C ABI, on a registered host array as the Fortran driver uses it.

The loop (sweep_module.f90:60-226) is restated on the host around the
library's one-iteration entry: per iteration rsdft_gpu_eigensolver_sweep,
then the oracle's calc_fermi (fermi_mp_module.f90:95-284) and conv_check
(sweep_module.f90:255-266).  rsdft_gpu_calc_sweep must stop at the same
iteration with bitwise the same bands and eigenvalues (it runs the same
device steps), occupations and Fermi level within 1e-12, and the electron
count matched.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from rsdft_b200 import api

from test_gpu_parity import dev, host, prepare

pytestmark = pytest.mark.gpu


def host_loop(gpu, c, u, esp, diter, tol, mode):
    """The reference's loop, restated on the host around eigensolver_sweep."""
    ne = 2.0 * c.nocc
    res = np.zeros(c.nband)
    for it in range(1, diter + 1):
        esp0 = esp.copy()
        gpu.eigensolver_sweep(1, 1, u, esp, res, ncg=4, mloop=3, mode=mode)
        occ, ef = O.calc_fermi(esp, ne)
        m, conv = O.conv_check(esp, esp0, c.nocc, tol)
        if conv or it == diter:
            return it, conv, occ.ravel(), ef, res
    raise AssertionError


@pytest.mark.parametrize("mode", [api.MODE_FP64, api.MODE_MIXED_BF16X3])
def test_calc_sweep_matches_host_loop(gpu, cells, mode):
    c, o = prepare(gpu, cells, "si8")
    start = np.asfortranarray(o.gram_schmidt_t(c.psi0()))
    tol = 1e-9 if mode == api.MODE_FP64 else 1e-6  # eigenvalue change of the occupied bands (mb_ref)
    # reference loop on a device copy
    ua = dev(start)
    ea = np.zeros(c.nband)
    it_a, conv_a, occ_a, ef_a, _ = host_loop(gpu, c, ua, ea, 40, tol, mode)
    # the library's loop on a registered host array
    unk = np.array(start, order="F", copy=True)
    gpu.register_wf(unk)
    try:
        esp = np.zeros(c.nband)
        res = np.zeros(c.nband)
        occ = np.zeros(c.nband)
        r = gpu.calc_sweep(unk, esp, res, occ, diter=40, nelectron=2.0 * c.nocc, tol_esp=tol, mb_ref=c.nocc,
                           mode=mode)
        gpu.sync_to_host(unk)
    finally:
        gpu.unregister_wf(unk)
    assert r["converged"] and conv_a and r["iter"] == it_a, (r, it_a)
    assert np.array_equal(esp, ea)
    assert np.array_equal(unk, host(ua))
    assert np.abs(occ - occ_a).max() <= 1e-12 and abs(occ.sum() - 2.0 * c.nocc) <= 1e-10
    assert abs(r["efermi"] - ef_a) <= 1e-12 * max(1.0, abs(ef_a))


def test_calc_sweep_conv_check_3_and_errors(gpu, cells):
    c, o = prepare(gpu, cells, "si8")
    u = dev(o.gram_schmidt_t(c.psi0()))
    esp = torch.zeros(c.nband, dtype=torch.float64, device="cuda")
    res = torch.zeros_like(esp)
    occ = torch.zeros_like(esp)
    r = gpu.calc_sweep(u, esp, res, occ, diter=3, nelectron=2.0 * c.nocc, iconv_check=3, tol_esp=1e-30)
    assert r["iter"] == 3 and not r["converged"]
    e0 = host(esp).copy()
    # one more iteration: res = |esp - esp0| (none below tol_esp = 1e-30 unless exactly equal)
    r = gpu.calc_sweep(u, esp, res, occ, diter=1, nelectron=2.0 * c.nocc, iconv_check=3, tol_esp=1e-30)
    d = np.abs(host(esp) - e0)
    assert np.allclose(host(res), np.where(d < 1e-30, -1.0, d), rtol=0, atol=0)
    with pytest.raises(api.RsdftError) as e:
        gpu.calc_sweep(u, esp, res, occ, diter=1, nelectron=2.0 * c.nocc, iconv_check=1)
    assert e.value.code == -6
    with pytest.raises(api.RsdftError) as e:
        gpu.calc_sweep(u, esp, res, occ, diter=1, nelectron=2.0 * c.nocc, mb_ref=c.nband + 1)
    assert e.value.code == -1
