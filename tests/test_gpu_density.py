"""rsdft_gpu_calc_density against the reference's sum, calc_density's NCPP
branch (density_module.f90:129-136): rho = rho + occ(n) |unk(:, n)|^2 band
after band, for a host array and a device tensor."""
import numpy as np
import pytest

from rsdft_b200 import api

pytestmark = pytest.mark.gpu


def reference_density(unk, occ):
    rho = np.zeros(unk.shape[0])
    for n in range(unk.shape[1]):
        rho = rho + occ[n] * np.abs(unk[:, n]) ** 2
    return rho


def test_density_matches_the_reference_sum(gpu, cells):
    import torch

    cell = cells("si8_g12")
    gpu.setup(cell, with_forces=False)
    rng = np.random.default_rng(21)
    unk = np.asfortranarray(rng.standard_normal((cell.ML, 7)))
    occ = np.array([2.0, 2.0, 2.0, 1.5, 0.0, 0.5, 0.0])
    ref = reference_density(unk, occ)
    rho = np.zeros(cell.ML)
    gpu.calc_density(unk, occ, rho)
    assert np.abs(rho - ref).max() <= 1e-14 * ref.max()
    dev = api.fortran_empty(cell.ML, 7)
    dev.copy_(torch.from_numpy(np.ascontiguousarray(unk.T)).t())
    rho_d = torch.zeros(cell.ML, dtype=torch.float64, device="cuda")
    gpu.calc_density(dev, occ, rho_d)
    torch.cuda.synchronize()
    assert np.array_equal(rho_d.cpu().numpy(), rho)
