"""Failure detection on the GPU without a GPU fault: a kernel whose mbarrier
wait can never complete gives up after its clock budget and sets the error
flag, the next synchronize reports RSDFT_ETIMEOUT (and clears it), and the
context keeps working (an hpsi call afterwards still matches the oracle)."""
import numpy as np
import pytest

from rsdft_b200 import _lib

from test_gpu_parity import prepare

pytestmark = pytest.mark.gpu


def test_bounded_wait_reports_timeout_and_context_survives(gpu, cells):
    L = _lib.load()
    assert L.rsdft_gpu_synchronize() == 0
    assert L.rsdft_gpu_selftest_timeout(2_000_000) == 0  # ~1 ms of SM clock
    assert L.rsdft_gpu_synchronize() == -7  # RSDFT_ETIMEOUT
    assert b"bounded wait" in L.rsdft_gpu_last_error()
    assert L.rsdft_gpu_synchronize() == 0  # the flag was cleared
    assert L.rsdft_gpu_selftest_timeout(0) == -1  # EINVAL
    c, o = prepare(gpu, cells, "si8")
    rng = np.random.default_rng(3)
    psi = np.asfortranarray(rng.standard_normal((c.ML, 4)))
    hpsi = np.zeros_like(psi, order="F")
    gpu.hamiltonian(1, 1, psi, hpsi, 1, c.ML, 1, 4)
    ref = o.hamiltonian(psi)
    assert np.abs(hpsi - ref).max() <= 1e-12 * np.abs(ref).max()
