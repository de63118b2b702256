"""Two spin channels (MSP = 2): rsdft_gpu_set_vloc with Vloc(ML, 2), and
hamiltonian / conjugate_gradient / the one-call sweep with s = 2 use the
second channel (hamiltonian_module.f90:50: op_localpot with Vloc(:, s)),
against the oracle bound to that channel; s = 1 keeps the first."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from rsdft_b200 import _lib, api

from test_gpu_parity import TOL, dev, host, rel

pytestmark = pytest.mark.gpu


def _two_channels(gpu, c):
    gpu.setup(c)
    n1, n2, n3 = c.ngrid
    i = np.arange(c.ML)
    z = i // (n1 * n2)
    v2 = np.asarray(c.vloc) + 0.05 * np.cos(2 * np.pi * z / n3)  # a spin-split channel
    both = np.asfortranarray(np.stack([np.asarray(c.vloc), v2], axis=1))
    _lib.call("rsdft_gpu_set_vloc", both.ctypes.data, c.ML, 2)
    return v2


def test_hamiltonian_and_cg_second_spin(gpu, cells):
    c = cells("si8")
    v2 = _two_channels(gpu, c)
    nb = 8
    psi = np.asfortranarray(c.psi0()[:, :nb])
    out = api.fortran_empty(c.ML, nb)
    for s, vl in ((2, v2), (1, None)):
        o = O.Oracle(c, spin_vloc=vl)
        gpu.hamiltonian(1, s, dev(psi), out, 1, c.ML, 1, nb)
        torch.cuda.synchronize()
        assert rel(host(out), o.hamiltonian(psi)) <= TOL, s
    o = O.Oracle(c, spin_vloc=v2)
    q = o.gram_schmidt_t(psi)
    ru, resp, rres, _ = o.conjugate_gradient(q, 4, 3)
    u = dev(q)
    esp = torch.zeros(nb, dtype=torch.float64, device="cuda")
    res = torch.zeros_like(esp)
    gpu.conjugate_gradient(1, c.ML, nb, 1, 2, u, esp, res, ncg=4, mloop=3)
    torch.cuda.synchronize()
    assert rel(host(esp), resp) <= TOL
    assert rel(host(res), rres) <= TOL
    assert rel(host(u), ru) <= TOL


def test_sweep_second_spin(gpu, cells):
    """One eigensolver_sweep on channel 2 against the oracle's CG ->
    gram_schmidt_t -> subspace_diag_la on that channel."""
    c = cells("si8")
    v2 = _two_channels(gpu, c)
    nb = 16
    o = O.Oracle(c, spin_vloc=v2)
    q = o.gram_schmidt_t(np.asfortranarray(c.psi0()[:, :nb]))
    u0, _, _, _ = o.conjugate_gradient(q, 4, 3)
    _, w, _ = o.subspace_diag_la(o.gram_schmidt_t(u0))
    u = dev(q)
    esp = torch.zeros(nb, dtype=torch.float64, device="cuda")
    res = torch.zeros_like(esp)
    gpu.eigensolver_sweep(1, 2, u, esp, res, ncg=4, mloop=3)
    torch.cuda.synchronize()
    assert rel(host(esp), w) <= 1e-11
