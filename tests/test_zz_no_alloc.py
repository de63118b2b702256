"""rsdft_gpu_hamiltonian_noalloc: H psi for callers that cannot allocate
device memory during a call (a host code that gives all of its GPU memory to
its own pool, or a latency-bound loop that must not meet the allocator's
implicit synchronisation).  Its only scratch is a static device array of
RSDFT_NOALLOC_SCRATCH_VALUES doubles shared by every call.

Checked through the C ABI against rsdft_gpu_hamiltonian on two calls in a row
(the second with other bands and another band count, so a stale scratch would
show), within the 1e-12 relative tolerance of the other hpsi parity tests, and
for the clear rejection of a band count whose scratch would not fit.  The
entry is called before rsdft_gpu_hamiltonian every time, so a no-alloc path
that fell back on the library's workspace would find none yet; the first test
asserts that the library's workspace and the device's free memory do not
change across a call.  The file name makes pytest collect it last.
"""
import os
import re

import numpy as np
import pytest
import torch

from rsdft_b200 import _lib

from test_gpu_parity import dev, host, prepare, rel

pytestmark = pytest.mark.gpu

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "rsdft_gpu.h")


def scratch_values():
    txt = open(HEADER).read()
    return int(re.search(r"#define\s+RSDFT_NOALLOC_SCRATCH_VALUES\s+(\d+)L?", txt).group(1))


def both(gpu, c, psi):
    """(rsdft_gpu_hamiltonian, rsdft_gpu_hamiltonian_noalloc) of psi; the
    no-alloc entry runs first."""
    nb = psi.shape[1]
    t = dev(psi)
    h_ref = torch.empty_like(t)
    h_new = torch.full_like(t, float("nan"))
    gpu.hamiltonian_noalloc(1, 1, t, h_new, 1, c.ML, 1, nb)
    torch.cuda.synchronize()
    gpu.hamiltonian(1, 1, t, h_ref, 1, c.ML, 1, nb)
    torch.cuda.synchronize()
    return host(h_ref), host(h_new)


def test_noalloc_allocates_nothing(gpu, cells):
    """Across a call the library's own workspace does not grow, and across a
    second call (after the driver has loaded the kernels' code) the device's
    free memory does not change."""
    c, o = prepare(gpu, cells, "si64")
    lib = _lib.load()
    psi = np.asfortranarray(c.psi0()[:, :24])
    t = dev(psi)
    h = torch.full_like(t, float("nan"))
    torch.cuda.synchronize()
    ws0 = lib.rsdft_gpu_workspace_bytes()
    gpu.hamiltonian_noalloc(1, 1, t, h, 1, c.ML, 1, 24)
    torch.cuda.synchronize()
    assert lib.rsdft_gpu_workspace_bytes() == ws0
    free0 = torch.cuda.mem_get_info()[0]
    gpu.hamiltonian_noalloc(1, 1, t, h, 1, c.ML, 1, 24)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    assert lib.rsdft_gpu_workspace_bytes() == ws0
    assert rel(host(h), o.hamiltonian(psi)) <= 1e-12


def test_noalloc_matches_hamiltonian_twice(gpu, cells):
    c, _ = prepare(gpu, cells, "si64")
    psi0 = np.asfortranarray(c.psi0())
    # first call: all 160 bands
    ref1, new1 = both(gpu, c, psi0)
    assert np.isfinite(new1).all()
    assert rel(new1, ref1) <= 1e-12
    # second call: 37 other bands (reversed order, scaled), fewer than before
    psi1 = np.asfortranarray(-1.7 * psi0[:, ::-1][:, :37])
    ref2, new2 = both(gpu, c, psi1)
    assert np.isfinite(new2).all()
    assert rel(new2, ref2) <= 1e-12


def test_noalloc_rejects_oversized_scratch(gpu, cells):
    c, _ = prepare(gpu, cells, "si64")
    cap = scratch_values()
    nzlma = c.nzlma
    nb = cap // nzlma + 1            # one band more than the scratch holds
    assert nb * nzlma > cap and nb <= 65535
    t = torch.empty((nb, c.ML), dtype=torch.float64, device="cuda").t()
    h = torch.empty_like(t)
    with pytest.raises(_lib.RsdftError) as e:
        gpu.hamiltonian_noalloc(1, 1, t, h, 1, c.ML, 1, nb)
    assert e.value.code == -1 and "exceed" in str(e.value)
    del t, h
    # the context stays usable after the rejection
    psi = np.asfortranarray(c.psi0()[:, :8])
    ref, new = both(gpu, c, psi)
    assert rel(new, ref) <= 1e-12
