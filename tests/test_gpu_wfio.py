"""The wavefunction file from device-resident bands: a device tensor and a
registered host array (whose device mirror is what counts) are written band
by band through pinned buffers and must give the same bytes as the host
array; reading fills the device memory.  The file format itself is checked
against the reference's records on the CPU (tests/test_wfio.py).  The
session `gpu` fixture puts torch and the library on one stream, so torch's
copies and the library's transfers are ordered."""
import numpy as np
import pytest

from rsdft_b200 import api

pytestmark = pytest.mark.gpu

NG = (8, 6, 4)
ML = 8 * 6 * 4


@pytest.mark.parametrize("oc", [0, 4])
def test_device_tensor_round_trip(gpu, tmp_path, oc):
    import torch

    rng = np.random.default_rng(11 + oc)
    host = np.asfortranarray(rng.standard_normal((ML, 5)))
    dev = api.fortran_empty(ML, 5)
    dev.copy_(torch.from_numpy(np.ascontiguousarray(host.T)).t())
    api.write_wf(tmp_path / "h.dat1", host, NG, oc=oc)
    api.write_wf(tmp_path / "d.dat1", dev, NG, oc=oc)
    assert (tmp_path / "d.dat1").read_bytes() == (tmp_path / "h.dat1").read_bytes()
    back = api.fortran_empty(ML, 5)
    back.zero_()
    api.read_wf(tmp_path / "d.dat1", back, NG)
    torch.cuda.synchronize()
    want = host.astype(np.float32).astype(np.float64) if oc == 4 else host
    assert np.array_equal(back.cpu().numpy(), want)


def test_registered_array_uses_its_mirror(gpu, tmp_path):
    rng = np.random.default_rng(5)
    host = np.asfortranarray(rng.standard_normal((ML, 4)))
    original = host.copy(order="F")
    gpu.register_wf(host)  # the mirror now holds `original`
    try:
        host[:] = 0.0  # the host copy is stale from here on
        api.write_wf(tmp_path / "r.dat1", host, NG)
        ref = np.asfortranarray(original)
        api.write_wf(tmp_path / "ref.dat1", ref, NG)
        assert (tmp_path / "r.dat1").read_bytes() == (tmp_path / "ref.dat1").read_bytes()
        # reading fills the mirror; sync_to_host brings it back
        other = np.asfortranarray(rng.standard_normal((ML, 4)))
        api.write_wf(tmp_path / "o.dat1", other, NG, io_ctrl=3)
        api.read_wf(tmp_path / "o.dat1", host, NG, io_ctrl=3)
        assert np.all(host == 0.0)
        gpu.sync_to_host(host)
        assert np.array_equal(host, other)
    finally:
        gpu.unregister_wf(host)


def test_vrho_from_device_fields(gpu, tmp_path):
    """The density/potential file from device tensors equals the one from
    host arrays, and reading fills device tensors (format checked on the CPU
    in tests/test_vrho.py)."""
    import torch

    rng = np.random.default_rng(21)
    host = [np.asfortranarray(rng.standard_normal((ML, 2))) for _ in range(3)] + [rng.standard_normal(ML)]
    rho, vloc, vxc, vh = host

    def to_dev(a):
        if a.ndim == 1:
            return torch.from_numpy(a).cuda()
        d = api.fortran_empty(ML, a.shape[1])
        d.copy_(torch.from_numpy(np.ascontiguousarray(a.T)).t())
        return d

    kw = dict(aa=np.diag([10.26] * 3), aa_atom=np.full((3, 2), 0.25), ki_atom=[1, 1], zn_atom=[14], efermi=0.3)
    api.write_vrho(tmp_path / "h.dat1", NG, rho, vloc, vh, vxc, **kw)
    api.write_vrho(tmp_path / "d.dat1", NG, *(to_dev(a) for a in (rho, vloc, vh, vxc)), **kw)
    assert (tmp_path / "d.dat1").read_bytes() == (tmp_path / "h.dat1").read_bytes()
    back = [api.fortran_empty(ML, 2).zero_() for _ in range(3)] + [torch.zeros(ML, dtype=torch.float64, device="cuda")]
    ef = api.read_vrho(tmp_path / "d.dat1", NG, rho=back[0], vloc=back[1], vxc=back[2], vh=back[3], nspin=2)
    torch.cuda.synchronize()
    assert ef == 0.3
    for a, b in zip(host, back):
        assert np.array_equal(b.cpu().numpy(), a)
