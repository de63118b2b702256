"""RSDFT's wavefunction file through rsdft_gpu_write_wf / rsdft_gpu_read_wf,
on the CPU (host arrays need no device).

`reference_bytes` restates, record by record, what simple_wf_io_write
(io_write_module.f90:148-264) writes for one process with SYStype = 0 and
IO_ctrl = 0: Fortran sequential unformatted records, each framed by 4-byte
length markers.  The library's file must equal it byte for byte; the reader
must invert it, including a file whose LL2 grid map is not x-fastest (the
reader places points through the map, io_read_module.f90:322-329).
"""
import os
import struct

import numpy as np
import pytest

from rsdft_b200 import api
from rsdft_b200._lib import RsdftError

NG = (6, 5, 4)
ML = 6 * 5 * 4


def rec(payload: bytes) -> bytes:
    return struct.pack("<i", len(payload)) + payload + struct.pack("<i", len(payload))


def ints(*v) -> bytes:
    return np.asarray(v, dtype="<i4").tobytes()


def ll2_xfast(ng):
    n1, n2, n3 = ng
    i = np.arange(n1 * n2 * n3)
    return np.stack([i % n1, (i // n1) % n2, i // (n1 * n2)], axis=1).astype("<i4")  # (ML, 3) = LL2(3, ML)^T


def reference_bytes(unk4, ng, mbwr1, mbwr2, oc, occ, aa, bb, kbb, ll2=None, io_ctrl=0):
    """simple_wf_io_write's records (io_write_module.f90:148-170, :236-246)."""
    ml, mb, mk, ms = unk4.shape
    ll2 = ll2_xfast(ng) if ll2 is None else ll2
    out = []
    if oc < 10:
        out += [rec(ints(-1)), rec(ints(ml, *ng)), rec(ints(mb, mbwr1, mbwr2)), rec(ints(mk, ms, kbb.shape[1])),
                rec(ints(io_ctrl, oc, 1)), rec(ll2.tobytes()), rec(np.asfortranarray(occ).tobytes(order="F")),
                rec(np.concatenate([aa.ravel(order="F"), bb.ravel(order="F"), kbb.ravel(order="F")]).tobytes()),
                rec(ints(*([1] * 8)))]
        out += [rec(ints(0, c)) for c in (ml, mb, mk, ms)]
    else:
        out += [rec(ints(ml, *ng)), rec(ints(mb, mbwr1, mbwr2)), rec(ll2.tobytes()),
                rec(np.asfortranarray(occ).tobytes(order="F"))]
    data = []
    for s in range(ms):
        for k in range(mk):
            for n in range(mbwr1 - 1, mbwr2):
                v = unk4[:, n, k, s]
                data.append(rec((v.astype("<f4") if oc in (4, 5) else v.astype("<f8")).tobytes()))
    return b"".join(out), b"".join(data)


def case(mb=5, mk=1, ms=1, seed=0):
    rng = np.random.default_rng(seed)
    unk = np.asfortranarray(rng.standard_normal((ML, mb, mk, ms)))
    occ = np.asfortranarray(rng.uniform(0, 2, (mb, mk, ms)))
    aa = np.asfortranarray(np.diag([10.2, 10.2, 10.2]) + 0.1 * rng.standard_normal((3, 3)))
    bb = np.asfortranarray(2 * np.pi * np.linalg.inv(aa).T)
    kbb = np.asfortranarray(rng.standard_normal((3, 2)))
    return unk, occ, aa, bb, kbb


@pytest.mark.parametrize("oc", [0, 4, 10])
def test_file_equals_the_reference_records(tmp_path, oc):
    unk, occ, aa, bb, kbb = case()
    path = tmp_path / "wf.dat1"
    api.write_wf(path, unk, NG, mbwr1=2, mbwr2=4, oc=oc, occ=occ, aa=aa, bb=bb, kbb=kbb)
    head, data = reference_bytes(unk, NG, 2, 4, oc, occ, aa, bb, kbb)
    assert path.read_bytes() == head + data


def test_split_file_layout(tmp_path):
    unk, occ, aa, bb, kbb = case(mk=2, ms=2, seed=1)
    path = tmp_path / "wf.dat1"
    api.write_wf(path, unk, NG, oc=0, io_ctrl=3, occ=occ, aa=aa, bb=bb, kbb=kbb)
    head, data = reference_bytes(unk, NG, 1, 5, 0, occ, aa, bb, kbb, io_ctrl=3)
    assert path.read_bytes() == head
    assert (tmp_path / "wf.dat1.00000").read_bytes() == data


@pytest.mark.parametrize("oc,io_ctrl", [(0, 0), (4, 0), (5, 3), (10, 0)])
def test_round_trip(tmp_path, oc, io_ctrl):
    unk, occ, aa, bb, kbb = case(mb=4, mk=2, ms=2, seed=2)
    path = tmp_path / "wf.dat1"
    api.write_wf(path, unk, NG, oc=oc, io_ctrl=io_ctrl, occ=occ, aa=aa, bb=bb, kbb=kbb)
    back = np.asfortranarray(np.zeros_like(unk))
    occ2 = np.asfortranarray(np.zeros_like(occ))
    hdr = api.read_wf(path, back, NG, io_ctrl=io_ctrl, occ=occ2)
    want = unk.astype(np.float32).astype(np.float64) if oc in (4, 5) else unk
    assert np.array_equal(back, want)
    assert np.array_equal(occ2, occ)
    assert (hdr["ML"], hdr["ML1"], hdr["ML2"], hdr["ML3"]) == (ML, *NG)
    assert (hdr["MB"], hdr["MB1"], hdr["MB2"]) == (4, 1, 4)
    if oc < 10:
        assert (hdr["MK"], hdr["MS"], hdr["MMBZ"], hdr["IO_ctrl"], hdr["OC"], hdr["TYPE_WF"]) == (2, 2, 2, io_ctrl,
                                                                                                  oc, 1)


def test_band_subset_and_reference_correction(tmp_path):
    unk, occ, aa, bb, kbb = case(mb=6, seed=3)
    path = tmp_path / "wf.dat1"
    api.write_wf(path, unk, NG, mbwr1=3, mbwr2=5, occ=occ)
    back = np.asfortranarray(np.full_like(unk, 7.0))
    hdr = api.read_wf(path, back, NG)
    assert (hdr["MB1"], hdr["MB2"]) == (3, 5)
    assert np.array_equal(back[:, 2:5], unk[:, 2:5])
    assert np.all(back[:, [0, 1, 5]] == 7.0)  # bands outside the file's range are left alone
    # a band range outside 1..MB falls back to the whole range (io_write_module.f90:80-81)
    api.write_wf(path, unk, NG, mbwr1=0, mbwr2=99, occ=occ)
    assert api.read_wf(path, back, NG)["MB1"] == 1 and api.read_wf(path, back, NG)["MB2"] == 6
    assert np.array_equal(back, unk)


def test_reader_follows_the_grid_map(tmp_path):
    """A file whose LL2 lists the points z fastest is placed through the map."""
    unk, occ, aa, bb, kbb = case(mb=3, seed=4)
    n1, n2, n3 = NG
    i = np.arange(ML)
    i3, i2, i1 = i % n3, (i // n3) % n2, i // (n3 * n2)  # z fastest in the file
    ll2 = np.stack([i1, i2, i3], axis=1).astype("<i4")
    grid_index = i1 + n1 * (i2 + n2 * i3)
    file_unk = np.asfortranarray(unk[grid_index])  # file point j holds grid point grid_index[j]
    head, data = reference_bytes(file_unk, NG, 1, 3, 0, occ, aa, bb, kbb, ll2=ll2)
    path = tmp_path / "wf.dat1"
    path.write_bytes(head + data)
    back = np.asfortranarray(np.zeros_like(unk))
    api.read_wf(path, back, NG)
    assert np.array_equal(back, unk)


def test_reader_takes_more_bands_than_it_stores(tmp_path):
    """A file with more bands, k points or spins than the target skips them."""
    unk, occ, aa, bb, kbb = case(mb=5, mk=2, ms=1, seed=5)
    path = tmp_path / "wf.dat1"
    api.write_wf(path, unk, NG, occ=occ, aa=aa, bb=bb, kbb=kbb)
    small = np.asfortranarray(np.zeros((ML, 3)))
    occ3 = np.asfortranarray(np.zeros((3, 1, 1)))
    hdr = api.read_wf(path, small, NG, occ=occ3)
    assert hdr["MB"] == 5 and hdr["MK"] == 2
    assert np.array_equal(small, unk[:, :3, 0, 0])
    assert np.array_equal(occ3[:, 0, 0], occ[:3, 0, 0])


def test_errors(tmp_path):
    unk, occ, aa, bb, kbb = case(seed=6)
    path = tmp_path / "wf.dat1"
    api.write_wf(path, unk, NG, occ=occ)
    back = np.asfortranarray(np.zeros_like(unk))
    with pytest.raises(RsdftError) as e:
        api.read_wf(path, back, (5, 6, 4))  # another grid of the same size
    assert e.value.code == -1 and "file grid" in str(e.value)
    with pytest.raises(RsdftError) as e:
        api.write_wf(path, unk, NG, io_ctrl=1)
    assert e.value.code == -6
    raw = path.read_bytes()
    (tmp_path / "cut.dat1").write_bytes(raw[:-100])  # truncated inside the last band
    with pytest.raises(RsdftError) as e:
        api.read_wf(tmp_path / "cut.dat1", back, NG)
    assert e.value.code == -1
    # complex data (TYPE_WF = 0) in the new format
    head, data = reference_bytes(unk, NG, 1, 5, 0, occ, aa, bb, kbb)
    cplx = head.replace(rec(ints(0, 0, 1)), rec(ints(0, 0, 0)), 1)
    (tmp_path / "cplx.dat1").write_bytes(cplx + data)
    with pytest.raises(RsdftError) as e:
        api.read_wf(tmp_path / "cplx.dat1", back, NG)
    assert e.value.code == -6
    # a grid map that lists a point twice
    ll2 = ll2_xfast(NG)
    ll2[1] = ll2[0]
    head, data = reference_bytes(unk, NG, 1, 5, 0, occ, aa, bb, kbb, ll2=ll2)
    (tmp_path / "dup.dat1").write_bytes(head + data)
    with pytest.raises(RsdftError) as e:
        api.read_wf(tmp_path / "dup.dat1", back, NG)
    assert e.value.code == -1 and "twice" in str(e.value)
    with pytest.raises(RsdftError):
        api.read_wf(tmp_path / "missing.dat1", back, NG)
    assert not os.path.exists(tmp_path / "missing.dat1")
