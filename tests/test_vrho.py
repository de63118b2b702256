"""RSDFT's density/potential file through rsdft_gpu_write_vrho /
rsdft_gpu_read_vrho, on the CPU (host arrays need no device).

`reference_bytes` restates, record by record, what write_data
(io_module.f90:97-226) writes for one process: the version record, the grid,
LL2, the lattice, the atoms, the Fermi energy, then rho, Vloc, Vh (first
spin only) and Vxc per spin, each a Fortran sequential unformatted record
framed by 4-byte length markers.  The library's file must equal it byte for
byte; the reader must invert it, place values through a permuted LL2
(read_data, io_module.f90:365-373) and accept the unversioned layout, which
has no lattice, atom or Fermi records (io_module.f90:288-296, :324-334).
"""
import struct

import numpy as np
import pytest

from rsdft_b200 import api
from rsdft_b200._lib import RsdftError

NG = (6, 5, 4)
ML = 6 * 5 * 4
VERSION = b"version3.0, comment_length=64"


def rec(payload: bytes) -> bytes:
    return struct.pack("<i", len(payload)) + payload + struct.pack("<i", len(payload))


def ints(*v) -> bytes:
    return np.asarray(v, dtype="<i4").tobytes()


def text(s: bytes) -> bytes:
    return s.ljust(64, b" ")


def ll2_xfast(ng):
    n1, n2, n3 = ng
    i = np.arange(n1 * n2 * n3)
    return np.stack([i % n1, (i // n1) % n2, i // (n1 * n2)], axis=1).astype("<i4")  # LL2(3, ML)^T


def fields(nspin, seed=0):
    rng = np.random.default_rng(seed)
    rho = np.asfortranarray(rng.uniform(0, 1, (ML, nspin)))
    vloc = np.asfortranarray(rng.standard_normal((ML, nspin)))
    vh = rng.standard_normal(ML)
    vxc = np.asfortranarray(rng.standard_normal((ML, nspin)))
    return rho, vloc, vh, vxc


def atoms(seed=1):
    rng = np.random.default_rng(seed)
    aa = np.asfortranarray(np.diag([10.26] * 3) + 0.01 * rng.standard_normal((3, 3)))
    aa_atom = np.asfortranarray(rng.uniform(0, 1, (3, 4)))
    ki_atom = np.array([1, 2, 1, 2], dtype=np.int32)
    zn_atom = np.array([14, 8], dtype=np.int32)
    return aa, aa_atom, ki_atom, zn_atom


def field_records(rho, vloc, vh, vxc, perm):
    """The per-spin field records (io_module.f90:125-215), grid points in the
    file's order: file point i holds the value of grid point perm[i]."""
    out = []
    for s in range(rho.shape[1]):
        out.append(rec(rho[perm, s].astype("<f8").tobytes()))
        out.append(rec(vloc[perm, s].astype("<f8").tobytes()))
        if s == 0:
            out.append(rec(vh[perm].astype("<f8").tobytes()))
        out.append(rec(vxc[perm, s].astype("<f8").tobytes()))
    return out


def reference_bytes(ng, rho, vloc, vh, vxc, aa, aa_atom, ki_atom, zn_atom, efermi, ll2=None, versioned=True):
    """write_data's records (io_module.f90:104-122 and the field loop)."""
    ml = int(np.prod(ng))
    ll2 = ll2_xfast(ng) if ll2 is None else ll2
    perm = ll2[:, 0] + ng[0] * (ll2[:, 1] + ng[1] * ll2[:, 2])
    out = [rec(text(VERSION))] if versioned else []
    out += [rec(ints(ml, *ng)), rec(ll2.tobytes())]
    if versioned:
        out += [rec(text(b"lattice aa(3,3)")), rec(aa.ravel(order="F").astype("<f8").tobytes()),
                rec(text(b"atom: Nelement Natom / aa_atom / ki_atom /zn_atom")),
                rec(ints(zn_atom.size, ki_atom.size)), rec(aa_atom.ravel(order="F").astype("<f8").tobytes()),
                rec(ki_atom.astype("<i4").tobytes()), rec(zn_atom.astype("<i4").tobytes()),
                rec(text(b"Fermi energy")), rec(struct.pack("<d", efermi))]
    return b"".join(out + field_records(rho, vloc, vh, vxc, perm))


@pytest.mark.parametrize("nspin", [1, 2])
def test_write_matches_reference_records(tmp_path, nspin):
    rho, vloc, vh, vxc = fields(nspin)
    aa, aa_atom, ki_atom, zn_atom = atoms()
    path = tmp_path / "vrho.dat1"
    api.write_vrho(path, NG, rho, vloc, vh, vxc, aa=aa, aa_atom=aa_atom, ki_atom=ki_atom, zn_atom=zn_atom,
                   efermi=0.2137)
    assert path.read_bytes() == reference_bytes(NG, rho, vloc, vh, vxc, aa, aa_atom, ki_atom, zn_atom, 0.2137)


@pytest.mark.parametrize("nspin", [1, 2])
def test_round_trip(tmp_path, nspin):
    rho, vloc, vh, vxc = fields(nspin, seed=3)
    aa, aa_atom, ki_atom, zn_atom = atoms()
    path = tmp_path / "vrho.dat1"
    api.write_vrho(path, NG, rho, vloc, vh, vxc, aa=aa, aa_atom=aa_atom, ki_atom=ki_atom, zn_atom=zn_atom,
                   efermi=-0.125)
    back = [np.asfortranarray(np.zeros_like(a)) for a in (rho, vloc, vh, vxc)]
    ef = api.read_vrho(path, NG, rho=back[0], vloc=back[1], vh=back[2], vxc=back[3], nspin=nspin)
    assert ef == -0.125
    for a, b in zip((rho, vloc, vh, vxc), back):
        assert np.array_equal(a, b)


def test_read_permuted_grid_map(tmp_path):
    """A file whose LL2 lists the points in another order (another process
    layout's gather) reads back onto the same grid."""
    rho, vloc, vh, vxc = fields(2, seed=5)
    aa, aa_atom, ki_atom, zn_atom = atoms()
    ll2 = ll2_xfast(NG)[np.random.default_rng(7).permutation(ML)]
    path = tmp_path / "perm.dat1"
    path.write_bytes(reference_bytes(NG, rho, vloc, vh, vxc, aa, aa_atom, ki_atom, zn_atom, 0.5, ll2=ll2))
    back = [np.asfortranarray(np.zeros_like(a)) for a in (rho, vloc, vh, vxc)]
    assert api.read_vrho(path, NG, rho=back[0], vloc=back[1], vh=back[2], vxc=back[3], nspin=2) == 0.5
    for a, b in zip((rho, vloc, vh, vxc), back):
        assert np.array_equal(a, b)


def test_read_unversioned_file(tmp_path):
    """The older layout: no version, lattice, atom or Fermi records; the
    Fermi energy is left as it was (None here)."""
    rho, vloc, vh, vxc = fields(1, seed=9)
    aa, aa_atom, ki_atom, zn_atom = atoms()
    path = tmp_path / "old.dat1"
    path.write_bytes(reference_bytes(NG, rho, vloc, vh, vxc, aa, aa_atom, ki_atom, zn_atom, 0.0, versioned=False))
    back = [np.asfortranarray(np.zeros_like(a)) for a in (rho, vloc, vh, vxc)]
    assert api.read_vrho(path, NG, rho=back[0], vloc=back[1], vh=back[2], vxc=back[3]) is None
    for a, b in zip((rho, vloc, vh, vxc), back):
        assert np.array_equal(a, b)


def test_read_selected_fields(tmp_path):
    rho, vloc, vh, vxc = fields(1, seed=11)
    path = tmp_path / "vrho.dat1"
    api.write_vrho(path, NG, rho, vloc, vh, vxc)
    only = np.zeros(ML)
    api.read_vrho(path, NG, vloc=only)
    assert np.array_equal(only, vloc[:, 0])


def test_errors(tmp_path):
    rho, vloc, vh, vxc = fields(1)
    path = tmp_path / "vrho.dat1"
    api.write_vrho(path, NG, rho, vloc, vh, vxc)
    with pytest.raises(RsdftError, match="grid"):
        api.read_vrho(path, (6, 5, 5), rho=np.zeros(6 * 5 * 5))
    with pytest.raises(RsdftError):
        api.read_vrho(tmp_path / "missing.dat1", NG, rho=np.zeros(ML))
    # a truncated file
    short = tmp_path / "short.dat1"
    short.write_bytes(path.read_bytes()[:-100])
    with pytest.raises(RsdftError, match="Vxc"):
        api.read_vrho(short, NG, rho=np.zeros(ML))
    # an LL2 entry off the grid
    bad = bytearray(path.read_bytes())
    at = len(rec(text(VERSION))) + len(rec(ints(ML, *NG))) + 4
    bad[at:at + 4] = struct.pack("<i", 99)
    badp = tmp_path / "bad.dat1"
    badp.write_bytes(bytes(bad))
    with pytest.raises(RsdftError, match="off the grid"):
        api.read_vrho(badp, NG, rho=np.zeros(ML))
    with pytest.raises(ValueError):
        api.write_vrho(path, NG, rho[:-1], vloc, vh, vxc)
