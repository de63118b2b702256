"""The C-ABI boundary on the CPU: the library loads, exports every symbol the
header declares, the binding table matches the header, and entries fail with a
status (not a crash) when no device is bound."""
import ctypes
import os
import re

import pytest

from rsdft_b200 import _lib, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "rsdft_gpu.h")


def declared():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(rsdft_gpu_\w+)\s*\(", txt)))


@pytest.fixture(scope="module")
def lib():
    build.build()
    return ctypes.CDLL(build.LIB)


def test_header_declares_entries():
    names = declared()
    assert "rsdft_gpu_hamiltonian" in names and "rsdft_gpu_conjugate_gradient" in names
    assert len(names) >= 20


def test_library_exports_all_declared(lib):
    for n in declared():
        assert hasattr(lib, n), f"{n} declared in rsdft_gpu.h but not exported"


def test_binding_table_matches_header():
    assert sorted(_lib.SIGNATURES) == declared()


def test_debug_build_exports_the_same_entries(lib):
    """The debug build (-DRSDFT_GPU_CHECK, in-kernel index checks) is built
    beside the normal one, exports every declared entry and says which it is;
    rsdft_gpu_checked_build touches no device."""
    import ctypes

    from rsdft_b200 import build

    path = build.build(check=True)
    dbg = ctypes.CDLL(path)
    for n in declared():
        assert hasattr(dbg, n), f"{n} missing from the debug build"
    assert dbg.rsdft_gpu_checked_build() == 1
    assert lib.rsdft_gpu_checked_build() == 0


def test_calls_without_context_fail_cleanly(lib):
    L = _lib.load()
    rc = L.rsdft_gpu_hamiltonian(1, 1, None, None, 1, 10, 1, 1)
    assert rc == -2  # ENOTINIT
    assert b"rsdft_gpu_init" in L.rsdft_gpu_last_error()
    rc = L.rsdft_gpu_conjugate_gradient(1, 10, 1, 1, 1, None, None, None, 4, 3, 4, 0)
    assert rc == -2


def test_init_reports_missing_device(lib):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a device is present")
    L = _lib.load()
    rc = L.rsdft_gpu_init(0)
    assert rc in (-1, -3)
    assert len(L.rsdft_gpu_last_error()) > 0


def test_every_entry_is_defined_once_and_opens_a_trace_range():
    """Each C-ABI entry is defined once in csrc and starts with RS_ENTRY() (an
    NVTX range named after it), except the plain getters."""
    import glob

    src = "".join(open(f).read() for f in sorted(glob.glob(os.path.join(ROOT, "rsdft_b200", "csrc", "*.cu"))))
    defs = re.findall(r'(?m)^(?:extern "C" )?(?:int|long long|const char\*) (rsdft_gpu_\w+)\([^)]*\)\s*\{\s*(\S+)', src)
    names = [n for n, _ in defs]
    assert sorted(names) == declared()
    getters = {"rsdft_gpu_last_error", "rsdft_gpu_kernel_launches", "rsdft_gpu_workspace_bytes",
               "rsdft_gpu_checked_build"}
    for name, first in defs:
        if name not in getters:
            assert first == "RS_ENTRY();", f"{name} does not open with RS_ENTRY()"
