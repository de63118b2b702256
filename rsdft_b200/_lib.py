"""ctypes binding of librsdft_gpu.so (the C ABI declared in include/rsdft_gpu.h).

Importing this module never compiles anything; ``load()`` raises if the
library has not been built (``python -m rsdft_b200.build``).  There is no CPU
fallback.  With ``RSDFT_GPU_CHECK=1`` in the environment the debug build
``librsdft_gpu_check.so`` (in-kernel index checks; ``python -m
rsdft_b200.build --check``) is loaded instead.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librsdft_gpu_check.so" if os.environ.get("RSDFT_GPU_CHECK") == "1"
                        else "librsdft_gpu.so")

_c_int, _c_long, _c_double, _vp = ctypes.c_int, ctypes.c_long, ctypes.c_double, ctypes.c_void_p

# name -> (restype, argtypes); must match include/rsdft_gpu.h
SIGNATURES = {
    "rsdft_gpu_init": (_c_int, [_c_int]),
    "rsdft_gpu_finalize": (_c_int, []),
    "rsdft_gpu_last_error": (ctypes.c_char_p, []),
    "rsdft_gpu_set_stream": (_c_int, [_vp]),
    "rsdft_gpu_synchronize": (_c_int, []),
    "rsdft_gpu_kernel_launches": (ctypes.c_longlong, []),
    "rsdft_gpu_workspace_bytes": (ctypes.c_longlong, []),
    "rsdft_gpu_selftest_timeout": (_c_int, [ctypes.c_longlong]),
    "rsdft_gpu_checked_build": (_c_int, []),
    "rsdft_gpu_selftest_check": (_c_int, []),
    "rsdft_gpu_set_grid": (_c_int, [_vp, _c_int, _c_double, _vp, _vp, _vp, _c_double]),
    "rsdft_gpu_set_vloc": (_c_int, [_vp, _c_long, _c_int]),
    "rsdft_gpu_set_nonlocal": (_c_int, [_c_int, _vp, _vp, _vp, _vp, _vp, _c_int, _vp]),
    "rsdft_gpu_register_wf": (_c_int, [_vp, _c_long, _c_int]),
    "rsdft_gpu_unregister_wf": (_c_int, [_vp]),
    "rsdft_gpu_sync_to_host": (_c_int, [_vp]),
    "rsdft_gpu_sync_to_device": (_c_int, [_vp]),
    "rsdft_gpu_hamiltonian": (_c_int, [_c_int, _c_int, _vp, _vp, _c_int, _c_int, _c_int, _c_int]),
    "rsdft_gpu_op_local": (_c_int, [_c_int, _vp, _vp, _c_long, _c_int, _c_int, _c_int]),
    "rsdft_gpu_op_nonlocal_project": (_c_int, [_vp, _c_long, _c_int, _vp]),
    "rsdft_gpu_op_nonlocal_add": (_c_int, [_vp, _vp, _c_long, _c_int]),
    "rsdft_gpu_gram": (_c_int, [_vp, _vp, _c_long, _c_long, _c_int, _c_int, _c_double, _c_int, _vp, _c_int]),
    "rsdft_gpu_overlap_cholesky": (_c_int, [_c_int, _vp, _c_int, _vp, _c_int, _vp]),
    "rsdft_gpu_rr_reduced": (_c_int, [_c_int, _vp, _c_int, _vp, _c_int, _vp, _vp, _c_int]),
    "rsdft_gpu_rotate": (_c_int, [_vp, _c_long, _c_long, _c_int, _vp, _c_int]),
    "rsdft_gpu_hamiltonian_noalloc": (_c_int, [_c_int, _c_int, _vp, _vp, _c_int, _c_int, _c_int, _c_int]),
    "rsdft_gpu_conjugate_gradient": (_c_int, [_c_int, _c_int, _c_int, _c_int, _c_int, _vp, _vp, _vp, _c_int,
                                              _c_int, _c_int, _c_int]),
    "rsdft_gpu_gram_schmidt": (_c_int, [_c_int, _c_int, _c_int, _c_int, _vp, _c_long, _c_int, _c_int, _c_int]),
    "rsdft_gpu_subspace_mate": (_c_int, [_c_int, _c_int, _vp, _c_long, _c_int, _vp, _c_int]),
    "rsdft_gpu_subspace_solv": (_c_int, [_c_int, _vp, _c_int, _vp, _vp, _c_int]),
    "rsdft_gpu_subspace_rotv": (_c_int, [_c_int, _c_int, _vp, _c_long, _c_int, _vp, _c_int]),
    "rsdft_gpu_subspace_diag": (_c_int, [_c_int, _c_int, _vp, _c_long, _c_int, _vp, _c_int]),
    "rsdft_gpu_orth_subspace_diag": (_c_int, [_c_int, _c_int, _vp, _c_long, _c_int, _vp, _c_int]),
    "rsdft_gpu_eigensolver_sweep": (_c_int, [_c_int, _c_int, _vp, _c_long, _c_int, _vp, _vp, _c_int, _c_int,
                                             _c_int, _c_int]),
    "rsdft_gpu_calc_sweep": (_c_int, [_vp, _c_long, _c_int, _c_int, _vp, _vp, _vp, _c_int, _c_int, _c_double, _c_int,
                                      _c_double, _c_int, _c_double, _c_double, _c_int, _c_int, _c_int, _c_int, _c_int,
                                      _vp, _vp, _vp]),
    "rsdft_gpu_esp_calc": (_c_int, [_c_int, _c_int, _vp, _c_int, _c_int, _c_int, _c_int, _vp]),
    "rsdft_gpu_residual": (_c_int, [_c_int, _c_int, _vp, _c_long, _c_int, _vp, _vp]),
    "rsdft_gpu_force_nloc": (_c_int, [_c_int, _vp, _c_long, _c_int, _vp, _vp]),
    "rsdft_gpu_hpsi_adjoint": (_c_int, [_vp, _vp, _c_long, _c_int, _vp, _vp, _vp]),
    "rsdft_gpu_calc_density": (_c_int, [_vp, _c_long, _c_int, _vp, _vp]),
    "rsdft_gpu_write_wf": (_c_int, [ctypes.c_char_p, _vp, _c_long, _c_int, _c_int, _c_int, _c_int, _c_int, _c_int,
                                    _c_int, _vp, _vp, _vp, _vp, _c_int, _vp]),
    "rsdft_gpu_read_wf": (_c_int, [ctypes.c_char_p, _vp, _c_long, _c_int, _c_int, _c_int, _c_int, _vp, _vp, _vp]),
    "rsdft_gpu_write_vrho": (_c_int, [ctypes.c_char_p, _vp, _vp, _c_int, _c_int, _vp, _vp, _vp, ctypes.c_double,
                                      _c_int, _vp, _vp, _vp, _vp]),
    "rsdft_gpu_read_vrho": (_c_int, [ctypes.c_char_p, _vp, _c_int, _vp, _vp, _vp, _vp, _vp]),
}

STATUS = {0: "OK", -1: "EINVAL", -2: "ENOTINIT", -3: "ECUDA", -4: "ESOLVER", -5: "ENOMEM", -6: "EUNSUP", -7: "ETIMEOUT", -8: "ECHECK"}

_lib = None


class RsdftError(RuntimeError):
    def __init__(self, func, code, msg):
        super().__init__(f"{func} -> {STATUS.get(code, code)} ({code}): {msg}")
        self.code = code
        self.func = func


def load(path: str = LIB_PATH):
    """Load the CUDA library (raises if it is missing: no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is missing: build it with `python -m rsdft_b200.build`")
        L = ctypes.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def call(name: str, *args) -> None:
    L = load()
    rc = getattr(L, name)(*args)
    if rc != 0:
        msg = L.rsdft_gpu_last_error()
        raise RsdftError(name, rc, msg.decode() if msg else "")
