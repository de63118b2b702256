import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def gpu():
    """The library bound to cuda:0 (GPU tests only)."""
    import torch

    if not torch.cuda.is_available():
        pytest.fail("GPU test run without a CUDA device")
    from rsdft_b200 import build as _build
    from rsdft_b200.api import RsdftGpu

    _build.build()
    g = RsdftGpu(0)
    # one stream for torch and the library, so copies and kernels are ordered
    st = torch.cuda.Stream()
    torch.cuda.set_stream(st)
    g.set_stream(st.cuda_stream)
    g._torch_stream = st
    return g


_cells = {}


def get_cell(name):
    from rsdft_b200.cell import build_cell

    if name not in _cells:
        _cells[name] = build_cell(name)
    return _cells[name]


@pytest.fixture(scope="session")
def cells():
    return get_cell
