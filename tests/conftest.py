import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU and libeplace.so")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Builds liboracle.so (gcc) and libeplace.so (nvcc) if sources changed."""
    from oracle import oracle

    oracle.lib()
    from eisenjoch_b200 import build

    build.build()


def rel_err(a, b):
    """max |a - b| / max |b|: the normwise relative error used by the parity
    tests (elementwise relative error is meaningless where b ~ 0)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    scale = np.abs(b).max() if b.size else 0.0
    if scale == 0.0:
        return float(np.abs(a).max()) if a.size else 0.0
    return float(np.abs(a - b).max() / scale)


def star_netlist(n):
    """The reference's make_context_with_cells(n) (tests/common/mod.rs:90-101)
    flattened: a 2x2 chip with one LUT BEL per tile, n <= 4 cells, cell_0
    driving one net whose users are cells 1..n-1."""
    from eisenjoch_b200 import Chip, Netlist

    if n >= 2:
        off = np.array([0, n], np.uint32)
        pins = np.arange(n, dtype=np.uint32)
    else:
        off = np.array([0], np.uint32)
        pins = np.zeros(0, np.uint32)
    return Netlist(num_cells=n, net_offsets=off, pin_cell=pins), Chip(2, 2)
