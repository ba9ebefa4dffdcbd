"""CPU checks of bench.py's own arithmetic: the FP64 field it uses as the
yardstick of the precision report equals the oracle's field solve."""

import numpy as np
import pytest

import bench
from oracle.oracle import FlatChip, FlatNetlist, Oracle
from tests.conftest import rel_err


@pytest.mark.parametrize("field_mode", [0, 1])
@pytest.mark.parametrize("shape", [(48, 64), (32, 32)])
def test_bench_fp64_field_equals_oracle(field_mode, shape):
    H, W = shape
    rng = np.random.default_rng(H + W + field_mode)
    d = rng.gamma(2.0, 0.5, (H, W))
    e = np.zeros(0, np.int32)
    orc = Oracle(FlatNetlist(0, np.zeros(1, np.uint32), np.zeros(0, np.uint32), e, e), FlatChip(W, H))
    rex, rey, rphi = orc.field(d, 1.0, want_phi=True, field_mode=field_mode)
    ex, ey, phi = (t.numpy() for t in bench.field_fp64(d, field_mode))
    assert rel_err(ex, rex) <= 1e-12 and rel_err(ey, rey) <= 1e-12 and rel_err(phi, rphi) <= 1e-12
