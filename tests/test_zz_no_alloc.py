"""The allocation-free density entry point (eplace_density_noalloc).

It exists for callers that cannot call cudaMalloc (graph-capture code,
real-time loops, applications whose device memory another component owns):
they pass device buffers they already own and the library uses a fixed
array of its own as working memory.  This test gives it device buffers
(allocated here, by the test, with torch) and checks its density map and
overlap against the regular density entry point, on two calls in a row --
the second call proves the shared working array is cleared between calls.
The file is named so that pytest collects it last.
"""

import ctypes

import numpy as np
import pytest

import eisenjoch_b200 as E
from eisenjoch_b200 import _abi
from tests.conftest import rel_err

pytestmark = pytest.mark.gpu


def _positions(nl, chip, seed):
    rng = np.random.default_rng(seed)
    n = nl.num_cells
    cx = rng.uniform(0.3, 0.7, 6) * (chip.width - 1)
    cy = rng.uniform(0.3, 0.7, 6) * (chip.height - 1)
    k = rng.integers(0, 6, n)
    x = np.clip(cx[k] + rng.normal(0, chip.width * 0.05, n), 0, chip.width - 1).astype(np.float32)
    y = np.clip(cy[k] + rng.normal(0, chip.height * 0.05, n), 0, chip.height - 1).astype(np.float32)
    return x, y


def test_density_noalloc_matches_density_stage():
    import torch

    nl, chip = E.synth_netlist(E.SynthSpec(seed=5, num_cells=12000, num_nets=13200, num_pads=600, width=256,
                                           height=256, bins_x=128, bins_y=128, cluster_size=64,
                                           macro_fraction=0.05))
    L = _abi.lib()
    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    half = np.stack([nl.cell_w.astype(np.float32) * 0.5, nl.cell_h.astype(np.float32) * 0.5], axis=1)
    half_d = torch.from_numpy(np.ascontiguousarray(half)).to(dev)
    dens_d = torch.zeros((chip.bins_y, chip.bins_x), dtype=torch.float64, device=dev)
    ov_d = torch.zeros(1, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    with E.PlacementContext(nl, chip) as ctx:
        for call, seed in enumerate((31, 32)):
            x, y = _positions(nl, chip, seed)
            ref_d, ref_ov = ctx.density(x, y)
            pos_d = torch.from_numpy(np.ascontiguousarray(np.stack([x, y], axis=1))).to(dev)
            st = L.eplace_density_noalloc(
                ctypes.c_void_p(pos_d.data_ptr()), ctypes.c_void_p(half_d.data_ptr()), nl.num_cells, chip.width,
                chip.height, chip.bins_x, chip.bins_y, ctypes.c_void_p(dens_d.data_ptr()),
                ctypes.c_void_p(ov_d.data_ptr()), ctypes.c_void_p(stream.cuda_stream))
            assert st == _abi.EPLACE_OK, (call, st)
            torch.cuda.synchronize(dev)
            got = dens_d.cpu().numpy()
            # same tolerances as the density parity tests
            assert rel_err(got, ref_d) <= 1e-5, call
            assert abs(float(ov_d.item()) - ref_ov) <= 1e-6, call


def test_density_noalloc_rejects_oversized_grid():
    L = _abi.lib()
    st = L.eplace_density_noalloc(None, None, 0, 1024, 1024, 1024, 1024, ctypes.c_void_p(8), ctypes.c_void_p(8),
                                  None)
    assert st == _abi.EPLACE_ERR_INVALID
