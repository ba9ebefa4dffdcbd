"""The allocation-free density entry point (eplace_density_noalloc).

It serves callers that cannot call cudaMalloc: a real-time loop that must
not allocate or wait on the allocator, an application whose device memory is
owned and handed out by another component, code under a fixed device-memory
budget.  They pass device buffers they already own (here the test allocates
them with torch, standing in for such an owner) and the library uses a fixed
array of its own as working memory.

Checked through the C ABI, on two calls in a row each (the second proves the
shared working array is clean between calls):
  * against the regular density entry point: the same map bit for bit (both
    run the same fixed-point scatter), the overlap to 1e-12 relative (its
    FP64 sum may be split over a different number of blocks);
  * against the FP64 oracle: the parity tolerances of the density stage
    (normwise 1e-5, overlap 1e-6 absolute);
  * the 1x1-cell path (half_wh = NULL), an empty design, and the host-side
    rejection of oversized grids and misaligned pointers.
The file is named so that pytest collects it last.
"""

import ctypes

import numpy as np
import pytest

import eisenjoch_b200 as E
from eisenjoch_b200 import _abi
from oracle.oracle import Oracle
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


def _noalloc(torch, nl, chip, x, y, half_d, dens_d, ov_d):
    L = _abi.lib()
    dev = dens_d.device
    pos_d = torch.from_numpy(np.ascontiguousarray(np.stack([x, y], axis=1))).to(dev)
    stream = torch.cuda.current_stream(dev)
    bx, by = chip.bins_x or chip.width, chip.bins_y or chip.height  # 0: one bin per site
    st = L.eplace_density_noalloc(
        ctypes.c_void_p(pos_d.data_ptr() if nl.num_cells else 0),
        ctypes.c_void_p(half_d.data_ptr() if half_d is not None else 0), nl.num_cells, chip.width, chip.height,
        bx, by, ctypes.c_void_p(dens_d.data_ptr()), ctypes.c_void_p(ov_d.data_ptr()),
        ctypes.c_void_p(stream.cuda_stream))
    torch.cuda.synchronize(dev)
    return st, dens_d.cpu().numpy().copy(), float(ov_d.item())


def _check(torch, nl, chip, with_half):
    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    half_d = None
    if with_half:
        half = np.stack([nl.cell_w.astype(np.float32) * 0.5, nl.cell_h.astype(np.float32) * 0.5], axis=1)
        half_d = torch.from_numpy(np.ascontiguousarray(half)).to(dev)
    dens_d = torch.full((chip.bins_y or chip.height, chip.bins_x or chip.width), -1.0, dtype=torch.float64,
                        device=dev)
    ov_d = torch.full((1,), -1.0, dtype=torch.float64, device=dev)
    orc = Oracle(nl, chip)
    with E.PlacementContext(nl, chip) as ctx:
        for call, seed in enumerate((31, 32)):
            x, y = _positions(nl, chip, seed)
            ref_d, ref_ov = ctx.density(x, y)
            st, got, ov = _noalloc(torch, nl, chip, x, y, half_d, dens_d, ov_d)
            assert st == _abi.EPLACE_OK, (call, st)
            assert np.array_equal(got, ref_d), call
            assert abs(ov - ref_ov) <= 1e-12 * max(1.0, abs(ref_ov)), call
            od = orc.density(x, y)
            assert rel_err(got, od) <= 1e-5, call
            assert abs(ov - orc.overlap(od)) <= 1e-6, call


def test_density_noalloc_with_footprints():
    """Macros of 2..8 sites and two sites per bin edge."""
    import torch

    nl, chip = E.synth_netlist(E.SynthSpec(seed=5, num_cells=12000, num_nets=13200, num_pads=600, width=256,
                                           height=256, bins_x=128, bins_y=128, cluster_size=64,
                                           macro_fraction=0.05))
    _check(torch, nl, chip, with_half=True)


def test_density_noalloc_unit_cells():
    """All cells 1x1 and half_wh = NULL: the unit-cell path of the scatter."""
    import torch

    nl, chip = E.synth_netlist(E.SynthSpec(seed=6, num_cells=9000, num_nets=9900, num_pads=300, width=160,
                                           height=120, cluster_size=32))
    assert nl.cell_w is None
    _check(torch, nl, chip, with_half=False)


def test_density_noalloc_empty_design():
    """No cells: a zero map and overlap 0, also right after a call that
    filled the working array."""
    import torch

    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    full, chip = E.synth_netlist(E.SynthSpec(seed=7, num_cells=3000, num_nets=3300, num_pads=100, width=64,
                                             height=64, cluster_size=32))
    empty = E.Netlist(num_cells=0, net_offsets=np.zeros(1, np.uint32), pin_cell=np.zeros(0, np.uint32))
    dens_d = torch.full((64, 64), -1.0, dtype=torch.float64, device=dev)
    ov_d = torch.full((1,), -1.0, dtype=torch.float64, device=dev)
    x, y = _positions(full, chip, 3)
    st, got, _ = _noalloc(torch, full, chip, x, y, None, dens_d, ov_d)
    assert st == _abi.EPLACE_OK and got.sum() > 0
    e = np.zeros(0, np.float32)
    st, got, ov = _noalloc(torch, empty, chip, e, e, None, dens_d, ov_d)
    assert st == _abi.EPLACE_OK
    assert not got.any() and ov == 0.0


def test_density_noalloc_rejects_bad_arguments():
    """Rejected on the host, before anything reaches the device: a grid above
    the 512 x 512 working array, and device pointers that are not 8-byte
    aligned."""
    import torch

    L = _abi.lib()
    st = L.eplace_density_noalloc(None, None, 0, 1024, 1024, 1024, 1024, ctypes.c_void_p(8), ctypes.c_void_p(8),
                                  None)
    assert st == _abi.EPLACE_ERR_INVALID
    dev = torch.device("cuda:0")
    buf = torch.zeros(4096, dtype=torch.float64, device=dev)
    base = buf.data_ptr()
    assert base % 256 == 0
    for pos, half, dens, ov in ((base + 4, 0, base + 2048, base + 3072),
                                (base, base + 4, base + 2048, base + 3072),
                                (base, 0, base + 2052, base + 3072),
                                (base, 0, base + 2048, base + 3076)):
        st = L.eplace_density_noalloc(ctypes.c_void_p(pos), ctypes.c_void_p(half), 8, 64, 64, 16, 16,
                                      ctypes.c_void_p(dens), ctypes.c_void_p(ov), None)
        assert st == _abi.EPLACE_ERR_INVALID, (pos - base, half, dens - base, ov - base)
