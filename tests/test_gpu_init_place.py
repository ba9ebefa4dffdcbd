"""The device initial placement (csrc/init_place.cu) against the host form
(eplace_initial_placement_host, itself pinned to the oracle and the
reference's generator): the same BEL for every cell, bit for bit, on grids
with and without sites taken by fixed cells, a full chip, the benchmark
workload's million-site grid, a pre-bound cell (host form) and a problem with
too few BELs (placer/common.rs:27-117, context/rng.rs:19-61)."""

import numpy as np
import pytest

import eisenjoch_b200 as E

pytestmark = pytest.mark.gpu


def small_netlist(n, w, h, rng, fixed=0, on_logic=0.0):
    fx = rng.integers(0, w, fixed).astype(np.int32)
    fy = rng.integers(0, h, fixed).astype(np.int32)
    fl = (rng.random(fixed) < on_logic).astype(np.uint8)
    pins = np.array([0, 1] if n > 1 else [0, 0], np.uint32)
    return E.Netlist(num_cells=n, net_offsets=np.array([0, 2], np.uint32), pin_cell=pins, fixed_x=fx,
                     fixed_y=fy, fixed_on_logic=fl if fixed else None)


@pytest.mark.parametrize("n,w,h,fixed,seed", [
    (1, 1, 1, 0, 1),            # one site, one cell: no swap
    (2, 2, 1, 0, 7),
    (300, 24, 20, 0, 0),        # seed 0 runs as 1, as the reference's seed.max(1)
    (300, 24, 20, 40, 12345),   # sites taken by fixed cells
    (1024, 32, 32, 0, 99),      # full chip
    (5000, 128, 128, 400, 1),   # the 5k workload's shape with pads
    (4000, 97, 61, 30, 2 ** 63 + 5),
])
def test_device_initial_placement_equals_host(n, w, h, fixed, seed):
    rng = np.random.default_rng(n + fixed)
    nl = small_netlist(n, w, h, rng, fixed, on_logic=0.5)
    chip = E.Chip(w, h)
    hx, hy = E.initial_placement_host(nl, chip, seed)
    with E.PlacementContext(nl, chip) as ctx:
        for _ in range(2):  # a second call on the same context reuses the scratch
            dx, dy, dev = ctx.initial_placement(seed)
            assert dev
            assert np.array_equal(dx, hx) and np.array_equal(dy, hy)


def test_device_initial_placement_benchmark_grid():
    """The 200k-cell workload: a million-site shuffle."""
    nl, chip, cfg = E.workload("electro_200k_1024")
    hx, hy = E.initial_placement_host(nl, chip, cfg.seed)
    with E.PlacementContext(nl, chip) as ctx:
        dx, dy, dev = ctx.initial_placement(cfg.seed)
    assert dev
    assert np.array_equal(dx, hx) and np.array_equal(dy, hy)
    assert len(np.unique(dy.astype(np.int64) * chip.width + dx)) == nl.num_cells


def test_prebound_cell_takes_host_form():
    rng = np.random.default_rng(3)
    nl = small_netlist(200, 20, 20, rng)
    nl.cell_init_x = np.full(200, -1, np.int32)
    nl.cell_init_y = np.full(200, -1, np.int32)
    nl.cell_init_x[5], nl.cell_init_y[5] = 3, 4
    chip = E.Chip(20, 20)
    hx, hy = E.initial_placement_host(nl, chip, 11)
    with E.PlacementContext(nl, chip) as ctx:
        dx, dy, dev = ctx.initial_placement(11)
    assert not dev
    assert np.array_equal(dx, hx) and np.array_equal(dy, hy) and (dx[5], dy[5]) == (3, 4)


def test_too_few_bels():
    nl = E.Netlist(num_cells=100, net_offsets=np.array([0, 2], np.uint32), pin_cell=np.array([0, 1], np.uint32),
                   fixed_x=np.array([1, 2, 3], np.int32), fixed_y=np.array([1, 1, 1], np.int32),
                   fixed_on_logic=np.ones(3, np.uint8))  # 97 free sites for 100 cells
    chip = E.Chip(10, 10)
    with pytest.raises(E.NoBelsAvailable):
        E.initial_placement_host(nl, chip, 1)
    with E.PlacementContext(nl, chip) as ctx:
        with pytest.raises(E.NoBelsAvailable):
            ctx.initial_placement(1)
