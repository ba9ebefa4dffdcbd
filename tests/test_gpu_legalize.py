"""The device legaliser against the host legaliser and the oracle's
brute-force scan: identical bindings, identical FP64 displacement (bit for
bit) and the identical integer HPWL, on uniform, piled, tied (k + 1/2),
off-grid and over-full inputs, with and without macros, with the free map in
shared memory and in global memory; and whole runs with the device
legaliser equal to runs with the host legaliser."""

import numpy as np
import pytest

import eisenjoch_b200 as E
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

CASES = {
    "unit_128": E.SynthSpec(seed=1, num_cells=5000, num_nets=5500, num_pads=400, width=128, height=128,
                            bins_x=128, bins_y=128, cluster_size=32),
    "macro_256_bins128": E.SynthSpec(seed=5, num_cells=12000, num_nets=13200, num_pads=600, width=256, height=256,
                                     bins_x=128, bins_y=128, cluster_size=64, macro_fraction=0.05),
    "odd_90x60": E.SynthSpec(seed=7, num_cells=1500, num_nets=1650, num_pads=100, width=90, height=60,
                             cluster_size=32),
    # 1280 x 1280: the free map (215 KB) lives in global memory
    "global_map_1280": E.SynthSpec(seed=8, num_cells=40000, num_nets=44000, num_pads=800, width=1280, height=1280,
                                   bins_x=256, bins_y=256, cluster_size=64, macro_fraction=0.02),
}


@pytest.fixture(scope="module", params=sorted(CASES))
def case(request):
    nl, chip = E.synth_netlist(CASES[request.param])
    ctx = E.PlacementContext(nl, chip)
    yield request.param, nl, chip, ctx
    ctx.close()


def layouts(nl, chip, seed):
    """Uniform, piled (a few tight clusters: long searches), and positions
    on half-integers (ties between two or four nearest sites)."""
    rng = np.random.default_rng(seed)
    n, W, H = nl.num_cells, chip.width, chip.height
    out = {}
    out["uniform"] = (rng.uniform(0, W - 1, n), rng.uniform(0, H - 1, n))
    k = rng.integers(0, 4, n)
    cx, cy = rng.uniform(0.2, 0.8, 4) * (W - 1), rng.uniform(0.2, 0.8, 4) * (H - 1)
    out["piled"] = (cx[k] + rng.normal(0, W * 0.01, n), cy[k] + rng.normal(0, H * 0.01, n))
    out["half"] = (np.floor(rng.uniform(0, W - 1, n)) + 0.5 * rng.integers(0, 2, n),
                   np.floor(rng.uniform(0, H - 1, n)) + 0.5 * rng.integers(0, 2, n))
    res = {}
    for name, (x, y) in out.items():
        res[name] = (np.clip(x, 0, W - 1).astype(np.float32), np.clip(y, 0, H - 1).astype(np.float32))
    return res


def test_device_legalizer_matches_host(case):
    name, nl, chip, ctx = case
    for lname, (x, y) in layouts(nl, chip, 23).items():
        hx, hy, hd = ctx.legalize(x, y)
        dx, dy, dd, dh = ctx.legalize_device(x, y)
        assert np.array_equal(dx, hx) and np.array_equal(dy, hy), (name, lname)
        assert dd == hd, (name, lname, dd, hd)
        assert dh == E.hpwl_host(nl, chip, hx, hy), (name, lname)


def test_device_legalizer_matches_oracle_scan():
    """Against the oracle's exhaustive scan (the reference's loop as written)."""
    nl, chip = E.synth_netlist(CASES["odd_90x60"])
    ctx = E.PlacementContext(nl, chip)
    orc = Oracle(nl, chip)
    try:
        for lname, (x, y) in layouts(nl, chip, 31).items():
            dx, dy, dd, dh = ctx.legalize_device(x, y)
            st, ox, oy, od = orc.legalize(x, y, 0)
            assert st == 0
            assert np.array_equal(dx, ox) and np.array_equal(dy, oy), lname
            assert dd == od, lname
            assert dh == orc.hpwl(dx, dy)
    finally:
        ctx.close()


def test_device_legalizer_off_grid_positions():
    """Unclamped inputs (outside [0, W-1]) skip the nearest-point shortcut
    and are searched from the clamped row, as on the host."""
    nl, chip = E.synth_netlist(CASES["odd_90x60"])
    ctx = E.PlacementContext(nl, chip)
    try:
        rng = np.random.default_rng(5)
        n = nl.num_cells
        x = rng.uniform(-20, chip.width + 20, n).astype(np.float32)
        y = rng.uniform(-20, chip.height + 20, n).astype(np.float32)
        hx, hy, hd = ctx.legalize(x, y)
        dx, dy, dd, _ = ctx.legalize_device(x, y)
        assert np.array_equal(dx, hx) and np.array_equal(dy, hy)
        assert dd == hd
    finally:
        ctx.close()


def test_device_legalizer_full_chip():
    """Exactly as many cells as sites: every site is used; one more cell
    than sites: NoBelsAvailable, as on the host."""
    W = H = 24
    n = W * H
    nl = E.Netlist(num_cells=n, net_offsets=np.array([0, 2], np.uint32), pin_cell=np.array([0, 1], np.uint32))
    chip = E.Chip(W, H)
    ctx = E.PlacementContext(nl, chip)
    try:
        rng = np.random.default_rng(9)
        x = np.full(n, 11.3, np.float32) + rng.normal(0, 1, n).astype(np.float32)
        y = np.full(n, 12.6, np.float32) + rng.normal(0, 1, n).astype(np.float32)
        hx, hy, hd = ctx.legalize(x, y)
        dx, dy, dd, _ = ctx.legalize_device(x, y)
        assert np.array_equal(dx, hx) and np.array_equal(dy, hy) and dd == hd
        assert len(np.unique(dy * W + dx)) == n
    finally:
        ctx.close()
    nl2 = E.Netlist(num_cells=n + 1, net_offsets=np.array([0, 2], np.uint32), pin_cell=np.array([0, 1], np.uint32))
    ctx2 = E.PlacementContext(nl2, chip)
    try:
        x = np.full(n + 1, 3.0, np.float32)
        with pytest.raises(E.NoBelsAvailable):
            ctx2.legalize(x, x)
        with pytest.raises(E.NoBelsAvailable):
            ctx2.legalize_device(x, x)
    finally:
        ctx2.close()


@pytest.mark.parametrize("field_mode", [1, 0])
def test_run_with_device_legalizer_equals_host(field_mode):
    nl, chip, cfg = E.workload("electro_5k_128")
    if field_mode == 0:
        cfg.max_iters = 60
    a = E.place_electro(nl, chip, cfg, E.RunOptions(field_mode=field_mode, legal_mode=0))
    b = E.place_electro(nl, chip, cfg, E.RunOptions(field_mode=field_mode, legal_mode=1))
    assert a.hpwl == b.hpwl and a.best_iter == b.best_iter and a.iters == b.iters
    assert np.array_equal(a.bel_tile, b.bel_tile)
    assert np.array_equal(a.x, b.x) and np.array_equal(a.y, b.y)
    assert a.trajectory == b.trajectory


def test_run_with_device_legalizer_macros():
    nl, chip = E.synth_netlist(CASES["macro_256_bins128"])
    cfg = E.ElectroPlaceCfg(max_iters=80)
    a = E.place_electro(nl, chip, cfg, E.RunOptions(field_mode=1, legal_mode=0))
    b = E.place_electro(nl, chip, cfg, E.RunOptions(field_mode=1, legal_mode=1))
    assert a.hpwl == b.hpwl and a.best_iter == b.best_iter
    assert np.array_equal(a.bel_tile, b.bel_tile)
    assert a.trajectory == b.trajectory


def test_device_legalizer_bench_geometry():
    """The benchmark job's geometry (200k cells, 5 % macros, 1024^2 sites)
    with the cells drawn into one central pile, as in the crowded middle of
    a run (many cells end up ~200 sites from their target, in long chains
    of cells that depend on each other): the device legaliser's bindings,
    displacement and HPWL equal the host legaliser's bit for bit."""
    nl, chip, _ = E.workload("electro_200k_1024")
    rng = np.random.default_rng(41)
    n, W = nl.num_cells, chip.width
    x = np.clip(rng.normal(W / 2, W * 0.13, n), 0, W - 1).astype(np.float32)
    y = np.clip(rng.normal(W / 2, W * 0.13, n), 0, W - 1).astype(np.float32)
    with E.PlacementContext(nl, chip) as ctx:
        hx, hy, hd = ctx.legalize(x, y)
        dx, dy, dd, dh = ctx.legalize_device(x, y)
    assert np.array_equal(dx, hx) and np.array_equal(dy, hy)
    assert dd == hd
    assert dh == E.hpwl_host(nl, chip, hx, hy)
