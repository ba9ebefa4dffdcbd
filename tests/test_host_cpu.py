"""CPU tests of the product library without a GPU: the C ABI loads and
exports every function include/eplace.h declares, the config defaults,
and the host parts of the path (initial placement, legaliser, HPWL,
generator, the place_cells flattening) against the oracle."""

import ctypes
import os
import re

import numpy as np
import pytest

import eisenjoch_b200 as E
from eisenjoch_b200 import _abi
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    with open(os.path.join(ROOT, "include", "eplace.h")) as f:
        text = f.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(eplace_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_function():
    L = _abi.lib()
    names = header_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(L, n), n
    assert set(names) == set(_abi.PROTOTYPES), set(names) ^ set(_abi.PROTOTYPES)
    assert L.eplace_abi_version() == 1


def test_config_defaults_match_reference():  # tests/electro_place_tests.rs:97-109
    c = _abi.Cfg()
    _abi.lib().eplace_cfg_default(ctypes.byref(c))
    py = E.ElectroPlaceCfg()
    assert (c.seed, c.wl_coeff, c.target_util, c.timing_driven, c.target_density, c.timing_weight,
            c.nesterov_step_size, c.max_iters, c.legalize_interval) == (1, 0.5, 0.7, 0, 1.0, 0.0, 0.1, 500, 5)
    assert (py.seed, py.wl_coeff, py.target_util, py.timing_driven, py.target_density, py.timing_weight,
            py.nesterov_step_size, py.max_iters, py.legalize_interval) == (1, 0.5, 0.7, False, 1.0, 0.0, 0.1, 500, 5)


def test_context_needs_a_device_here():
    nl, chip = E.synth_netlist(E.SynthSpec(seed=1, num_cells=10, num_nets=11, num_pads=2, width=8, height=8))
    with pytest.raises(E.EplaceError) as e:
        E.PlacementContext(nl, chip)
    assert e.value.status == _abi.EPLACE_ERR_NO_DEVICE


# --- generator --------------------------------------------------------------
def test_generator_is_deterministic_and_well_formed():
    spec = E.SynthSpec(seed=3, num_cells=5000, num_nets=5500, num_pads=400, width=128, height=128)
    a, chip = E.synth_netlist(spec)
    b, _ = E.synth_netlist(spec)
    assert np.array_equal(a.pin_cell, b.pin_cell) and np.array_equal(a.net_offsets, b.net_offsets)
    deg = np.diff(a.net_offsets.astype(np.int64))
    # cell pins only (pads are appended users)
    cell_deg = np.array([(a.pin_cell[a.net_offsets[n]:a.net_offsets[n + 1]] < 5000).sum() for n in range(5500)])
    frac2 = (cell_deg == 2).mean()
    assert 0.55 < frac2 < 0.65
    assert ((cell_deg >= 21) & (cell_deg <= 200)).mean() < 0.05
    assert deg.sum() == a.num_pins == cell_deg.sum() + 400
    for n in range(0, 5500, 37):
        cells = a.pin_cell[a.net_offsets[n]:a.net_offsets[n + 1]]
        assert len(np.unique(cells)) == len(cells)
        assert cells[0] < 5000  # the driver is a cell
    # pads on the perimeter walk, all distinct
    on_edge = (a.fixed_x == 0) | (a.fixed_x == 127) | (a.fixed_y == 0) | (a.fixed_y == 127)
    assert on_edge.all() and len(set(zip(a.fixed_x, a.fixed_y))) == 400


def test_generator_macros():
    nl, _ = E.synth_netlist(E.SynthSpec(seed=2, num_cells=20000, num_nets=22000, num_pads=100, width=512,
                                        height=512, bins_x=256, bins_y=256, cluster_size=64, macro_fraction=0.05))
    m = nl.cell_w > 1
    assert 0.04 < m.mean() < 0.06
    assert nl.cell_w[m].min() == 2 and nl.cell_w[m].max() == 8 and (nl.cell_w == nl.cell_h).all()


# --- host parts against the oracle -------------------------------------------
def _case(seed, n, w, macro=0.0, fixed_logic=0):
    nl, chip = E.synth_netlist(E.SynthSpec(seed=seed, num_cells=n, num_nets=int(1.1 * n), num_pads=12, width=w,
                                           height=w, cluster_size=16, macro_fraction=macro))
    if fixed_logic:
        rng = np.random.default_rng(seed)
        tiles = rng.choice(w * w, fixed_logic, replace=False)
        nl.fixed_x = np.concatenate([nl.fixed_x, (tiles % w).astype(np.int32)])
        nl.fixed_y = np.concatenate([nl.fixed_y, (tiles // w).astype(np.int32)])
        nl.fixed_on_logic = np.concatenate([np.zeros(12, np.uint8), np.ones(fixed_logic, np.uint8)])
    return nl, chip


@pytest.mark.parametrize("macro,fixed", [(0.0, 0), (0.05, 0), (0.0, 40), (0.05, 40)])
def test_host_legaliser_equals_reference_scan(macro, fixed):
    nl, chip = _case(21, 220, 32, macro, fixed)
    o = O.Oracle(nl, chip)
    rng = np.random.default_rng(7)
    for trial in range(9):
        if trial % 3 == 0:
            x = (rng.integers(0, 62, nl.num_cells) / 2.0).astype(np.float32)
            y = (rng.integers(0, 62, nl.num_cells) / 2.0).astype(np.float32)
        elif trial % 3 == 1:
            x = np.clip(rng.normal(9, 2.5, nl.num_cells), 0, 31).astype(np.float32)
            y = np.clip(rng.normal(22, 2.5, nl.num_cells), 0, 31).astype(np.float32)
        else:
            x = rng.uniform(0, 31, nl.num_cells).astype(np.float32)
            y = rng.uniform(0, 31, nl.num_cells).astype(np.float32)
        st, ox, oy, od = o.legalize(x, y, 0)
        if st != 0:  # fragmentation left no block for a macro: both must fail alike
            assert st == 1
            with pytest.raises(E.NoBelsAvailable):
                E.placer.legalize_host(nl, chip, x, y)
            continue
        sx, sy, d = E.placer.legalize_host(nl, chip, x, y)
        assert np.array_equal(sx, ox) and np.array_equal(sy, oy) and d == od
        assert E.placer.hpwl_host(nl, chip, sx, sy) == o.hpwl(sx, sy)


@pytest.mark.parametrize("seed", [1, 7, 99])
def test_host_initial_placement_equals_oracle(seed):
    nl, chip = _case(22, 400, 32, 0.05, 30)
    sx, sy = E.placer.initial_placement_host(nl, chip, seed)
    st, ox, oy = O.Oracle(nl, chip).initial_placement(seed)
    assert st == 0 and np.array_equal(sx, ox) and np.array_equal(sy, oy)


def test_host_errors():
    nl, chip = _case(23, 20, 8)
    bad = E.Netlist(num_cells=2, net_offsets=np.array([0, 2], np.uint32), pin_cell=np.array([0, 9], np.uint32))
    with pytest.raises(E.EplaceError):
        E.placer.hpwl_host(bad, chip, np.zeros(2, np.int32), np.zeros(2, np.int32))
    full = E.Netlist(num_cells=70, net_offsets=np.array([0], np.uint32), pin_cell=np.zeros(0, np.uint32))
    with pytest.raises(E.NoBelsAvailable):
        E.placer.initial_placement_host(full, chip, 1)


def test_lock_others_flattening():
    """with_locked_others (placer/common.rs:502-530): bound cells outside the
    set become fixed cells on their logic BELs; pin ids are remapped."""
    nl, chip = _case(24, 30, 8)
    nl.cell_init_x = (np.arange(30) % 8).astype(np.int32)
    nl.cell_init_y = (np.arange(30) // 8).astype(np.int32)
    sub, target = E.lock_others(nl, [3, 5, 11])
    assert sub.num_cells == 3 and sub.num_fixed == nl.num_fixed + 27
    assert (sub.fixed_on_logic[nl.num_fixed:] == 1).all()
    # every pin still names the same physical location
    def loc(n, pid):
        if pid < n.num_cells:
            return (int(n.cell_init_x[pid]), int(n.cell_init_y[pid]))
        f = pid - n.num_cells
        return (int(n.fixed_x[f]), int(n.fixed_y[f]))
    for p in range(nl.num_pins):
        assert loc(nl, nl.pin_cell[p]) == loc(sub, sub.pin_cell[p])


def test_footprint_estimate_grows_with_the_job():
    """The engine's admission estimate (eplace_footprint) is host-only: it
    validates the netlist and grows with cells, pins and bins."""
    small = E.synth_netlist(E.SynthSpec(seed=3, num_cells=1000, num_nets=1100, num_pads=50, width=64, height=64))
    big = E.synth_netlist(E.SynthSpec(seed=3, num_cells=8000, num_nets=8800, num_pads=200, width=128, height=128))
    fs, fb = E.footprint(*small), E.footprint(*big)
    assert 0 < fs < fb
    nl, chip = small
    assert fb - fs > 7000 * 96  # per-cell state at least
    bad = E.Netlist(num_cells=2, net_offsets=np.array([0, 2], np.uint32), pin_cell=np.array([0, 9], np.uint32))
    assert E.footprint(bad, chip) == 0


def test_mixed_job_streams_are_seeded_and_feasible():
    """The batched / served job generators: deterministic, cell counts in
    range, bins a power of two in [64, 512], total footprint of every job
    below 70% of its sites."""
    a, b = E.batched_specs(64), E.batched_specs(64)
    assert a == b and len(a) == 64
    assert all(2000 <= s.num_cells <= 200000 for s in a)
    assert all(s.bins_x in (64, 128, 256, 512) and s.width == 2 * s.bins_x for s in a)
    specs, arr = E.served_stream(50, 40.0)
    assert arr[0] == 0 and np.all(np.diff(arr) >= 0)
    assert all(1000 <= s.num_cells <= 300000 for s in specs)
    for sp in a[:8] + specs[:4]:
        nl, chip = E.synth_netlist(sp)
        area = (nl.cell_w.astype(int) * nl.cell_h.astype(int)).sum()
        assert area < 0.7 * chip.width * chip.height


def test_engine_without_gpu_reports_no_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(E.EplaceError) as ei:
        E.JobServer()
    assert ei.value.status == E._abi.EPLACE_ERR_NO_DEVICE


@pytest.mark.parametrize("spec", [
    E.SynthSpec(seed=1, num_cells=5000, num_nets=5500, num_pads=400, width=128, height=128, cluster_size=32),
    E.SynthSpec(seed=9, num_cells=20000, num_nets=22000, num_pads=300, width=256, height=256, bins_x=128,
                bins_y=128, cluster_size=64, macro_fraction=0.05),
    E.SynthSpec(seed=4, num_cells=3, num_nets=10, num_pads=0, width=4, height=4),
    E.SynthSpec(seed=5, num_cells=0, num_nets=3, num_pads=6, width=8, height=1),
    E.SynthSpec(seed=6, num_cells=700, num_nets=0, num_pads=17, width=40, height=30, cluster_size=7,
                locality=0.9, macro_fraction=0.2, macro_min=3, macro_max=5),
])
def test_oracle_generator_equals_product_generator(spec):
    """The CPU reference arm generates its inputs with the oracle's copy of
    the generator (so it never loads the product library): both copies must
    emit the same netlist bytes."""
    a, ca = E.synth_netlist(spec)
    b, cb = O.synth(spec)
    for k in ("net_offsets", "pin_cell", "fixed_x", "fixed_y", "cell_w", "cell_h"):
        va, vb = getattr(a, k), getattr(b, k)
        assert (va is None) == (vb is None), k
        if va is not None:
            assert va.dtype == vb.dtype and np.array_equal(va, vb), k
    assert (ca.width, ca.height, ca.bins_x, ca.bins_y) == (cb.width, cb.height, cb.bins_x, cb.bins_y)


def test_workload_table_is_plain_data():
    """bench.py's CPU arm reads the workload table as JSON; the product's
    WORKLOADS is built from the same file."""
    import json
    with open(os.path.join(ROOT, "eisenjoch_b200", "workloads.json")) as f:
        table = {k: v for k, v in json.load(f).items() if not k.startswith("_")}
    assert set(table) == set(E.WORKLOADS)
    for name, w in table.items():
        spec = E.WORKLOADS[name]["spec"]
        for k, v in w["spec"].items():
            assert getattr(spec, k) == v, (name, k)
        assert E.WORKLOADS[name]["cfg"] == w["cfg"]


@pytest.mark.parametrize("simd", ["0", "1", "2"])
def test_host_legalizer_dense_pile_equals_oracle(simd, monkeypatch):
    """A central pile (cells up to ~60 sites from their nearest free site,
    long row searches) with 5 % macros: the product's host legaliser equals
    the oracle's ring search (the reference's choice and tie-break) site for
    site, and the FP64 displacement bit for bit, in each of its search forms
    (EPLACE_LEGAL_SIMD: 0 scalar, 1 four rows per step with AVX2, 2 eight
    rows per step with AVX-512 where the CPU has them)."""
    monkeypatch.setenv("EPLACE_LEGAL_SIMD", simd)
    nl, chip = E.synth_netlist(E.SynthSpec(seed=12, num_cells=20000, num_nets=22000, num_pads=300, width=256,
                                           height=256, cluster_size=64, macro_fraction=0.05))
    rng = np.random.default_rng(4)
    n = nl.num_cells
    x = np.clip(rng.normal(128, 28, n), 0, 255).astype(np.float32)
    y = np.clip(rng.normal(128, 28, n), 0, 255).astype(np.float32)
    sx, sy, disp = E.legalize_host(nl, chip, x, y)
    st, ox, oy, odisp = O.Oracle(nl, chip).legalize(x, y, 1)
    assert st == 0
    assert np.array_equal(sx, ox) and np.array_equal(sy, oy)
    assert disp == odisp
    far = (sx - x) ** 2 + (sy - y) ** 2 > 400
    assert far.sum() > 1000  # the pile is real: many long searches


@pytest.mark.parametrize("simd", ["0", "1", "2"])
def test_host_legalizer_ties_equal_oracle(simd, monkeypatch):
    """Targets on the integer and half-integer lattice (ties between sites
    of equal cost everywhere: the nearest-site fast path, the 3 x 3 block
    around it and the row search all break them by lowest tile) in a pile
    with an off-centre second pile near the chip edge, unit cells only."""
    monkeypatch.setenv("EPLACE_LEGAL_SIMD", simd)
    nl, chip = E.synth_netlist(E.SynthSpec(seed=13, num_cells=12000, num_nets=12000, num_pads=100, width=160,
                                           height=160, cluster_size=32))
    rng = np.random.default_rng(5)
    n = nl.num_cells
    centre = np.where(rng.random(n) < 0.7, 80.0, 8.0)
    x = np.clip(np.round(rng.normal(centre, 20, n) * 2) / 2, 0, 159).astype(np.float32)
    y = np.clip(np.round(rng.normal(centre, 20, n) * 2) / 2, 0, 159).astype(np.float32)
    sx, sy, disp = E.legalize_host(nl, chip, x, y)
    st, ox, oy, odisp = O.Oracle(nl, chip).legalize(x, y, 1)
    assert st == 0
    assert np.array_equal(sx, ox) and np.array_equal(sy, oy)
    assert disp == odisp


def test_pin_weights_equal_oracle():
    """compute_pin_weights (placer/common.rs:381-407), the weights the
    optimal-transport placer shares (opt_trans_place/mod.rs:110): per cell
    the sum of 1/degree over its nets of two pins or more, pads excluded,
    a net without a driver counted by its users; bit for bit against the
    oracle, plus a hand-checked case."""
    nl, chip = E.synth_netlist(E.SynthSpec(seed=21, num_cells=3000, num_nets=3300, num_pads=120, width=64,
                                           height=64, cluster_size=32))
    drv = np.ones(nl.num_nets, np.uint8)
    drv[::7] = 0
    nl.net_has_driver = drv
    w = E.pin_weights(nl, chip)
    assert np.array_equal(w, O.Oracle(nl, chip).pin_weights())
    # three cells, one pad (cell 3): nets {0,1}, {0,1,2}, {2,3}, {1}
    small = E.Netlist(num_cells=3, net_offsets=np.array([0, 2, 5, 7, 8], np.uint32),
                      pin_cell=np.array([0, 1, 0, 1, 2, 2, 3, 1], np.uint32),
                      fixed_x=np.array([0], np.int32), fixed_y=np.array([0], np.int32))
    w = E.pin_weights(small, E.Chip(4, 4))
    assert np.array_equal(w, np.array([1 / 2 + 1 / 3, 1 / 2 + 1 / 3, 1 / 3 + 1 / 2]))


def test_host_hpwl_large_netlist_equals_oracle():
    """The HPWL of a netlist of 2^19 pins and more is summed in four pieces
    of the degree table (as a lone job's checkpoints do): the same integer
    as the oracle's net-by-net walk."""
    sp = E.SynthSpec(seed=4, num_cells=80000, num_nets=88000, num_pads=800, width=512, height=512, bins_x=256,
                     bins_y=256, cluster_size=64, macro_fraction=0.05)
    nl, chip = E.synth_netlist(sp)
    assert nl.num_pins >= 1 << 19
    rng = np.random.default_rng(3)
    sx = rng.integers(0, chip.width - 8, nl.num_cells).astype(np.int32)
    sy = rng.integers(0, chip.height - 8, nl.num_cells).astype(np.int32)
    assert E.placer.hpwl_host(nl, chip, sx, sy) == O.Oracle(nl, chip).hpwl(sx, sy)
