"""CPU tests of the FP64 oracle: pinned against the golden fixtures
(tests/golden, generated from scipy and independent Python restatements)
and against the reference's own unit tests, ported."""

import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests.conftest import star_netlist

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


# --- transforms: rustdct conventions = scipy / 2 ---------------------------
@pytest.mark.parametrize("backend", [0, 1])
def test_transforms_match_golden(backend):
    g = np.load(os.path.join(GOLDEN, "transforms.npz"))
    for n in (1, 2, 3, 4, 5, 8, 16, 31, 64, 128, 512):
        x = g["x_%d" % n]
        for name, fn in (("dct2", O.dct2), ("dct3", O.dct3), ("dst3", O.dst3)):
            ref = g["%s_%d" % (name, n)] / 2.0
            got = fn(x, backend)
            assert np.abs(got - ref).max() <= 1e-11 * max(1.0, np.abs(ref).max()), (name, n, backend)


def test_transform_backends_agree():
    rng = np.random.default_rng(0)
    for n in (2, 8, 64, 256, 1024):
        x = rng.standard_normal(n)
        for fn in (O.dct2, O.dct3, O.dst3):
            assert np.abs(fn(x, 0) - fn(x, 1)).max() <= 1e-12 * n


def test_dct3_inverts_scaled_dct2():
    # DCT-III(DCT-II(x)) = (N/2) x for rustdct's unnormalised pair
    x = np.random.default_rng(1).standard_normal(64)
    assert np.allclose(O.dct3(O.dct2(x)), 32 * x, atol=1e-10)


# --- RNG (context/rng.rs) ----------------------------------------------------
def test_rng_matches_golden():
    with open(os.path.join(GOLDEN, "rng.json")) as f:
        g = json.load(f)
    for seed, seq in g["seeds"].items():
        assert [str(v) for v in O.rng_sequence(int(seed), 8)] == seq
    assert list(O.rng_shuffle(7, range(10))) == g["shuffle_seed_7_range_10"]
    assert list(O.rng_shuffle(1, range(33))) == g["shuffle_seed_1_range_33"]


# --- WA (solver/wa.rs tests :120-230) --------------------------------------
def test_wa_golden_values_and_gradients():
    with open(os.path.join(GOLDEN, "wa.json")) as f:
        cases = json.load(f)
    for c in cases:
        assert abs(O.wa_axis_value(c["coords"], c["coeff"]) - c["value"]) <= 1e-12
        assert np.allclose(O.wa_axis_grad(c["coords"], c["coeff"]), c["grad"], atol=1e-12)


def test_wa_two_points_approximates_hpwl():  # wa.rs:120-137
    wl = O.wa_wirelength([(0.0, 0.0), (3.0, 4.0)], 0.5)
    assert 0.0 < wl < 8.0
    assert abs(O.wa_wirelength([(0.0, 0.0), (3.0, 4.0)], 5.0) - 7.0) < 1.0


def test_wa_single_and_empty():  # wa.rs:139-147
    assert O.wa_wirelength([(1.0, 2.0)], 0.5) == 0.0
    assert O.wa_wirelength(np.zeros((0, 2)), 0.5) == 0.0


def test_wa_gradient_finite_differences():  # wa.rs:150-173
    coords = [1.0, 4.0, 2.0, 6.0]
    g = O.wa_axis_grad(coords, 0.5)
    for i in range(4):
        cp, cm = list(coords), list(coords)
        cp[i] += 1e-6
        cm[i] -= 1e-6
        fd = (O.wa_axis_value(cp, 0.5) - O.wa_axis_value(cm, 0.5)) / 2e-6
        assert abs(fd - g[i]) < 1e-4


def test_wa_gradient_2d_finite_differences():  # wa.rs:175-215
    pos = [(1.0, 2.0), (4.0, 1.0), (2.0, 5.0)]
    gx = O.wa_axis_grad([p[0] for p in pos], 0.5)
    gy = O.wa_axis_grad([p[1] for p in pos], 0.5)
    for i in range(3):
        for ax in range(2):
            pp = [list(p) for p in pos]
            pm = [list(p) for p in pos]
            pp[i][ax] += 1e-6
            pm[i][ax] -= 1e-6
            fd = (O.wa_wirelength(pp, 0.5) - O.wa_wirelength(pm, 0.5)) / 2e-6
            assert abs(fd - (gx if ax == 0 else gy)[i]) < 1e-4


def test_wa_higher_coeff_is_sharper():  # wa.rs:217-230
    pos = [(0.0, 0.0), (5.0, 0.0), (2.0, 3.0)]
    lo, hi = O.wa_wirelength(pos, 0.1), O.wa_wirelength(pos, 2.0)
    assert abs(hi - 8.0) <= abs(lo - 8.0) + 0.5


# --- NesterovSolver (solver/nesterov.rs tests :231-400) ---------------------
def test_nesterov_quadratic():
    s = O.NesterovSolver(2, 0.1)
    s.set_positions([5.0, 3.0])
    for _ in range(500):
        y = s.look_ahead()
        s.step(y)
    assert np.abs(s.positions()).max() < 1e-3


def test_nesterov_faster_than_gd():
    n, iters, step = 10, 50, 0.05
    init = np.arange(1, n + 1, dtype=float)
    s = O.NesterovSolver(n, step)
    s.set_positions(init)
    for _ in range(iters):
        s.step(s.look_ahead())
    gd = init.copy()
    for _ in range(iters):
        gd = gd - step * gd
    assert (s.positions() ** 2).sum() < (gd ** 2).sum()


def test_nesterov_adaptive_restart():
    s = O.NesterovSolver(2, 0.1)
    s.set_positions([1.0, 1.0])
    s.step([0.1, 0.1])
    assert s.iter_count > 0 and s.fista_param > 1.0
    disp = s.positions() - s.x_prev
    s.adaptive_restart(disp)
    assert s.iter_count == 0 and abs(s.fista_param - 1.0) < 1e-10


def test_nesterov_rosenbrock():
    s = O.NesterovSolver(2, 1e-4)
    s.set_positions([-1.0, 1.0])
    for _ in range(50000):
        x0, x1 = s.look_ahead()
        g = [-2.0 * (1.0 - x0) - 400.0 * x0 * (x1 - x0 * x0), 200.0 * (x1 - x0 * x0)]
        s.adaptive_restart(g)
        s.step(g)
    p = s.positions()
    assert abs(p[0] - 1.0) < 0.2 and abs(p[1] - 1.0) < 0.2


def test_nesterov_bb_and_lipschitz():
    s = O.NesterovSolver(2, 0.1)
    s.set_positions([2.0, 3.0])
    s.step([2.0, 3.0])
    cur = s.positions()
    assert s.bb_step_size([2.0, 3.0], cur) > 0.0
    assert s.lipschitz_step_size([2.0, 3.0], cur) > 0.0
    s2 = O.NesterovSolver(2, 0.1)
    s2.set_positions([1.0, 2.0])
    s2.step([0.5, 0.5])
    assert abs(s2.lipschitz_step_size([1.0, 1.0], [1.0, 1.0]) - 0.1) < 1e-10
    assert s2.bb_step_size([1.0, 1.0], [1.0, 1.0]) is None


def test_nesterov_fista_grows():
    s = O.NesterovSolver(2, 0.1)
    s.set_positions([1.0, 1.0])
    prev = s.fista_param
    for _ in range(10):
        s.step([0.1, 0.1])
        assert s.fista_param > prev
        prev = s.fista_param


# --- density / overlap / field (density.rs tests :284-350) ------------------
def _cells(xs, ys, w=8, h=8):
    from eisenjoch_b200 import Chip, Netlist

    n = len(xs)
    nl = Netlist(num_cells=n, net_offsets=np.array([0], np.uint32), pin_cell=np.zeros(0, np.uint32))
    return O.Oracle(nl, Chip(w, h)), np.asarray(xs, float), np.asarray(ys, float)


def test_overlap_kat():
    assert O.overlap_of([4.0, 0.0, 0.0, 0.0]) == 0.75
    assert O.overlap_of([0.0, 0.0]) == 0.0


def test_density_map_single_cell():
    o, x, y = _cells([4.0], [4.0])
    d = o.density(x, y)
    assert d[4, 4] > 0.0 and abs(d.sum() - 1.0) < 1e-12
    # footprint [3.5, 4.5]^2 straddles four bins equally
    assert np.allclose(d[3:5, 3:5], 0.25)


def test_overlap_spread_and_clustered():
    o, x, y = _cells([1.0, 3.0, 5.0, 7.0], [1.0, 3.0, 5.0, 7.0])
    assert o.overlap(o.density(x, y)) < 0.01
    o, x, y = _cells([4.5] * 8, [4.5] * 8)
    d = o.density(x, y)
    assert d[4, 4] == 8.0 and o.overlap(d) > 0.0


def test_field_and_gradient_finite():
    o, x, y = _cells([2.0, 6.0, 4.0], [2.0, 6.0, 4.0])
    ex, ey = o.field(o.density(x, y), 1.0)
    assert np.isfinite(ex).all() and np.isfinite(ey).all()
    gx, gy = o.gather(x, y, ex, ey)
    assert np.isfinite(gx).all() and np.isfinite(gy).all()


def test_uniform_density_gives_zero_field():
    d = np.full((16, 16), 0.7)
    o, _, _ = _cells([0.0], [0.0], 16, 16)
    for mode in (0, 1):
        ex, ey = o.field(d, 1.0, field_mode=mode)
        assert np.abs(ex).max() < 1e-12 and np.abs(ey).max() < 1e-12


def test_target_density_has_no_effect():
    rng = np.random.default_rng(3)
    d = rng.uniform(0, 2, (16, 16))
    o, _, _ = _cells([0.0], [0.0], 16, 16)
    a = o.field(d, 1.0)
    b = o.field(d, 0.3)
    assert np.abs(a[0] - b[0]).max() < 1e-12 and np.abs(a[1] - b[1]).max() < 1e-12


def test_potential_gradient_mode_is_derivative_of_potential():
    """Extension mode: Ex equals d(phi)/dx of the DCT-III synthesis of
    phi_hat, checked against a central difference of that synthesis
    evaluated off the bin centres."""
    W = H = 32
    rng = np.random.default_rng(4)
    d = rng.uniform(0, 2, (H, W))
    o, _, _ = _cells([0.0], [0.0], W, H)
    ex, ey, phi = o.field(d, 1.0, want_phi=True, field_mode=1)

    def synth(xc, yc):
        kx = np.arange(W)
        ky = np.arange(H)
        cx = np.cos(np.pi * kx * (xc + 0.5) / W) * np.where(kx == 0, 0.5, 1.0)
        cy = np.cos(np.pi * ky * (yc + 0.5) / H) * np.where(ky == 0, 0.5, 1.0)
        return cy @ phi @ cx

    h = 1e-5
    for (xi, yi) in [(3, 5), (17, 2), (30, 29)]:
        dx = (synth(xi + h, yi) - synth(xi - h, yi)) / (2 * h)
        dy = (synth(xi, yi + h) - synth(xi, yi - h)) / (2 * h)
        assert abs(ex[yi, xi] - dx) < 1e-6 * max(1, abs(dx))
        assert abs(ey[yi, xi] - dy) < 1e-6 * max(1, abs(dy))


# --- legaliser and HPWL -----------------------------------------------------
def _synth(seed, n, w, macro=0.0, pads=10):
    import eisenjoch_b200 as E

    return E.synth_netlist(E.SynthSpec(seed=seed, num_cells=n, num_nets=int(1.1 * n), num_pads=pads, width=w,
                                       height=w, cluster_size=16, macro_fraction=macro))


@pytest.mark.parametrize("macro", [0.0, 0.05])
def test_ring_legaliser_equals_exhaustive_scan(macro):
    nl, chip = _synth(11, 300, 32, macro)
    o = O.Oracle(nl, chip)
    rng = np.random.default_rng(5)
    for trial in range(12):
        if trial % 3 == 0:  # exact half-integer ties
            x = rng.integers(0, 62, nl.num_cells) / 2.0
            y = rng.integers(0, 62, nl.num_cells) / 2.0
        elif trial % 3 == 1:  # a pile
            x = np.clip(rng.normal(20, 2, nl.num_cells), 0, 31)
            y = np.clip(rng.normal(8, 2, nl.num_cells), 0, 31)
        else:
            x = rng.uniform(0, 31, nl.num_cells)
            y = rng.uniform(0, 31, nl.num_cells)
        a = o.legalize(x, y, 0)
        b = o.legalize(x, y, 1)
        assert a[0] == b[0] == 0
        assert np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2]) and a[3] == b[3]


def test_hpwl_reference_kats():  # tests/metrics_tests.rs:343-381
    from eisenjoch_b200 import Chip, Netlist

    # two cells on one net at (0,0) and (1,1): HPWL = 2
    nl = Netlist(num_cells=2, net_offsets=np.array([0, 2], np.uint32), pin_cell=np.array([0, 1], np.uint32))
    o = O.Oracle(nl, Chip(2, 2))
    assert o.hpwl(np.array([0, 1]), np.array([0, 1])) == 2
    # three cells at tiles 0, 1, 3: one net, total = that net
    nl3 = Netlist(num_cells=3, net_offsets=np.array([0, 3], np.uint32), pin_cell=np.arange(3, dtype=np.uint32))
    assert O.Oracle(nl3, Chip(2, 2)).hpwl(np.array([0, 1, 1]), np.array([0, 0, 1])) == 2
    # a net without a driver contributes nothing
    nd = Netlist(num_cells=2, net_offsets=np.array([0, 2], np.uint32), pin_cell=np.array([0, 1], np.uint32),
                 net_has_driver=np.array([0], np.uint8))
    assert O.Oracle(nd, Chip(2, 2)).hpwl(np.array([0, 1]), np.array([0, 1])) == 0


def test_initial_placement_is_shuffled_free_bels():
    """initial_placement: the free logic BELs in tile order, shuffled once
    with the reference RNG, handed out in cell order."""
    nl, chip = _synth(12, 50, 16)
    st, sx, sy = O.Oracle(nl, chip).initial_placement(99)
    assert st == 0
    avail = O.rng_shuffle(99, range(16 * 16))
    assert np.array_equal(sy * 16 + sx, avail[:50])


# --- the reference's electro tests on the oracle (tests/electro_place_tests.rs)
class _Cfg:
    def __init__(self, **kw):
        d = dict(seed=1, wl_coeff=0.5, target_util=0.7, timing_driven=0, target_density=1.0, timing_weight=0.0,
                 nesterov_step_size=0.1, max_iters=500, legalize_interval=5)
        d.update(kw)
        self.__dict__.update(d)


@pytest.mark.parametrize("n,seed,iters", [(2, 42, 10), (4, 123, 10), (1, 1, 5)])
def test_oracle_places_small_designs(n, seed, iters):
    nl, chip = star_netlist(n)
    st, r = O.Oracle(nl, chip).place(_Cfg(seed=seed, max_iters=iters, legalize_interval=2))
    assert st == 0
    tiles = r["site_y"] * 2 + r["site_x"]
    assert len(np.unique(tiles)) == n


def test_oracle_deterministic_and_empty():
    nl, chip = star_netlist(3)
    cfg = _Cfg(seed=99, max_iters=10, legalize_interval=2)
    a = O.Oracle(nl, chip).place(cfg)[1]
    b = O.Oracle(nl, chip).place(cfg)[1]
    assert np.array_equal(a["site_x"], b["site_x"]) and np.array_equal(a["site_y"], b["site_y"])
    nl0, chip0 = star_netlist(0)
    st, r = O.Oracle(nl0, chip0).place(_Cfg())
    assert st == 0 and r["iters"] == 0


def test_oracle_rejects_zero_interval():
    nl, chip = star_netlist(2)
    st, _ = O.Oracle(nl, chip).place(_Cfg(legalize_interval=0))
    assert st == 4


def test_oracle_no_bels():
    from eisenjoch_b200 import Netlist

    nl = Netlist(num_cells=5, net_offsets=np.array([0, 5], np.uint32), pin_cell=np.arange(5, dtype=np.uint32))
    _, chip = star_netlist(2)
    st, _ = O.Oracle(nl, chip).place(_Cfg(max_iters=3))
    assert st == 1


def test_job_summaries_fixture():
    """The committed oracle job records: the reference field does not
    converge on the 5k workload; the potential-gradient field does."""
    with open(os.path.join(GOLDEN, "job_summaries.json")) as f:
        d = json.load(f)
    assert not d["electro_5k_128:reference_field"]["converged"]
    assert d["electro_5k_128"]["converged"] and d["electro_200k_1024"]["converged"]


def test_stable_wa_shift_equals_reference_where_finite():
    """The oracle's overflow-free WA shift (per-net max / min, the shift the
    CUDA kernel uses) gives the reference's gradient wherever the reference's
    mean shift (wa.rs:58) stays finite, and stays finite where it does not."""
    rng = np.random.default_rng(3)
    n, w = 400, 64
    off = np.cumsum([0] + [int(d) for d in rng.integers(2, 30, 60)]).astype(np.uint32)
    pins = rng.integers(0, n, int(off[-1])).astype(np.uint32)
    nl = O.FlatNetlist(n, off, pins, np.zeros(0, np.int32), np.zeros(0, np.int32))
    orc = O.Oracle(nl, O.FlatChip(w, w))
    x, y = rng.uniform(0, w - 1, n), rng.uniform(0, w - 1, n)
    for coeff in (0.1, 0.5, 2.0):
        a = orc.wa_gradient(x, y, coeff)
        b = orc.wa_gradient(x, y, coeff, wa_mode=1)
        for ga, gb in zip(a, b):
            assert np.isfinite(ga).all()
            np.testing.assert_allclose(gb, ga, rtol=1e-9, atol=1e-12 * np.abs(ga).max())
    # 2048-site spans: the mean shift overflows FP64, the stable one does not
    x2 = rng.uniform(0, 2047, n)
    ra = orc.wa_gradient(x2, y, 1.0)[0]
    rb = orc.wa_gradient(x2, y, 1.0, wa_mode=1)[0]
    assert not np.isfinite(ra).all() and np.isfinite(rb).all()
    ok = np.isfinite(ra)
    np.testing.assert_allclose(rb[ok], ra[ok], rtol=1e-9, atol=1e-12 * np.abs(ra[ok]).max())
