"""Parity of every CUDA stage with the FP64 CPU oracle, teacher-forced: the
oracle gets exactly the FP32 inputs the kernel gets (as FP64).

Tolerances (FP32 path, stated per quantity):
  WA gradient, field, potential spectrum: normwise relative error
      max|gpu - oracle| / max|oracle| <= 1e-4
  density map, gathered density gradient: normwise <= 1e-5
  overlap: absolute <= 1e-6
  HPWL, legalised sites: bit-exact
"""

import numpy as np
import pytest

import eisenjoch_b200 as E
from oracle.oracle import Oracle, fista_sequence
from tests.conftest import rel_err, star_netlist

pytestmark = pytest.mark.gpu

CASES = {
    # 5k unit cells on 128^2 sites / bins, 400 pads (reference geometry)
    "unit_128": E.SynthSpec(seed=1, num_cells=5000, num_nets=5500, num_pads=400, width=128, height=128,
                            bins_x=128, bins_y=128, cluster_size=32),
    # macros 2..8 and 2x2 sites per bin (the extension)
    "macro_256_bins128": E.SynthSpec(seed=5, num_cells=12000, num_nets=13200, num_pads=600, width=256, height=256,
                                     bins_x=128, bins_y=128, cluster_size=64, macro_fraction=0.05),
    # odd sizes: non-power-of-two, non-square bin grid (the unfolded FP32 transform)
    "odd_90x60": E.SynthSpec(seed=7, num_cells=1500, num_nets=1650, num_pads=100, width=90, height=60,
                             cluster_size=32),
    # non-square grid with sides multiples of 8 (the folded FP32 transform, K not split)
    "fold_96x48": E.SynthSpec(seed=9, num_cells=2000, num_nets=2200, num_pads=120, width=96, height=48,
                              cluster_size=32),
}


@pytest.fixture(scope="module", params=sorted(CASES))
def case(request):
    nl, chip = E.synth_netlist(CASES[request.param])
    ctx = E.PlacementContext(nl, chip)
    orc = Oracle(nl, chip)
    yield request.param, nl, chip, ctx, orc
    ctx.close()


def positions(nl, chip, seed, clustered=False):
    rng = np.random.default_rng(seed)
    n = nl.num_cells
    if clustered:
        cx = rng.uniform(0.3, 0.7, 8) * (chip.width - 1)
        cy = rng.uniform(0.3, 0.7, 8) * (chip.height - 1)
        k = rng.integers(0, 8, n)
        x = cx[k] + rng.normal(0, chip.width * 0.03, n)
        y = cy[k] + rng.normal(0, chip.height * 0.03, n)
    else:
        x = rng.uniform(0, chip.width - 1, n)
        y = rng.uniform(0, chip.height - 1, n)
    x = np.clip(x, 0, chip.width - 1).astype(np.float32)
    y = np.clip(y, 0, chip.height - 1).astype(np.float32)
    return x, y


@pytest.mark.parametrize("clustered", [False, True])
def test_wa_gradient(case, clustered):
    name, nl, chip, ctx, orc = case
    x, y = positions(nl, chip, 11, clustered)
    gx, gy = ctx.wa_grad(x, y, 0.5)
    rx, ry = orc.wa_gradient(x, y, 0.5)
    assert rel_err(gx, rx) <= 1e-4, name
    assert rel_err(gy, ry) <= 1e-4, name


def test_wa_gradient_sharp_coefficient(case):
    """wl_coeff = 5: the reference shifts exponents by the pin mean
    (wa.rs:58), so exp() overflows to inf -> NaN in FP64 once a pin sits
    more than ~142 sites from its net's mean.  The kernel's max/min shift is
    mathematically identical and stays finite; parity is checked on every
    cell the reference computes, finiteness on the rest."""
    name, nl, chip, ctx, orc = case
    x, y = positions(nl, chip, 12)
    gx, gy = ctx.wa_grad(x, y, 5.0)
    rx, ry = orc.wa_gradient(x, y, 5.0)
    ok = np.isfinite(rx) & np.isfinite(ry)
    assert np.isfinite(gx).all() and np.isfinite(gy).all()
    assert ok.sum() >= 50
    assert rel_err(gx[ok], rx[ok]) <= 1e-4 and rel_err(gy[ok], ry[ok]) <= 1e-4


def test_wa_gradient_where_reference_overflows(case):
    """Positions spread over the whole chip with wl_coeff = 2: nets whose
    pins sit > ~177 sites from their mean overflow in the reference's FP64
    formula.  On the cells the reference computes, parity holds; the kernel
    is finite everywhere."""
    name, nl, chip, ctx, orc = case
    x, y = positions(nl, chip, 19)
    gx, gy = ctx.wa_grad(x, y, 2.0)
    rx, ry = orc.wa_gradient(x, y, 2.0)
    ok = np.isfinite(rx) & np.isfinite(ry)
    assert np.isfinite(gx).all() and np.isfinite(gy).all()
    if ok.any():
        assert rel_err(gx[ok], rx[ok]) <= 1e-4 and rel_err(gy[ok], ry[ok]) <= 1e-4


@pytest.mark.parametrize("clustered", [False, True])
def test_density_and_overlap(case, clustered):
    name, nl, chip, ctx, orc = case
    x, y = positions(nl, chip, 13, clustered)
    d, ov = ctx.density(x, y)
    rd = orc.density(x, y)
    assert rel_err(d, rd) <= 1e-5
    assert abs(ov - orc.overlap(rd)) <= 1e-6
    # mass: every cell's area inside the chip lands in the map
    assert abs(d.sum() - rd.sum()) <= 1e-5 * rd.sum()


@pytest.mark.parametrize("dct_mode", [E._abi.EPLACE_DCT_FP32_SIMT, E._abi.EPLACE_DCT_FP32_FFT])
@pytest.mark.parametrize("clustered", [False, True])
def test_field(case, clustered, dct_mode):
    """Both FP32 transforms (the FFT form falls back to the GEMMs on grids
    that are not powers of two)."""
    name, nl, chip, ctx, orc = case
    x, y = positions(nl, chip, 14, clustered)
    rd = orc.density(x, y)
    ex, ey, phi = ctx.field(rd, want_phi=True, dct_mode=dct_mode)
    rex, rey, rphi = orc.field(rd, 1.0, want_phi=True)
    assert rel_err(ex, rex) <= 1e-4, name
    assert rel_err(ey, rey) <= 1e-4, name
    assert rel_err(phi, rphi) <= 1e-4, name


TC = E._abi.EPLACE_DCT_BF16X3_TC


@pytest.mark.parametrize("field_mode", [0, 1])
def test_field_tensor_core_bf16x3(case, field_mode):
    """The tcgen05 BF16 three-term split GEMMs (FP32 accumulate) against the
    FP64 oracle: normwise relative error <= 1e-4 on field and potential
    spectrum.  Bin grids whose height is not a multiple of 128 are refused."""
    name, nl, chip, ctx, orc = case
    x, y = positions(nl, chip, 21, True)
    rd = orc.density(x, y)
    by, bx = ctx.bins
    if by % 128 or bx % 64:
        with pytest.raises(E.EplaceError):
            ctx.field(rd, dct_mode=TC)
        return
    ex, ey, phi = ctx.field(rd, dct_mode=TC, want_phi=True, field_mode=field_mode)
    rex, rey, rphi = orc.field(rd, 1.0, want_phi=True, field_mode=field_mode)
    assert rel_err(ex, rex) <= 1e-4, (name, rel_err(ex, rex))
    assert rel_err(ey, rey) <= 1e-4, (name, rel_err(ey, rey))
    assert rel_err(phi, rphi) <= 1e-4


def test_field_potential_gradient_mode(case):
    """The opt-in potential-gradient field (extension) against the oracle's
    same mode."""
    name, nl, chip, ctx, orc = case
    x, y = positions(nl, chip, 18, True)
    rd = orc.density(x, y)
    ex, ey = ctx.field(rd, field_mode=E._abi.EPLACE_FIELD_POTENTIAL_GRADIENT)
    rex, rey = orc.field(rd, 1.0, field_mode=1)
    assert rel_err(ex, rex) <= 1e-4 and rel_err(ey, rey) <= 1e-4


def test_gather(case):
    name, nl, chip, ctx, orc = case
    x, y = positions(nl, chip, 15, True)
    rd = orc.density(x, y)
    rex, rey = orc.field(rd, 1.0)
    ex, ey = rex.astype(np.float32), rey.astype(np.float32)
    gx, gy = ctx.gather(x, y, ex, ey)
    ox, oy = orc.gather(x, y, ex, ey)
    assert rel_err(gx, ox) <= 1e-5 and rel_err(gy, oy) <= 1e-5


@pytest.mark.parametrize("it,initialized", [(0, False), (7, True), (60, True), (9, False)])
def test_fused_step(case, it, initialized):
    name, nl, chip, ctx, orc = case
    rng = np.random.default_rng(100 + it)
    n = nl.num_cells
    x, y = positions(nl, chip, 16, True)
    xp = np.clip(x + rng.normal(0, 0.3, n), 0, chip.width - 1).astype(np.float32)
    yp = np.clip(y + rng.normal(0, 0.3, n), 0, chip.height - 1).astype(np.float32)
    a = fista_sequence(it)
    m = 0.0 if it == 0 else (a - 1) / ((1 + np.sqrt(1 + 4 * a * a)) / 2)
    lx = np.clip(x + m * (x.astype(np.float64) - xp), 0, chip.width - 1).astype(np.float32)
    ly = np.clip(y + m * (y.astype(np.float64) - yp), 0, chip.height - 1).astype(np.float32)
    gwx, gwy = orc.wa_gradient(lx, ly, 0.5)
    gwx, gwy = gwx.astype(np.float32), gwy.astype(np.float32)
    rd = orc.density(lx, ly)
    rex, rey = orc.field(rd, 1.0)
    ex, ey = rex.astype(np.float32), rey.astype(np.float32)
    gpx = (rng.normal(0, 0.05, n)).astype(np.float32)
    gpy = (rng.normal(0, 0.05, n)).astype(np.float32)
    lam = 3.7 if initialized else 0.0
    state = dict(x=x.copy(), y=y.copy(), x_prev=xp.copy(), y_prev=yp.copy(), gprev_x=gpx.copy(), gprev_y=gpy.copy())
    scal = [lam, 1.0 if initialized else 0.0, 0.1, 0.2]
    nx, ny, ax, ay, nlx, nly = ctx.step(it, lx, ly, gwx, gwy, ex, ey, state, scal)
    gdx, gdy = orc.gather(lx, ly, ex, ey)
    ostate = dict(x=x, y=y, x_prev=xp, y_prev=yp, gprev_x=gpx, gprev_y=gpy, step_x=0.1, step_y=0.2,
                  density_penalty=lam, initialized=initialized)
    ref, norms = orc.step(it, ostate, gwx, gwy, gdx, gdy)
    assert abs(scal[0] - ref["density_penalty"]) <= 1e-9 * max(1.0, abs(ref["density_penalty"]))
    assert bool(scal[1]) == ref["initialized"]
    assert abs(ax - ref["step_x"]) <= 1e-5 * ref["step_x"] and abs(ay - ref["step_y"]) <= 1e-5 * ref["step_y"]
    for k in ("x", "y", "x_prev", "y_prev"):
        assert np.abs(state[k] - ref[k]).max() <= 2e-4 + 1e-5 * np.abs(ref[k]).max(), k
    assert rel_err(state["gprev_x"], ref["gprev_x"]) <= 1e-4
    assert rel_err(state["gprev_y"], ref["gprev_y"]) <= 1e-4
    assert abs(nx - norms[0]) <= 1e-4 * norms[0] + 1e-6 and abs(ny - norms[1]) <= 1e-4 * norms[1] + 1e-6
    assert np.abs(nlx - ref["look_x"]).max() <= 5e-4 and np.abs(nly - ref["look_y"]).max() <= 5e-4


def test_hpwl_bit_exact(case):
    name, nl, chip, ctx, orc = case
    rng = np.random.default_rng(3)
    sx = rng.integers(0, chip.width, nl.num_cells).astype(np.int32)
    sy = rng.integers(0, chip.height, nl.num_cells).astype(np.int32)
    if nl.cell_w is not None:
        sx = np.minimum(sx, chip.width - nl.cell_w.astype(np.int32))
        sy = np.minimum(sy, chip.height - nl.cell_h.astype(np.int32))
    assert ctx.hpwl(sx, sy) == orc.hpwl(sx, sy)


def test_legalizer_bit_exact(case):
    name, nl, chip, ctx, orc = case
    for clustered in (False, True):
        x, y = positions(nl, chip, 17, clustered)
        sx, sy, disp = ctx.legalize(x, y)
        st, ox, oy, odisp = orc.legalize(x, y, 1)
        assert st == 0
        assert np.array_equal(sx, ox) and np.array_equal(sy, oy)
        assert disp == odisp


# --- whole loop ------------------------------------------------------------
def test_full_run_matches_oracle():
    """5k-cell reference-geometry run with the reference field formula,
    against the FP64 oracle: final legalised HPWL within 0.5 %, the same
    convergence, the exit iteration within one interval, the reported HPWL
    equal to its binding's.

    Trajectory: the reference formula does not spread cells, and from about
    iteration 25 the loop oscillates on a plateau (overlap 0.60-0.70) that
    never converges.  Up to iteration 20 (five checkpoints) the runs agree
    checkpoint by checkpoint: overlap within 2e-3 absolute, legalised HPWL
    within 0.5 %.  On the plateau, FP32 and FP64 rounding decorrelate the
    oscillation, so the test checks its statistics instead: over iterations
    >= 50 the mean overlap within 0.02 and both runs inside [0.55, 0.75]."""
    nl, chip, cfg = E.workload("electro_5k_128")
    r = E.place_electro(nl, chip, cfg)
    orc = Oracle(nl, chip)
    st, o = orc.place(cfg, dct_backend=1, legal_method=1)
    assert st == 0
    assert r.converged == o["converged"]
    assert abs(r.hpwl - o["hpwl"]) <= 0.005 * o["hpwl"], (r.hpwl, o["hpwl"])
    # the exit iteration may differ by a legalisation interval at most
    assert abs(r.iters - o["iters"]) <= cfg.legalize_interval
    # the GPU's reported HPWL is the integer HPWL of its own binding
    bx, by = r.bel_tile % chip.width, r.bel_tile // chip.width
    assert orc.hpwl(bx, by) == r.hpwl
    assert len(np.unique(r.bel_tile)) == nl.num_cells
    ours = {t["iter"]: t for t in r.trajectory}
    assert len(o["trajectory"]) == len(r.trajectory) and all(t["iter"] in ours for t in o["trajectory"])
    early = [t for t in o["trajectory"] if t["iter"] <= 20]
    assert len(early) == 5
    for t in early:
        assert abs(ours[t["iter"]]["overlap"] - t["overlap"]) <= 2e-3, t["iter"]
        assert abs(ours[t["iter"]]["hpwl"] - t["hpwl"]) <= 0.005 * t["hpwl"], t["iter"]
    late_g = np.array([ours[t["iter"]]["overlap"] for t in o["trajectory"] if t["iter"] >= 50])
    late_o = np.array([t["overlap"] for t in o["trajectory"] if t["iter"] >= 50])
    assert abs(late_g.mean() - late_o.mean()) <= 0.02, (late_g.mean(), late_o.mean())
    for v in (late_g, late_o):
        assert v.min() >= 0.55 and v.max() <= 0.75


def test_full_run_potential_gradient_mode():
    """Extension mode: the same loop with the potential-gradient field
    spreads the cells and converges (overlap < 0.10), like the oracle's."""
    nl, chip, cfg = E.workload("electro_5k_128")
    opts = E.RunOptions(field_mode=E._abi.EPLACE_FIELD_POTENTIAL_GRADIENT)
    r = E.place_electro(nl, chip, cfg, opts)
    st, o = Oracle(nl, chip).place(cfg, field_mode=1)
    assert st == 0 and o["converged"] and r.converged
    assert r.overlap < 0.1
    assert abs(r.hpwl - o["hpwl"]) <= 0.005 * o["hpwl"], (r.hpwl, o["hpwl"])


def test_full_run_tensor_core_mode():
    """Mixed-precision form (BF16x3 tensor-core transform): same job outcome
    as the FP64 oracle (potential-gradient field, 5k-cell workload)."""
    nl, chip, cfg = E.workload("electro_5k_128")
    opts = E.RunOptions(field_mode=E._abi.EPLACE_FIELD_POTENTIAL_GRADIENT, dct_mode=TC)
    r = E.place_electro(nl, chip, cfg, opts)
    st, o = Oracle(nl, chip).place(cfg, field_mode=1)
    assert r.converged and o["converged"]
    assert abs(r.hpwl - o["hpwl"]) <= 0.005 * o["hpwl"], (r.hpwl, o["hpwl"])


def test_deterministic():
    nl, chip, cfg = E.workload("electro_5k_128")
    cfg.max_iters = 60
    with E.PlacementContext(nl, chip) as ctx:
        a = ctx.run(cfg)
        b = ctx.run(cfg)
    assert np.array_equal(a.bel_tile, b.bel_tile)
    assert a.trajectory == b.trajectory
    assert np.array_equal(a.x, b.x)


# --- reference tests (tests/electro_place_tests.rs) on the flat form --------
@pytest.mark.parametrize("n,seed,iters", [(2, 42, 10), (4, 123, 10), (1, 1, 5)])
def test_reference_small_designs(n, seed, iters):
    nl, chip = star_netlist(n)
    cfg = E.ElectroPlaceCfg(seed=seed, max_iters=iters, legalize_interval=2)
    r = E.place_electro(nl, chip, cfg)
    assert len(np.unique(r.bel_tile)) == n and (r.bel_tile >= 0).all() and (r.bel_tile < 4).all()
    o = Oracle(nl, chip).place(cfg)[1]
    assert np.array_equal(r.bel_tile, o["site_y"] * 2 + o["site_x"])


def test_reference_deterministic_seed99():
    nl, chip = star_netlist(3)
    cfg = E.ElectroPlaceCfg(seed=99, max_iters=10, legalize_interval=2)
    a = E.place_electro(nl, chip, cfg)
    b = E.PlacerElectro().place(nl, chip, cfg)
    assert np.array_equal(a.bel_tile, b.bel_tile)


def test_no_cells_is_ok():
    nl, chip = star_netlist(0)
    r = E.place_electro(nl, chip, E.ElectroPlaceCfg())
    assert r.iters == 0


def test_errors():
    nl, chip = star_netlist(4)
    with pytest.raises(E.EplaceError):
        E.place_electro(nl, chip, E.ElectroPlaceCfg(legalize_interval=0))
    big = E.Netlist(num_cells=5, net_offsets=np.array([0, 5], np.uint32), pin_cell=np.arange(5, dtype=np.uint32))
    with pytest.raises(E.NoBelsAvailable):
        E.place_electro(big, chip, E.ElectroPlaceCfg(max_iters=3))
    with pytest.raises(RuntimeError, match="ElectroPlace error"):
        E.place(big, chip, placer="electro", max_iters=3)
    bad = E.Netlist(num_cells=2, net_offsets=np.array([0, 2], np.uint32), pin_cell=np.array([0, 7], np.uint32))
    with pytest.raises(E.EplaceError):
        E.place_electro(bad, chip, E.ElectroPlaceCfg())


def test_place_cells_keeps_others():
    nl, chip = E.synth_netlist(E.SynthSpec(seed=9, num_cells=300, num_nets=330, num_pads=20, width=32, height=32))
    first = E.place_electro(nl, chip, E.ElectroPlaceCfg(max_iters=40))
    nl.cell_init_x = (first.bel_tile % 32).astype(np.int32)
    nl.cell_init_y = (first.bel_tile // 32).astype(np.int32)
    target = np.arange(0, 300, 7)
    tiles, _ = E.PlacerElectro().place_cells(nl, chip, E.ElectroPlaceCfg(max_iters=20), target)
    others = np.setdiff1d(np.arange(300), target)
    assert np.array_equal(tiles[others], first.bel_tile[others])
    assert len(np.unique(tiles)) == 300


def test_ctx_load_equals_fresh_context():
    """A context re-targeted at another netlist (eplace_ctx_load, buffers
    kept) gives exactly the result of a fresh context, for a smaller and a
    larger design and a different bin grid."""
    specs = [E.SynthSpec(seed=21, num_cells=3000, num_nets=3300, num_pads=200, width=96, height=96),
             E.SynthSpec(seed=22, num_cells=6000, num_nets=6600, num_pads=300, width=128, height=128,
                         bins_x=64, bins_y=64, macro_fraction=0.03),
             E.SynthSpec(seed=23, num_cells=1500, num_nets=1650, num_pads=100, width=64, height=64)]
    cfg = E.ElectroPlaceCfg(max_iters=60)
    opts = E.RunOptions(field_mode=1)
    first = E.synth_netlist(specs[0])
    ctx = E.PlacementContext(*first)
    try:
        for spec in specs:
            nl, chip = E.synth_netlist(spec)
            ctx.load(nl, chip)
            a = ctx.run(cfg, opts)
            with E.PlacementContext(nl, chip) as fresh:
                b = fresh.run(cfg, opts)
            c = E.place_electro(nl, chip, cfg, opts)  # one-shot: a kept context, re-loaded
            assert c.hpwl == b.hpwl and np.array_equal(c.bel_tile, b.bel_tile) and c.trajectory == b.trajectory
            assert a.hpwl == b.hpwl and a.iters == b.iters and a.best_iter == b.best_iter
            assert np.array_equal(a.bel_tile, b.bel_tile)
            assert a.trajectory == b.trajectory
    finally:
        ctx.close()


def test_wa_gradient_every_degree_class():
    """Nets at both edges of every degree class of the WA kernel (one thread
    per net up to a warp per net, and the three-pass loop beyond 224 pins),
    pads on some nets, and one cell on 150 nets (which lowers the packed
    gradient's fixed-point scale): parity with the FP64 oracle."""
    rng = np.random.default_rng(31)
    n, nf, w = 3000, 60, 96
    degrees = [1, 2, 3, 4, 5, 8, 9, 16, 17, 32, 33, 64, 65, 128, 129, 224, 225, 600] * 6
    off, pins = [0], []
    for k, d in enumerate(degrees):
        net = rng.choice(n + nf, size=d, replace=False)
        if k < 150 and 7 not in net:
            net[-1] = 7  # cell 7 joins 150 nets
        pins.extend(int(p) for p in net)
        off.append(len(pins))
    fx = rng.integers(0, w, nf).astype(np.int32)
    fy = rng.integers(0, w, nf).astype(np.int32)
    nl = E.Netlist(num_cells=n, net_offsets=np.array(off, np.uint32), pin_cell=np.array(pins, np.uint32),
                   fixed_x=fx, fixed_y=fy)
    chip = E.Chip(w, w)
    orc = Oracle(nl, chip)
    with E.PlacementContext(nl, chip) as ctx:
        for seed, coeff in ((3, 0.5), (4, 0.1)):
            r = np.random.default_rng(seed)
            x = r.uniform(0, w - 1, n).astype(np.float32)
            y = r.uniform(0, w - 1, n).astype(np.float32)
            gx, gy = ctx.wa_grad(x, y, coeff)
            rx, ry = orc.wa_gradient(x, y, coeff)
            assert rel_err(gx, rx) <= 1e-4 and rel_err(gy, ry) <= 1e-4, coeff
