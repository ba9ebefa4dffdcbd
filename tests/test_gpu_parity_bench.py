"""Parity with the FP64 oracle at the benchmark configurations' sizes.

Stage parity, teacher-forced (the oracle gets exactly the FP32 inputs the
kernels get), on the 200,000-cell / 1024^2-site / 512^2-bin workload (the
benchmark's single job) and on the 800,000-cell / 2048^2-site / 1024^2-bin
workload (the precision form): WA gradient, density map and overlap, field
and potential spectrum in both transforms (FP32 SIMT and BF16x3 tcgen05) and
both field formulas, field gather, the fused step, HPWL.

Whole jobs against the committed oracle runs (tests/golden/job_summaries.json,
made by tests/golden/make_job_summaries.py): the same convergence, the exit
iteration within one legalisation interval, the final legalised HPWL within
0.5 %, and at every checkpoint both runs reach the overlap within 2e-3
absolute and the legalised HPWL within 0.5 %.

Tolerances (stated per quantity, as in test_gpu_parity.py):
  WA gradient, field, potential spectrum: normwise max|gpu-oracle|/max|oracle| <= 1e-4
  density map, gathered density gradient: normwise <= 1e-5
  overlap: absolute <= 1e-6
  HPWL of a binding, legalised sites: bit-exact

On the 2048^2-site workload the reference's WA formula (exponents shifted by
the pin mean, wa.rs:58) overflows FP64 on the first iteration; the oracle's
job record and the WA comparisons there use its overflow-free shift (per-net
max / min, the same function and the shift the kernel uses), and the WA test
also checks every cell the reference formula still computes.
"""

import json
import os

import numpy as np
import pytest

import eisenjoch_b200 as E
from oracle.oracle import Oracle, fista_sequence
from tests.conftest import rel_err

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
TC = E._abi.EPLACE_DCT_BF16X3_TC
SIMT = E._abi.EPLACE_DCT_FP32_SIMT
FFT = E._abi.EPLACE_DCT_FP32_FFT

OVERLAP_TOL = 2e-3      # checkpoint overlap, absolute
HPWL_TOL = 0.005        # legalised HPWL, relative


def golden(key):
    with open(os.path.join(HERE, "golden", "job_summaries.json")) as f:
        return json.load(f)[key]


@pytest.fixture(scope="module", params=["electro_200k_1024", "electro_800k_2048"])
def bench_case(request):
    nl, chip, cfg = E.workload(request.param)
    ctx = E.PlacementContext(nl, chip)
    orc = Oracle(nl, chip)
    yield request.param, nl, chip, ctx, orc
    ctx.close()


def positions(nl, chip, seed, clustered):
    rng = np.random.default_rng(seed)
    n = nl.num_cells
    if clustered:
        cx = rng.uniform(0.3, 0.7, 16) * (chip.width - 1)
        cy = rng.uniform(0.3, 0.7, 16) * (chip.height - 1)
        k = rng.integers(0, 16, n)
        x = cx[k] + rng.normal(0, chip.width * 0.04, n)
        y = cy[k] + rng.normal(0, chip.height * 0.04, n)
    else:
        x = rng.uniform(0, chip.width - 1, n)
        y = rng.uniform(0, chip.height - 1, n)
    return (np.clip(x, 0, chip.width - 1).astype(np.float32), np.clip(y, 0, chip.height - 1).astype(np.float32))


@pytest.mark.parametrize("clustered", [False, True])
def test_wa_gradient_bench(bench_case, clustered):
    name, nl, chip, ctx, orc = bench_case
    x, y = positions(nl, chip, 41, clustered)
    gx, gy = ctx.wa_grad(x, y, 0.5)
    sx, sy = orc.wa_gradient(x, y, 0.5, wa_mode=1)
    assert rel_err(gx, sx) <= 1e-4 and rel_err(gy, sy) <= 1e-4, (name, rel_err(gx, sx), rel_err(gy, sy))
    rx, ry = orc.wa_gradient(x, y, 0.5)  # the reference's mean shift
    ok = np.isfinite(rx) & np.isfinite(ry)
    assert np.isfinite(gx).all() and np.isfinite(gy).all()
    if ok.any():
        assert rel_err(gx[ok], rx[ok]) <= 1e-4 and rel_err(gy[ok], ry[ok]) <= 1e-4


@pytest.mark.parametrize("clustered", [False, True])
def test_density_bench(bench_case, clustered):
    name, nl, chip, ctx, orc = bench_case
    x, y = positions(nl, chip, 42, clustered)
    d, ov = ctx.density(x, y)
    rd = orc.density(x, y)
    assert rel_err(d, rd) <= 1e-5, (name, rel_err(d, rd))
    assert abs(ov - orc.overlap(rd)) <= 1e-6


@pytest.mark.parametrize("dct_mode", [SIMT, TC, FFT])
@pytest.mark.parametrize("field_mode", [0, 1])
def test_field_bench(bench_case, dct_mode, field_mode):
    """Field and potential spectrum of a clustered density map, all three
    transforms, both field formulas."""
    name, nl, chip, ctx, orc = bench_case
    x, y = positions(nl, chip, 43, True)
    rd = orc.density(x, y)
    ex, ey, phi = ctx.field(rd, dct_mode=dct_mode, want_phi=True, field_mode=field_mode)
    rex, rey, rphi = orc.field(rd, 1.0, want_phi=True, field_mode=field_mode)
    errs = rel_err(ex, rex), rel_err(ey, rey), rel_err(phi, rphi)
    assert max(errs) <= 1e-4, (name, dct_mode, field_mode, errs)


def test_gather_bench(bench_case):
    name, nl, chip, ctx, orc = bench_case
    x, y = positions(nl, chip, 44, True)
    rd = orc.density(x, y)
    rex, rey = orc.field(rd, 1.0, field_mode=1)
    ex, ey = rex.astype(np.float32), rey.astype(np.float32)
    gx, gy = ctx.gather(x, y, ex, ey)
    ox, oy = orc.gather(x, y, ex, ey)
    assert rel_err(gx, ox) <= 1e-5 and rel_err(gy, oy) <= 1e-5, (name, rel_err(gx, ox), rel_err(gy, oy))


@pytest.mark.parametrize("it,initialized", [(0, False), (23, True)])
def test_fused_step_bench(bench_case, it, initialized):
    """The fused gather / penalty / precondition / Barzilai-Borwein / FISTA
    step, teacher-forced at the benchmark sizes (the step's FP64 reductions
    run over 200k and 800k cells here)."""
    name, nl, chip, ctx, orc = bench_case
    rng = np.random.default_rng(200 + it)
    n = nl.num_cells
    x, y = positions(nl, chip, 45, True)
    xp = np.clip(x + rng.normal(0, 0.3, n), 0, chip.width - 1).astype(np.float32)
    yp = np.clip(y + rng.normal(0, 0.3, n), 0, chip.height - 1).astype(np.float32)
    a = fista_sequence(it)
    m = 0.0 if it == 0 else (a - 1) / ((1 + np.sqrt(1 + 4 * a * a)) / 2)
    lx = np.clip(x + m * (x.astype(np.float64) - xp), 0, chip.width - 1).astype(np.float32)
    ly = np.clip(y + m * (y.astype(np.float64) - yp), 0, chip.height - 1).astype(np.float32)
    gwx, gwy = orc.wa_gradient(lx, ly, 0.5, wa_mode=1)
    gwx, gwy = gwx.astype(np.float32), gwy.astype(np.float32)
    rd = orc.density(lx, ly)
    rex, rey = orc.field(rd, 1.0, field_mode=1)
    ex, ey = rex.astype(np.float32), rey.astype(np.float32)
    gpx = rng.normal(0, 0.05, n).astype(np.float32)
    gpy = rng.normal(0, 0.05, n).astype(np.float32)
    lam = 2.3 if initialized else 0.0
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
    # FP32 holds these coordinates to one ulp of the largest; the look-ahead
    # x + m (x - x_prev) carries the position error times 1 + m < 2 and rounds
    # once more: 5e-4 sites plus 8 ulps of the largest coordinate.
    tol = 5e-4 + 8 * float(np.spacing(np.float32(max(chip.width, chip.height))))
    assert np.abs(nlx - ref["look_x"]).max() <= tol and np.abs(nly - ref["look_y"]).max() <= tol


def test_hpwl_bit_exact_bench(bench_case):
    name, nl, chip, ctx, orc = bench_case
    rng = np.random.default_rng(46)
    sx = rng.integers(0, chip.width, nl.num_cells).astype(np.int32)
    sy = rng.integers(0, chip.height, nl.num_cells).astype(np.int32)
    sx = np.minimum(sx, chip.width - nl.cell_w.astype(np.int32))
    sy = np.minimum(sy, chip.height - nl.cell_h.astype(np.int32))
    assert ctx.hpwl(sx, sy) == orc.hpwl(sx, sy)


# --- whole jobs against the oracle's committed runs -------------------------
def compare_job(r, g, cfg, orc, chip, label):
    """Checks a GPU PlacementResult against an oracle job record."""
    assert g["status"] == 0, label
    assert r.converged == g["converged"], label
    assert abs(r.iters - g["iters"]) <= cfg.legalize_interval, (label, r.iters, g["iters"])
    assert abs(r.hpwl - g["hpwl"]) <= HPWL_TOL * g["hpwl"], (label, r.hpwl, g["hpwl"])
    bx, by = r.bel_tile % chip.width, r.bel_tile // chip.width
    assert orc.hpwl(bx, by) == r.hpwl, label  # the reported HPWL is its own binding's
    ours = {t["iter"]: t for t in r.trajectory}
    common = [c for c in g["checkpoints"] if c["iter"] in ours]
    assert len(common) >= min(len(ours), len(g["checkpoints"])) - 1, label
    d_ov = max(abs(ours[c["iter"]]["overlap"] - c["overlap"]) for c in common)
    d_hp = max(abs(ours[c["iter"]]["hpwl"] - c["hpwl"]) / c["hpwl"] for c in common)
    assert d_ov <= OVERLAP_TOL, (label, d_ov)
    assert d_hp <= HPWL_TOL, (label, d_hp)
    return d_ov, d_hp


@pytest.mark.parametrize("dct_mode", [SIMT, FFT])
def test_full_run_200k_matches_oracle(dct_mode):
    """The benchmark's job (potential-gradient field, FP32 GEMM and FFT
    transforms) against the oracle's 200k run: convergence, exit iteration,
    final HPWL and the overlap / HPWL trajectory over all checkpoints."""
    nl, chip, cfg = E.workload("electro_200k_1024")
    r = E.place_electro(nl, chip, cfg, E.RunOptions(field_mode=1, dct_mode=dct_mode))
    compare_job(r, golden("electro_200k_1024"), cfg, Oracle(nl, chip), chip, "200k dct %d" % dct_mode)


@pytest.mark.parametrize("dct_mode", [SIMT, TC, FFT])
def test_full_run_800k_precision_forms(dct_mode):
    """The precision form: the 800k job with the BF16x3 tensor-core
    transform and with the FP32 transform, each against the FP64 oracle's
    run (overflow-free WA shift)."""
    nl, chip, cfg = E.workload("electro_800k_2048")
    r = E.place_electro(nl, chip, cfg, E.RunOptions(field_mode=1, dct_mode=dct_mode))
    compare_job(r, golden("electro_800k_2048:stable_wa"), cfg, Oracle(nl, chip), chip, "800k dct %d" % dct_mode)
