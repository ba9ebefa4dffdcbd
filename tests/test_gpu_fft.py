"""The FFT form of the spectral solve (EPLACE_DCT_FP32_FFT, csrc/fft.cu)
against the FP64 oracle's field (density.rs:96-166): power-of-two bin grids
from 16 to 1024 per axis, square and not, both field formulas, the
potential spectrum too; grids the FFT does not take fall back to the FP32
GEMMs and give their bits; a whole job in this form converges like the
oracle's.

Tolerance: normwise relative error max|gpu - oracle| / max|oracle| <= 1e-4
(the FFT's FP32 rounding error grows with log N)."""

import numpy as np
import pytest

import eisenjoch_b200 as E
from oracle.oracle import Oracle
from tests.conftest import rel_err

pytestmark = pytest.mark.gpu

FFT = E._abi.EPLACE_DCT_FP32_FFT
SIMT = E._abi.EPLACE_DCT_FP32_SIMT


def grid_problem(bx, by, seed):
    """A chip of bx x by sites (one bin per site) with a few cells, and a
    clustered density map on it."""
    rng = np.random.default_rng(seed)
    nl = E.Netlist(num_cells=4, net_offsets=np.array([0, 2], np.uint32), pin_cell=np.array([0, 1], np.uint32))
    chip = E.Chip(bx, by)
    yy, xx = np.mgrid[0:by, 0:bx]
    d = np.zeros((by, bx))
    for _ in range(6):
        cx, cy = rng.uniform(0, bx), rng.uniform(0, by)
        s = rng.uniform(0.05, 0.2) * max(bx, by)
        d += rng.uniform(0.5, 3.0) * np.exp(-((xx - cx) ** 2 + (yy - cy) ** 2) / (2 * s * s))
    d += rng.uniform(0, 0.2, d.shape)
    # mean = the cells' area per bin, the charge both sides subtract (a
    # constant only moves the zero frequency, which the solve drops)
    d += 4.0 / d.size - d.mean()
    return nl, chip, d.ravel()


@pytest.mark.parametrize("bx,by", [(16, 16), (32, 128), (128, 64), (256, 256), (64, 1024), (1024, 1024)])
@pytest.mark.parametrize("field_mode", [0, 1])
def test_fft_field_matches_oracle(bx, by, field_mode):
    nl, chip, d = grid_problem(bx, by, bx * 7 + by)
    orc = Oracle(nl, chip)
    with E.PlacementContext(nl, chip) as ctx:
        ex, ey, phi = ctx.field(d, dct_mode=FFT, want_phi=True, field_mode=field_mode)
    rex, rey, rphi = orc.field(d, 1.0, want_phi=True, field_mode=field_mode)
    errs = rel_err(ex, rex), rel_err(ey, rey), rel_err(phi, rphi)
    assert max(errs) <= 1e-4, (bx, by, field_mode, errs)


@pytest.mark.parametrize("bx,by", [(90, 60), (96, 48), (2048, 16)])
def test_fft_falls_back_to_gemm(bx, by):
    """Grids outside the FFT's (not powers of two, or above 1024 bins) run the
    FP32 GEMMs: the same bits as asking for them."""
    nl, chip, d = grid_problem(bx, by, 3)
    with E.PlacementContext(nl, chip) as ctx:
        a = ctx.field(d, dct_mode=FFT, field_mode=1)
        b = ctx.field(d, dct_mode=SIMT, field_mode=1)
    assert all(np.array_equal(u, v) for u, v in zip(a, b))


def test_fft_and_gemm_agree_on_the_benchmark_grid():
    """512^2 bins: FFT and GEMM fields agree within both forms' error."""
    nl, chip, d = grid_problem(512, 512, 11)
    with E.PlacementContext(nl, chip) as ctx:
        a = ctx.field(d, dct_mode=FFT, want_phi=True, field_mode=1)
        b = ctx.field(d, dct_mode=SIMT, want_phi=True, field_mode=1)
    assert max(rel_err(u, v) for u, v in zip(a, b)) <= 1e-4


def test_full_run_fft_mode():
    """A whole job with the FFT transform (5k cells, 128^2 bins, potential-
    gradient field) ends like the oracle's."""
    nl, chip, cfg = E.workload("electro_5k_128")
    r = E.place_electro(nl, chip, cfg, E.RunOptions(field_mode=E._abi.EPLACE_FIELD_POTENTIAL_GRADIENT, dct_mode=FFT))
    st, o = Oracle(nl, chip).place(cfg, field_mode=1)
    assert st == 0 and o["converged"] and r.converged
    assert abs(r.hpwl - o["hpwl"]) <= 0.005 * o["hpwl"], (r.hpwl, o["hpwl"])


def test_fft_run_is_deterministic_and_reuses_graphs():
    nl, chip, cfg = E.workload("electro_5k_128")
    cfg.max_iters = 40
    opts = E.RunOptions(field_mode=1, dct_mode=FFT)
    with E.PlacementContext(nl, chip) as ctx:
        a = ctx.run(cfg, opts)
        b = ctx.run(cfg, E.RunOptions(field_mode=1, dct_mode=SIMT))
        c = ctx.run(cfg, opts)
    assert a.hpwl == c.hpwl and np.array_equal(a.bel_tile, c.bel_tile)
    assert abs(a.hpwl - b.hpwl) <= 0.005 * b.hpwl
