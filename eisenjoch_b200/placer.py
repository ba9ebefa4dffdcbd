"""Host-side mirror of the reference ElectroPlace interface over libeplace.so.

Reference interface mirrored here:
  * ElectroPlaceCfg and its defaults  (crates/nextpnr/src/placer/electro_place/config.rs:5-40)
  * place_electro(ctx, cfg)           (crates/nextpnr/src/placer/electro_place/mod.rs:65)
  * PlacerElectro.place / place_cells (electro_place/mod.rs:45-63, trait placer/mod.rs:31-52)
  * PlacerError variants              (crates/nextpnr/src/placer/mod.rs:20-28)
  * Context.place(placer="electro", seed=, max_iters=) and its RuntimeError
    mapping                           (crates/npnr-python/src/lib.rs:224-245, :293-302)

The reference works on a Context (chip database + netlist arena).  Here the
caller hands over the same information flattened: a site grid (Chip) and a
CSR netlist (Netlist).  All computation happens in the CUDA library; this
module only marshals arrays.
"""

import ctypes
import json
import os
from dataclasses import dataclass, field, fields
from typing import List, Optional, Sequence

import numpy as np

from . import _abi
from ._abi import P


# ---------------------------------------------------------------------------
# Configuration
# ---------------------------------------------------------------------------
@dataclass
class ElectroPlaceCfg:
    """ElectroPlaceCfg (electro_place/config.rs:5-40), same fields and defaults."""

    seed: int = 1
    wl_coeff: float = 0.5
    target_util: float = 0.7
    timing_driven: bool = False
    target_density: float = 1.0
    timing_weight: float = 0.0
    nesterov_step_size: float = 0.1
    max_iters: int = 500
    legalize_interval: int = 5

    def to_c(self):
        c = _abi.Cfg()
        for f in fields(self):
            v = getattr(self, f.name)
            setattr(c, f.name, int(v) if f.name in ("seed", "max_iters", "legalize_interval", "timing_driven") else float(v))
        return c


@dataclass
class RunOptions:
    """Build-only knobs with no reference counterpart (eplace_opts)."""

    dct_mode: int = _abi.EPLACE_DCT_FP32_FFT
    legal_threads: int = 0
    use_graphs: bool = True
    verbose: int = 0
    max_inflight: int = 3
    field_mode: int = _abi.EPLACE_FIELD_REFERENCE
    legal_mode: int = _abi.EPLACE_LEGAL_HOST
    wait_limit_us: int = 0  # bound of each device grid-barrier wait; 0 = about 2 s

    def to_c(self):
        o = _abi.Opts()
        _abi.lib().eplace_opts_default(ctypes.byref(o))
        o.dct_mode = int(self.dct_mode)
        o.legal_threads = int(self.legal_threads)
        o.use_graphs = int(bool(self.use_graphs))
        o.verbose = int(self.verbose)
        o.max_inflight = int(self.max_inflight)
        o.field_mode = int(self.field_mode)
        o.legal_mode = int(self.legal_mode)
        o.wait_limit_us = int(self.wait_limit_us)
        return o


# ---------------------------------------------------------------------------
# Errors (placer/mod.rs:20-28)
# ---------------------------------------------------------------------------
class PlacerError(RuntimeError):
    """Base of the reference's PlacerError variants."""

    status = -1

    def __init__(self, msg, status=None):
        super().__init__(msg)
        if status is not None:
            self.status = status


class NoBelsAvailable(PlacerError):
    status = _abi.EPLACE_ERR_NO_BELS

    def __init__(self, what):
        super().__init__("No valid BELs available for cell type %s" % what)


class PlacementFailed(PlacerError):
    status = _abi.EPLACE_ERR_PLACEMENT_FAILED

    def __init__(self, what):
        super().__init__("Placement failed: %s" % what)


class InitialPlacementFailed(PlacerError):
    status = _abi.EPLACE_ERR_INITIAL_PLACEMENT

    def __init__(self, what):
        super().__init__("Initial placement failed: could not place cell %s" % what)


class EplaceError(RuntimeError):
    """Library errors with no PlacerError counterpart (invalid input, OOM,
    CUDA failure, bounded-wait timeout, no device)."""

    def __init__(self, status, msg):
        super().__init__("eplace status %d: %s" % (status, msg))
        self.status = status


def _raise(status, ctx=None):
    msg = _abi.last_error(ctx)
    if status == _abi.EPLACE_ERR_NO_BELS:
        raise NoBelsAvailable(msg)
    if status == _abi.EPLACE_ERR_PLACEMENT_FAILED:
        raise PlacementFailed(msg)
    if status == _abi.EPLACE_ERR_INITIAL_PLACEMENT:
        raise InitialPlacementFailed(msg)
    raise EplaceError(status, msg)


def check(status, ctx=None):
    if status != _abi.EPLACE_OK:
        _raise(status, ctx)


# ---------------------------------------------------------------------------
# Problem description
# ---------------------------------------------------------------------------
@dataclass
class Chip:
    """W x H site grid, one logic BEL per site (tile = y*W + x); bins_x/bins_y
    0 means one density bin per site (the reference's grid)."""

    width: int
    height: int
    bins_x: int = 0
    bins_y: int = 0

    def to_c(self):
        return _abi.Chip(self.width, self.height, self.bins_x, self.bins_y)


def _opt(a, dtype):
    return None if a is None else np.ascontiguousarray(a, dtype=dtype)


@dataclass
class Netlist:
    """CSR netlist.  Pin ids < num_cells are movable cells in solver order,
    num_cells + f is fixed cell f; each net lists its driver first."""

    num_cells: int
    net_offsets: np.ndarray
    pin_cell: np.ndarray
    fixed_x: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    fixed_y: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    cell_w: Optional[np.ndarray] = None
    cell_h: Optional[np.ndarray] = None
    cell_init_x: Optional[np.ndarray] = None
    cell_init_y: Optional[np.ndarray] = None
    fixed_on_logic: Optional[np.ndarray] = None
    net_has_driver: Optional[np.ndarray] = None

    def __post_init__(self):
        self.net_offsets = np.ascontiguousarray(self.net_offsets, dtype=np.uint32)
        self.pin_cell = np.ascontiguousarray(self.pin_cell, dtype=np.uint32)
        self.fixed_x = np.ascontiguousarray(self.fixed_x, dtype=np.int32)
        self.fixed_y = np.ascontiguousarray(self.fixed_y, dtype=np.int32)
        self.cell_w = _opt(self.cell_w, np.uint8)
        self.cell_h = _opt(self.cell_h, np.uint8)
        self.cell_init_x = _opt(self.cell_init_x, np.int32)
        self.cell_init_y = _opt(self.cell_init_y, np.int32)
        self.fixed_on_logic = _opt(self.fixed_on_logic, np.uint8)
        self.net_has_driver = _opt(self.net_has_driver, np.uint8)

    @property
    def num_fixed(self):
        return int(self.fixed_x.shape[0])

    @property
    def num_nets(self):
        return int(self.net_offsets.shape[0]) - 1 if self.net_offsets.shape[0] else 0

    @property
    def num_pins(self):
        return int(self.pin_cell.shape[0])

    def to_c(self):
        n = _abi.Netlist()
        n.num_cells = self.num_cells
        n.num_fixed = self.num_fixed
        n.num_nets = self.num_nets
        n.cell_w = _abi.ptr(self.cell_w, ctypes.c_uint8)
        n.cell_h = _abi.ptr(self.cell_h, ctypes.c_uint8)
        n.cell_init_x = _abi.ptr(self.cell_init_x, ctypes.c_int32)
        n.cell_init_y = _abi.ptr(self.cell_init_y, ctypes.c_int32)
        n.fixed_x = _abi.ptr(self.fixed_x, ctypes.c_int32)
        n.fixed_y = _abi.ptr(self.fixed_y, ctypes.c_int32)
        n.fixed_on_logic = _abi.ptr(self.fixed_on_logic, ctypes.c_uint8)
        n.net_offsets = _abi.ptr(self.net_offsets, ctypes.c_uint32)
        n.pin_cell = _abi.ptr(self.pin_cell, ctypes.c_uint32)
        n.net_has_driver = _abi.ptr(self.net_has_driver, ctypes.c_uint8)
        return n


# ---------------------------------------------------------------------------
# Synthetic generator
# ---------------------------------------------------------------------------
@dataclass
class SynthSpec:
    """Seeded synthetic netlist (no reference counterpart)."""

    seed: int
    num_cells: int
    num_nets: int
    num_pads: int
    width: int
    height: int
    bins_x: int = 0
    bins_y: int = 0
    cluster_size: int = 32
    locality: float = 0.6
    macro_fraction: float = 0.0
    macro_min: int = 2
    macro_max: int = 8

    def to_c(self):
        s = _abi.SynthSpec()
        for f in fields(self):
            setattr(s, f.name, getattr(self, f.name))
        return s


def synth_netlist(spec: SynthSpec):
    """Generates (Netlist, Chip) from a SynthSpec through the C library."""
    L = _abi.lib()
    cs = spec.to_c()
    info = _abi.SynthInfo()
    check(L.eplace_synth_size(ctypes.byref(cs), ctypes.byref(info)))
    cw = np.ones(spec.num_cells, np.uint8)
    ch = np.ones(spec.num_cells, np.uint8)
    fx = np.zeros(spec.num_pads, np.int32)
    fy = np.zeros(spec.num_pads, np.int32)
    off = np.zeros(spec.num_nets + 1, np.uint32)
    pins = np.zeros(info.num_pins, np.uint32)
    check(
        L.eplace_synth_fill(
            ctypes.byref(cs),
            _abi.ptr(cw, ctypes.c_uint8),
            _abi.ptr(ch, ctypes.c_uint8),
            _abi.ptr(fx, ctypes.c_int32),
            _abi.ptr(fy, ctypes.c_int32),
            _abi.ptr(off, ctypes.c_uint32),
            _abi.ptr(pins, ctypes.c_uint32),
        )
    )
    macro = spec.macro_fraction > 0
    nl = Netlist(
        num_cells=spec.num_cells,
        net_offsets=off,
        pin_cell=pins,
        fixed_x=fx,
        fixed_y=fy,
        cell_w=cw if macro else None,
        cell_h=ch if macro else None,
    )
    return nl, Chip(spec.width, spec.height, spec.bins_x, spec.bins_y)


# The benchmark workloads (seeded synthetic stand-ins for the configurations
# the placer is measured on; shapes and distributions as specified there),
# kept as data so that tools that must not load this package can read them.
def _load_workloads():
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "workloads.json")) as f:
        table = json.load(f)
    return {name: dict(spec=SynthSpec(**w["spec"]), cfg=dict(w["cfg"]))
            for name, w in table.items() if not name.startswith("_")}


WORKLOADS = _load_workloads()


def workload(name):
    w = WORKLOADS[name]
    nl, chip = synth_netlist(w["spec"])
    return nl, chip, ElectroPlaceCfg(**w["cfg"])


def mixed_job_spec(seed, num_cells):
    """One job of the mixed-size streams (same generator as the single
    instances): nets = 1.1 x cells, 5% macros, clusters of 64 with locality
    0.6, pads = cells / 100 (at least 40), bin grid = next power of two >=
    sqrt(cells) clamped to [64, 512], two sites per bin edge."""
    b = 64
    while b * b < num_cells and b < 512:
        b *= 2
    return SynthSpec(seed=seed, num_cells=int(num_cells), num_nets=int(round(1.1 * num_cells)),
                     num_pads=max(40, int(num_cells) // 100), width=2 * b, height=2 * b, bins_x=b, bins_y=b,
                     cluster_size=64, macro_fraction=0.05)


def mixed_job_specs(count, seed0, nmin, nmax, rng_seed):
    """count jobs with cell counts log-uniform in [nmin, nmax] (numpy
    default_rng(rng_seed)); job i has generator seed seed0 + i."""
    rng = np.random.default_rng(rng_seed)
    cells = np.exp(rng.uniform(np.log(nmin), np.log(nmax), count)).astype(np.int64)
    return [mixed_job_spec(seed0 + i, int(n)) for i, n in enumerate(cells)]


def batched_specs(count=64):
    """Batched form: instances of 2k..200k cells, instance i seed 1000 + i."""
    return mixed_job_specs(count, 1000, 2000, 200000, rng_seed=1000)


def served_stream(count, rate):
    """Served form: jobs of 1k..300k cells, job j seed 100000 + j, Poisson
    arrivals (seed 7) at `rate` jobs/s.  Returns (specs, arrival times in s,
    the first at 0)."""
    specs = mixed_job_specs(count, 100000, 1000, 300000, rng_seed=100000)
    gaps = np.random.default_rng(7).exponential(1.0 / rate, count)
    return specs, np.cumsum(gaps) - gaps[0]


# ---------------------------------------------------------------------------
# Results
# ---------------------------------------------------------------------------
@dataclass
class PlacementResult:
    """What place_electro leaves on the Context (cell -> BEL), plus the
    reference's trajectory log fields."""

    bel_tile: np.ndarray
    bel_x: np.ndarray
    bel_y: np.ndarray
    x: np.ndarray
    y: np.ndarray
    hpwl: int
    overlap: float
    iters: int
    best_iter: int
    converged: bool
    trajectory: List[dict]
    gpu_seconds: float
    total_seconds: float
    gpu_launches: int
    h2d_bytes: int
    d2h_bytes: int


class _ResultBuffers:
    def __init__(self, n, width, traj_cap):
        self.bel_tile = np.zeros(n, np.int32)
        self.bel_index = np.zeros(n, np.int32)
        self.x = np.zeros(n, np.float32)
        self.y = np.zeros(n, np.float32)
        self.traj = (_abi.TrajEntry * max(1, traj_cap))()
        self.width = width
        r = _abi.Result()
        r.bel_tile = _abi.ptr(self.bel_tile, ctypes.c_int32)
        r.bel_index = _abi.ptr(self.bel_index, ctypes.c_int32)
        r.x = _abi.ptr(self.x, ctypes.c_float)
        r.y = _abi.ptr(self.y, ctypes.c_float)
        r.traj = ctypes.cast(self.traj, P(_abi.TrajEntry))
        r.traj_capacity = traj_cap
        self.c = r

    def result(self):
        r = self.c
        traj = []
        for k in range(r.traj_len):
            t = self.traj[k]
            traj.append(
                dict(iter=t.iter, hpwl=t.hpwl, disp=t.displacement, step_x=t.step_x, step_y=t.step_y,
                     density_penalty=t.density_penalty, overlap=t.overlap)
            )
        return PlacementResult(
            bel_tile=self.bel_tile.copy(),
            bel_x=self.bel_tile % self.width,
            bel_y=self.bel_tile // self.width,
            x=self.x.copy(),
            y=self.y.copy(),
            hpwl=int(r.hpwl),
            overlap=float(r.overlap),
            iters=int(r.iters),
            best_iter=int(r.best_iter),
            converged=bool(r.converged),
            trajectory=traj,
            gpu_seconds=float(r.gpu_seconds),
            total_seconds=float(r.total_seconds),
            gpu_launches=int(r.gpu_launches),
            h2d_bytes=int(r.h2d_bytes),
            d2h_bytes=int(r.d2h_bytes),
        )


def _traj_cap(cfg):
    return int(cfg.max_iters // max(1, cfg.legalize_interval) + 2)


# ---------------------------------------------------------------------------
# Context: the device-resident netlist
# ---------------------------------------------------------------------------
class PlacementContext:
    """Owns an eplace_ctx: the netlist uploaded to one GPU.  Re-running on
    the same context re-uses the device copy (inputs resident in HBM)."""

    def __init__(self, netlist: Netlist, chip: Chip, device: int = 0):
        self.netlist = netlist
        self.chip = chip
        self._lib = _abi.lib()
        self._nl_c = netlist.to_c()  # keeps pointers alive with the arrays
        self._chip_c = chip.to_c()
        h = ctypes.c_void_p()
        check(self._lib.eplace_ctx_create(ctypes.byref(self._nl_c), ctypes.byref(self._chip_c), device, ctypes.byref(h)))
        self.handle = h

    def load(self, netlist: Netlist, chip: Chip):
        """Re-targets this context at another netlist (eplace_ctx_load):
        device buffers are kept and only grow."""
        nl_c, chip_c = netlist.to_c(), chip.to_c()
        self._check(self._lib.eplace_ctx_load(self.handle, ctypes.byref(nl_c), ctypes.byref(chip_c)))
        self.netlist, self.chip, self._nl_c, self._chip_c = netlist, chip, nl_c, chip_c

    def close(self):
        if self.handle:
            self._lib.eplace_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, st):
        if st != _abi.EPLACE_OK:
            _raise(st, self.handle)

    def run(self, cfg: Optional[ElectroPlaceCfg] = None, opts: Optional[RunOptions] = None) -> PlacementResult:
        cfg = cfg or ElectroPlaceCfg()
        opts = opts or RunOptions()
        cc, oc = cfg.to_c(), opts.to_c()
        buf = _ResultBuffers(self.netlist.num_cells, self.chip.width, _traj_cap(cfg))
        self._check(self._lib.eplace_run(self.handle, ctypes.byref(cc), ctypes.byref(oc), ctypes.byref(buf.c)))
        return buf.result()

    # --- stage entry points (one kernel family each) ---------------------
    def wa_grad(self, x, y, wl_coeff=0.5):
        n = self.netlist.num_cells
        x, y = _abi.f32(x), _abi.f32(y)
        gx, gy = np.zeros(n, np.float32), np.zeros(n, np.float32)
        F = ctypes.c_float
        self._check(self._lib.eplace_stage_wa_grad(self.handle, wl_coeff, _abi.ptr(x, F), _abi.ptr(y, F),
                                                   _abi.ptr(gx, F), _abi.ptr(gy, F)))
        return gx, gy

    def density(self, x, y):
        by, bx = self.bins
        x, y = _abi.f32(x), _abi.f32(y)
        d = np.zeros((by, bx), np.float64)
        ov = ctypes.c_double()
        F = ctypes.c_float
        self._check(self._lib.eplace_stage_density(self.handle, _abi.ptr(x, F), _abi.ptr(y, F),
                                                   _abi.ptr(d, ctypes.c_double), ctypes.byref(ov)))
        return d, ov.value

    def field(self, density, dct_mode=_abi.EPLACE_DCT_FP32_FFT, want_phi=False, field_mode=_abi.EPLACE_FIELD_REFERENCE):
        by, bx = self.bins
        d = _abi.f64(density).reshape(by, bx)
        ex, ey = np.zeros((by, bx), np.float32), np.zeros((by, bx), np.float32)
        phi = np.zeros((by, bx), np.float32) if want_phi else None
        F = ctypes.c_float
        self._check(self._lib.eplace_stage_field(self.handle, _abi.ptr(d, ctypes.c_double), dct_mode, field_mode,
                                                 _abi.ptr(ex, F), _abi.ptr(ey, F), _abi.ptr(phi, F)))
        return (ex, ey, phi) if want_phi else (ex, ey)

    def gather(self, x, y, ex, ey):
        n = self.netlist.num_cells
        F = ctypes.c_float
        x, y, ex, ey = _abi.f32(x), _abi.f32(y), _abi.f32(ex), _abi.f32(ey)
        gx, gy = np.zeros(n, np.float32), np.zeros(n, np.float32)
        self._check(self._lib.eplace_stage_gather(self.handle, _abi.ptr(x, F), _abi.ptr(y, F), _abi.ptr(ex, F),
                                                  _abi.ptr(ey, F), _abi.ptr(gx, F), _abi.ptr(gy, F)))
        return gx, gy

    def step(self, it, look_x, look_y, gwl_x, gwl_y, ex, ey, state, scal):
        """Teacher-forced fused step.  state: dict of float32 arrays x, y,
        x_prev, y_prev, gprev_x, gprev_y (updated in place); scal: list
        [density_penalty, initialized, step_x, step_y] (updated in place).
        Returns (step_norm_x, step_norm_y, alpha_x, alpha_y, next_look_x, next_look_y)."""
        n = self.netlist.num_cells
        F = ctypes.c_float
        arrs = [_abi.f32(a) for a in (look_x, look_y, gwl_x, gwl_y, ex, ey)]
        st = {k: _abi.f32(state[k]).copy() for k in ("x", "y", "x_prev", "y_prev", "gprev_x", "gprev_y")}
        sc = np.array(scal, np.float64)
        out = np.zeros(4, np.float64)
        nlx, nly = np.zeros(n, np.float32), np.zeros(n, np.float32)
        self._check(self._lib.eplace_stage_step(
            self.handle, it, *[_abi.ptr(a, F) for a in arrs],
            *[_abi.ptr(st[k], F) for k in ("x", "y", "x_prev", "y_prev", "gprev_x", "gprev_y")],
            _abi.ptr(sc, ctypes.c_double), _abi.ptr(out, ctypes.c_double), _abi.ptr(nlx, F), _abi.ptr(nly, F)))
        state.update(st)
        scal[:] = list(sc)
        return out[0], out[1], out[2], out[3], nlx, nly

    def initial_placement(self, seed: int):
        """initial_placement (placer/common.rs:27-117) as eplace_run makes it:
        on the device unless a cell is pre-bound.  Returns (site_x, site_y,
        on_device)."""
        n = self.netlist.num_cells
        sx, sy = np.zeros(n, np.int32), np.zeros(n, np.int32)
        dev = ctypes.c_int32(0)
        self._check(self._lib.eplace_stage_initial_placement(self.handle, seed, _abi.ptr(sx, ctypes.c_int32),
                                                             _abi.ptr(sy, ctypes.c_int32), ctypes.byref(dev)))
        return sx, sy, bool(dev.value)

    def hpwl(self, site_x, site_y):
        v = ctypes.c_int64()
        sx, sy = np.ascontiguousarray(site_x, np.int32), np.ascontiguousarray(site_y, np.int32)
        self._check(self._lib.eplace_stage_hpwl(self.handle, _abi.ptr(sx, ctypes.c_int32), _abi.ptr(sy, ctypes.c_int32),
                                                ctypes.byref(v)))
        return int(v.value)

    def legalize(self, x, y):
        n = self.netlist.num_cells
        x, y = _abi.f32(x), _abi.f32(y)
        sx, sy = np.zeros(n, np.int32), np.zeros(n, np.int32)
        d = ctypes.c_double()
        F = ctypes.c_float
        self._check(self._lib.eplace_legalize(self.handle, _abi.ptr(x, F), _abi.ptr(y, F), _abi.ptr(sx, ctypes.c_int32),
                                              _abi.ptr(sy, ctypes.c_int32), ctypes.byref(d)))
        return sx, sy, d.value

    def legalize_device(self, x, y):
        """The same legalisation on the GPU plus the device HPWL of the
        binding: (site_x, site_y, displacement, hpwl)."""
        n = self.netlist.num_cells
        x, y = _abi.f32(x), _abi.f32(y)
        sx, sy = np.zeros(n, np.int32), np.zeros(n, np.int32)
        d, h = ctypes.c_double(), ctypes.c_int64()
        F = ctypes.c_float
        self._check(self._lib.eplace_stage_legalize(self.handle, _abi.ptr(x, F), _abi.ptr(y, F),
                                                    _abi.ptr(sx, ctypes.c_int32), _abi.ptr(sy, ctypes.c_int32),
                                                    ctypes.byref(d), ctypes.byref(h)))
        return sx, sy, d.value, int(h.value)

    STAGES = ("wa_grad", "density_scatter", "density_final", "dct_gemm1", "dct_gemm2_spectral",
              "dct_gemm3", "dct_gemm4", "gather_step")

    def profile_stages(self, cfg: Optional[ElectroPlaceCfg] = None, reps=20, opts: Optional[RunOptions] = None):
        """Mean device milliseconds per launch of each iteration kernel (CUDA
        events on the context's own stream)."""
        cfg = cfg or ElectroPlaceCfg()
        cc, oc = cfg.to_c(), (opts or RunOptions()).to_c()
        out = np.zeros(8, np.float64)
        self._check(self._lib.eplace_profile_stages(self.handle, ctypes.byref(cc), ctypes.byref(oc), reps,
                                                    _abi.ptr(out, ctypes.c_double)))
        return dict(zip(self.STAGES, out.tolist()))

    @property
    def bins(self):
        bx = self.chip.bins_x or self.chip.width
        by = self.chip.bins_y or self.chip.height
        return by, bx


# ---------------------------------------------------------------------------
# Host-only parts of the path (no device needed)
# ---------------------------------------------------------------------------
def legalize_host(netlist: Netlist, chip: Chip, x, y):
    """Greedy legaliser (electro_place/mod.rs:206-255) without a context."""
    n = netlist.num_cells
    x, y = _abi.f32(x), _abi.f32(y)
    sx, sy = np.zeros(n, np.int32), np.zeros(n, np.int32)
    d = ctypes.c_double()
    nl_c, chip_c = netlist.to_c(), chip.to_c()
    F = ctypes.c_float
    check(_abi.lib().eplace_legalize_host(ctypes.byref(nl_c), ctypes.byref(chip_c), _abi.ptr(x, F), _abi.ptr(y, F),
                                          _abi.ptr(sx, ctypes.c_int32), _abi.ptr(sy, ctypes.c_int32), ctypes.byref(d)))
    return sx, sy, d.value


def hpwl_host(netlist: Netlist, chip: Chip, site_x, site_y):
    """total_hpwl (metrics/wirelength.rs:46-51) without a context."""
    sx, sy = np.ascontiguousarray(site_x, np.int32), np.ascontiguousarray(site_y, np.int32)
    v = ctypes.c_int64()
    nl_c, chip_c = netlist.to_c(), chip.to_c()
    check(_abi.lib().eplace_hpwl_host(ctypes.byref(nl_c), ctypes.byref(chip_c), _abi.ptr(sx, ctypes.c_int32),
                                      _abi.ptr(sy, ctypes.c_int32), ctypes.byref(v)))
    return int(v.value)


def pin_weights(netlist: Netlist, chip: Chip):
    """compute_pin_weights (placer/common.rs:381-407) without a context: the
    per-cell weights the optimal-transport placer also takes
    (opt_trans_place/mod.rs:110)."""
    w = np.zeros(netlist.num_cells, np.float64)
    nl_c, chip_c = netlist.to_c(), chip.to_c()
    check(_abi.lib().eplace_pin_weights(ctypes.byref(nl_c), ctypes.byref(chip_c), _abi.ptr(w, ctypes.c_double)))
    return w


def initial_placement_host(netlist: Netlist, chip: Chip, seed: int):
    """initial_placement (placer/common.rs:27-117) without a context."""
    n = netlist.num_cells
    sx, sy = np.zeros(n, np.int32), np.zeros(n, np.int32)
    nl_c, chip_c = netlist.to_c(), chip.to_c()
    check(_abi.lib().eplace_initial_placement_host(ctypes.byref(nl_c), ctypes.byref(chip_c), seed,
                                                   _abi.ptr(sx, ctypes.c_int32), _abi.ptr(sy, ctypes.c_int32)))
    return sx, sy


# ---------------------------------------------------------------------------
# Reference entry points
# ---------------------------------------------------------------------------
# ---------------------------------------------------------------------------
# Job engine (eplace_server_*): many jobs on one GPU, continuously batched
# ---------------------------------------------------------------------------
@dataclass
class JobInfo:
    queued_seconds: float
    run_seconds: float
    latency_seconds: float
    footprint_bytes: int


class JobServer:
    """Placement jobs admitted by device footprint and run concurrently on
    one GPU (include/eplace.h, job engine).  submit() copies the inputs and
    returns at once; wait() returns the PlacementResult, equal to
    place_electro's on the same inputs."""

    def __init__(self, device: int = 0, max_jobs: int = 16, hbm_budget: int = 0, legal_threads: int = 0,
                 opts: Optional[RunOptions] = None):
        self.handle = None
        self._lib = _abi.lib()
        c = _abi.ServerCfg()
        self._lib.eplace_server_cfg_default(ctypes.byref(c))
        c.device, c.max_jobs, c.hbm_budget, c.legal_threads = device, max_jobs, hbm_budget, legal_threads
        c.opts = (opts or RunOptions()).to_c()
        h = ctypes.c_void_p()
        check(self._lib.eplace_server_create(ctypes.byref(c), ctypes.byref(h)))
        self.handle = h
        self._meta = {}

    def submit(self, netlist: Netlist, chip: Chip, cfg: Optional[ElectroPlaceCfg] = None) -> int:
        cfg = cfg or ElectroPlaceCfg()
        nl_c, chip_c, cc = netlist.to_c(), chip.to_c(), cfg.to_c()
        jid = ctypes.c_uint64()
        check(self._lib.eplace_server_submit(self.handle, ctypes.byref(nl_c), ctypes.byref(chip_c), ctypes.byref(cc),
                                             ctypes.byref(jid)))
        self._meta[jid.value] = (netlist.num_cells, chip.width, _traj_cap(cfg))
        return jid.value

    def wait(self, job_id: int, timeout_ms: int = -1):
        """(PlacementResult, JobInfo), or None while the job is still running
        (timeout_ms >= 0).  Raises the job's PlacerError / EplaceError."""
        n, width, cap = self._meta[job_id]
        buf = _ResultBuffers(n, width, cap)
        info = _abi.JobInfo()
        st = self._lib.eplace_server_wait(self.handle, job_id, timeout_ms, ctypes.byref(buf.c), ctypes.byref(info))
        if st == _abi.EPLACE_PENDING:
            return None
        del self._meta[job_id]
        check(st)
        return buf.result(), JobInfo(info.queued_seconds, info.run_seconds, info.latency_seconds,
                                     int(info.footprint_bytes))

    def stats(self):
        s = _abi.ServerStats()
        check(self._lib.eplace_server_stats_get(self.handle, ctypes.byref(s)))
        return {k: (float if t is ctypes.c_double else int)(getattr(s, k)) for k, t in _abi.ServerStats._fields_}

    def close(self):
        if self.handle:
            self._lib.eplace_server_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def footprint(netlist: Netlist, chip: Chip) -> int:
    """Admission estimate of a job's device bytes (eplace_footprint)."""
    nl_c, chip_c = netlist.to_c(), chip.to_c()
    return int(_abi.lib().eplace_footprint(ctypes.byref(nl_c), ctypes.byref(chip_c)))


def place_electro(netlist: Netlist, chip: Chip, cfg: Optional[ElectroPlaceCfg] = None,
                  opts: Optional[RunOptions] = None, device: int = 0) -> PlacementResult:
    """place_electro (electro_place/mod.rs:65-204) through the C ABI's
    one-shot eplace_place: host buffers in, BEL bindings out."""
    cfg = cfg or ElectroPlaceCfg()
    opts = opts or RunOptions()
    L = _abi.lib()
    nl_c, chip_c, cc, oc = netlist.to_c(), chip.to_c(), cfg.to_c(), opts.to_c()
    buf = _ResultBuffers(netlist.num_cells, chip.width, _traj_cap(cfg))
    check(L.eplace_place(ctypes.byref(nl_c), ctypes.byref(chip_c), ctypes.byref(cc), ctypes.byref(oc), device,
                         ctypes.byref(buf.c)))
    return buf.result()


def lock_others(netlist: Netlist, cells: Sequence[int]):
    """with_locked_others (placer/common.rs:502-530) on the flat form: every
    bound movable cell outside `cells` becomes a fixed cell on its logic BEL.
    Returns (sub_netlist, target_ids)."""
    n = netlist.num_cells
    target = np.unique(np.asarray(cells, np.int64))
    if target.size and (target.min() < 0 or target.max() >= n):
        raise ValueError("cell index out of range")
    is_t = np.zeros(n, bool)
    is_t[target] = True
    ix = netlist.cell_init_x if netlist.cell_init_x is not None else np.full(n, -1, np.int32)
    iy = netlist.cell_init_y if netlist.cell_init_y is not None else np.full(n, -1, np.int32)
    others = np.nonzero(~is_t)[0]
    bound = others[ix[others] >= 0]
    unbound_others = others[ix[others] < 0]
    if unbound_others.size:
        # The reference would place them too (they are not locked); the flat
        # form cannot express "movable but outside the set", so refuse.
        raise PlacementFailed("cells outside the target set must be bound")
    new_id = np.full(n + netlist.num_fixed, -1, np.int64)
    new_id[target] = np.arange(target.size)
    nt = target.size
    new_id[bound] = nt + netlist.num_fixed + np.arange(bound.size)
    new_id[n:] = nt + np.arange(netlist.num_fixed)
    fol = netlist.fixed_on_logic if netlist.fixed_on_logic is not None else np.zeros(netlist.num_fixed, np.uint8)
    sub = Netlist(
        num_cells=int(nt),
        net_offsets=netlist.net_offsets,
        pin_cell=new_id[netlist.pin_cell].astype(np.uint32),
        fixed_x=np.concatenate([netlist.fixed_x, ix[bound]]),
        fixed_y=np.concatenate([netlist.fixed_y, iy[bound]]),
        cell_w=None if netlist.cell_w is None else netlist.cell_w[target],
        cell_h=None if netlist.cell_h is None else netlist.cell_h[target],
        cell_init_x=ix[target],
        cell_init_y=iy[target],
        fixed_on_logic=np.concatenate([fol, np.ones(bound.size, np.uint8)]),
        net_has_driver=netlist.net_has_driver,
    )
    return sub, target


class PlacerElectro:
    """impl Placer for PlacerElectro (electro_place/mod.rs:45-63)."""

    def place(self, netlist: Netlist, chip: Chip, cfg: Optional[ElectroPlaceCfg] = None, **kw) -> PlacementResult:
        return place_electro(netlist, chip, cfg, **kw)

    def place_cells(self, netlist: Netlist, chip: Chip, cfg: Optional[ElectroPlaceCfg], cells: Sequence[int], **kw):
        """Places only `cells`; every other bound cell is held fixed.  Returns
        bel_tile for all cells of `netlist` (others unchanged)."""
        sub, target = lock_others(netlist, cells)
        r = place_electro(sub, chip, cfg, **kw)
        n = netlist.num_cells
        ix = netlist.cell_init_x if netlist.cell_init_x is not None else np.full(n, -1, np.int32)
        iy = netlist.cell_init_y if netlist.cell_init_y is not None else np.full(n, -1, np.int32)
        tiles = np.where(ix >= 0, iy * chip.width + ix, -1).astype(np.int32)
        tiles[target] = r.bel_tile
        return tiles, r


def place(netlist: Netlist, chip: Chip, *, placer="electro", seed=1, max_iters=None, **_ignored):
    """Context.place (npnr-python/src/lib.rs:224-245, :293-302): the electro
    arm builds ElectroPlaceCfg::default(), overrides seed and max_iters only,
    and maps PlacerError to RuntimeError("ElectroPlace error: ...")."""
    if placer != "electro":
        raise ValueError("Unknown placer: %s. Available: electro" % placer)
    cfg = ElectroPlaceCfg(seed=seed)
    if max_iters is not None:
        cfg.max_iters = max_iters
    try:
        return place_electro(netlist, chip, cfg)
    except PlacerError as e:
        raise RuntimeError("ElectroPlace error: %s" % e) from e
