"""ctypes binding of the FP64 CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: the parity checker for the CUDA path and the
timed CPU baseline.  Only tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline / reference arm import this module; the product package never
does.

Each method names the reference function it restates (paths relative to
the reference project root, crates/nextpnr/src/...).  Inputs are any object
with the Netlist / Chip attributes of eisenjoch_b200.placer (duck-typed, so
this module does not import the product).
"""

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liboracle.so")

P = ctypes.POINTER


class _Problem(ctypes.Structure):
    _fields_ = [
        ("width", ctypes.c_int32),
        ("height", ctypes.c_int32),
        ("bins_x", ctypes.c_int32),
        ("bins_y", ctypes.c_int32),
        ("num_cells", ctypes.c_uint32),
        ("num_fixed", ctypes.c_uint32),
        ("num_nets", ctypes.c_uint32),
        ("cell_w", P(ctypes.c_uint8)),
        ("cell_h", P(ctypes.c_uint8)),
        ("cell_init_x", P(ctypes.c_int32)),
        ("cell_init_y", P(ctypes.c_int32)),
        ("fixed_x", P(ctypes.c_int32)),
        ("fixed_y", P(ctypes.c_int32)),
        ("fixed_on_logic", P(ctypes.c_uint8)),
        ("net_offsets", P(ctypes.c_uint32)),
        ("pin_cell", P(ctypes.c_uint32)),
        ("net_has_driver", P(ctypes.c_uint8)),
    ]


class _Cfg(ctypes.Structure):
    _fields_ = [
        ("seed", ctypes.c_uint64),
        ("wl_coeff", ctypes.c_double),
        ("target_util", ctypes.c_double),
        ("timing_driven", ctypes.c_uint8),
        ("target_density", ctypes.c_double),
        ("timing_weight", ctypes.c_double),
        ("nesterov_step_size", ctypes.c_double),
        ("max_iters", ctypes.c_uint64),
        ("legalize_interval", ctypes.c_uint64),
    ]


class _Traj(ctypes.Structure):
    _fields_ = [
        ("iter", ctypes.c_int32),
        ("hpwl", ctypes.c_double),
        ("displacement", ctypes.c_double),
        ("step_x", ctypes.c_double),
        ("step_y", ctypes.c_double),
        ("density_penalty", ctypes.c_double),
        ("overlap", ctypes.c_double),
    ]


class _Result(ctypes.Structure):
    _fields_ = [
        ("site_x", P(ctypes.c_int32)),
        ("site_y", P(ctypes.c_int32)),
        ("best_x", P(ctypes.c_double)),
        ("best_y", P(ctypes.c_double)),
        ("traj", P(_Traj)),
        ("traj_capacity", ctypes.c_uint32),
        ("traj_len", ctypes.c_uint32),
        ("hpwl", ctypes.c_int64),
        ("final_overlap", ctypes.c_double),
        ("iters", ctypes.c_uint32),
        ("best_iter", ctypes.c_int32),
        ("converged", ctypes.c_int),
        ("overlap_trace_last", ctypes.c_double),
        ("first_nonfinite_grad_iter", ctypes.c_int32),
    ]


class _Nest(ctypes.Structure):
    _fields_ = [
        ("x", P(ctypes.c_double)),
        ("x_prev", P(ctypes.c_double)),
        ("n", ctypes.c_size_t),
        ("step_size", ctypes.c_double),
        ("iter", ctypes.c_uint64),
        ("a", ctypes.c_double),
    ]


class _State(ctypes.Structure):
    _fields_ = [
        ("sx", _Nest),
        ("sy", _Nest),
        ("prev_grad", P(ctypes.c_double)),
        ("density_penalty", ctypes.c_double),
        ("density_initialized", ctypes.c_int),
    ]


class _SynthSpec(ctypes.Structure):
    _fields_ = [
        ("seed", ctypes.c_uint64),
        ("num_cells", ctypes.c_uint32),
        ("num_nets", ctypes.c_uint32),
        ("num_pads", ctypes.c_uint32),
        ("width", ctypes.c_int32),
        ("height", ctypes.c_int32),
        ("bins_x", ctypes.c_int32),
        ("bins_y", ctypes.c_int32),
        ("cluster_size", ctypes.c_uint32),
        ("locality", ctypes.c_double),
        ("macro_fraction", ctypes.c_double),
        ("macro_min", ctypes.c_uint32),
        ("macro_max", ctypes.c_uint32),
    ]


_lib = None


def build():
    """Compiles liboracle.so with the committed Makefile (gcc only)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        srcs = [os.path.join(_HERE, f) for f in ("eplace_oracle.c", "orc_synth.c", "eplace_oracle.h")]
        if not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < max(map(os.path.getmtime, srcs)):
            build()
        L = ctypes.CDLL(LIB_PATH)
        d, i32, u64, f64p = ctypes.c_double, ctypes.c_int32, ctypes.c_uint64, P(ctypes.c_double)
        L.orc_rng_next.restype = u64
        L.orc_rng_next.argtypes = [P(u64)]
        L.orc_rng_shuffle_i32.argtypes = [P(u64), P(i32), ctypes.c_size_t]
        L.orc_initial_placement.restype = ctypes.c_int
        L.orc_initial_placement.argtypes = [P(_Problem), u64, P(i32), P(i32)]
        L.orc_pin_weights.argtypes = [P(_Problem), f64p]
        L.orc_wa_axis_value.restype = d
        L.orc_wa_axis_value.argtypes = [f64p, ctypes.c_size_t, d]
        L.orc_wa_axis_grad.argtypes = [f64p, ctypes.c_size_t, d, f64p]
        L.orc_wa_gradient.argtypes = [P(_Problem), f64p, f64p, d, f64p, f64p]
        L.orc_density.argtypes = [P(_Problem), f64p, f64p, f64p]
        L.orc_overlap.restype = d
        L.orc_overlap.argtypes = [f64p, ctypes.c_size_t, d]
        for fn in ("orc_dct2", "orc_dct3", "orc_dst3"):
            getattr(L, fn).argtypes = [f64p, ctypes.c_size_t, ctypes.c_int]
        L.orc_field.restype = ctypes.c_int
        L.orc_field.argtypes = [f64p, i32, i32, d, ctypes.c_int, f64p, f64p, f64p]
        L.orc_potential.restype = ctypes.c_int
        L.orc_potential.argtypes = [f64p, i32, i32, ctypes.c_int, f64p]
        L.orc_gather.argtypes = [P(_Problem), f64p, f64p, f64p, f64p, f64p, f64p]
        L.orc_legalize.restype = ctypes.c_int
        L.orc_legalize.argtypes = [P(_Problem), f64p, f64p, ctypes.c_int, P(i32), P(i32), f64p]
        L.orc_hpwl.restype = ctypes.c_int64
        L.orc_hpwl.argtypes = [P(_Problem), P(i32), P(i32)]
        L.orc_place.restype = ctypes.c_int
        L.orc_place.argtypes = [P(_Problem), P(_Cfg), ctypes.c_int, ctypes.c_int, P(_Result), f64p]
        L.orc_set_field_mode.argtypes = [ctypes.c_int]
        L.orc_set_wa_mode.argtypes = [ctypes.c_int]
        L.orc_cfg_default.argtypes = [P(_Cfg)]
        L.orc_synth.restype = ctypes.c_int
        L.orc_synth.argtypes = [P(_SynthSpec), P(ctypes.c_uint32), P(ctypes.c_uint8), P(ctypes.c_uint8), P(i32),
                                P(i32), P(ctypes.c_uint32), P(ctypes.c_uint32)]
        L.orc_step.argtypes = [P(_Problem), P(_State), u64, f64p, f64p, f64p, d, d, f64p]
        L.orc_nesterov_init.argtypes = [P(_Nest), f64p, f64p, ctypes.c_size_t, d]
        L.orc_nesterov_set_positions.argtypes = [P(_Nest), f64p]
        L.orc_nesterov_momentum.restype = d
        L.orc_nesterov_momentum.argtypes = [P(_Nest)]
        L.orc_nesterov_look_ahead.argtypes = [P(_Nest), f64p]
        L.orc_nesterov_step.restype = d
        L.orc_nesterov_step.argtypes = [P(_Nest), f64p]
        L.orc_nesterov_clamp.argtypes = [P(_Nest), d, d]
        L.orc_nesterov_adaptive_restart.argtypes = [P(_Nest), f64p]
        L.orc_nesterov_lipschitz.restype = d
        L.orc_nesterov_lipschitz.argtypes = [P(_Nest), f64p, f64p]
        L.orc_nesterov_bb.restype = ctypes.c_int
        L.orc_nesterov_bb.argtypes = [P(_Nest), f64p, f64p, f64p]
        _lib = L
    return _lib


def _p(a, t):
    return None if a is None else a.ctypes.data_as(P(t))


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64)


# --- benchmark inputs -------------------------------------------------------
class FlatNetlist:
    """The flat netlist the oracle takes (the attributes of the product's
    Netlist, without importing it)."""

    def __init__(self, num_cells, net_offsets, pin_cell, fixed_x, fixed_y, cell_w=None, cell_h=None):
        self.num_cells = int(num_cells)
        self.net_offsets, self.pin_cell = net_offsets, pin_cell
        self.fixed_x, self.fixed_y = fixed_x, fixed_y
        self.cell_w, self.cell_h = cell_w, cell_h
        self.cell_init_x = self.cell_init_y = self.fixed_on_logic = self.net_has_driver = None

    @property
    def num_fixed(self):
        return int(self.fixed_x.size)

    @property
    def num_nets(self):
        return int(self.net_offsets.size - 1)

    @property
    def num_pins(self):
        return int(self.net_offsets[-1])


class FlatChip:
    def __init__(self, width, height, bins_x=0, bins_y=0):
        self.width, self.height, self.bins_x, self.bins_y = width, height, bins_x, bins_y


class Cfg:
    """ElectroPlaceCfg (electro_place/config.rs:5-40): the nine fields with
    the defaults of ElectroPlaceCfg::default() (config.rs:29-40), from the
    C restatement, then `overrides`."""

    def __init__(self, **overrides):
        c = _Cfg()
        lib().orc_cfg_default(ctypes.byref(c))
        for name, _ in _Cfg._fields_:
            setattr(self, name, getattr(c, name))
        for k, v in overrides.items():
            if not hasattr(self, k):
                raise AttributeError(k)
            setattr(self, k, v)


def synth(spec):
    """The seeded benchmark netlist of `spec` (any object with the fields of
    _SynthSpec), generated by the oracle's own copy of the generator.
    Returns (FlatNetlist, FlatChip)."""
    s = _SynthSpec()
    for name, _ in _SynthSpec._fields_:
        setattr(s, name, getattr(spec, name))
    L = lib()
    npins = ctypes.c_uint32()
    assert L.orc_synth(ctypes.byref(s), ctypes.byref(npins), None, None, None, None, None, None) == 0
    n, nn, f = spec.num_cells, spec.num_nets, spec.num_pads
    cw, ch = np.ones(n, np.uint8), np.ones(n, np.uint8)
    fx, fy = np.zeros(f, np.int32), np.zeros(f, np.int32)
    off, pins = np.zeros(nn + 1, np.uint32), np.zeros(npins.value, np.uint32)
    assert L.orc_synth(ctypes.byref(s), ctypes.byref(npins), _p(cw, ctypes.c_uint8), _p(ch, ctypes.c_uint8),
                       _p(fx, ctypes.c_int32), _p(fy, ctypes.c_int32), _p(off, ctypes.c_uint32),
                       _p(pins, ctypes.c_uint32)) == 0
    macro = spec.macro_fraction > 0
    nl = FlatNetlist(n, off, pins, fx, fy, cw if macro else None, ch if macro else None)
    return nl, FlatChip(spec.width, spec.height, spec.bins_x, spec.bins_y)


# --- transforms and WA on plain arrays -------------------------------------
def dct2(v, backend=1):
    """rustdct DCT-II (density.rs:211-229 calls it per row / column)."""
    v = _d(v).copy()
    lib().orc_dct2(_p(v, ctypes.c_double), v.size, backend)
    return v


def dct3(v, backend=1):
    v = _d(v).copy()
    lib().orc_dct3(_p(v, ctypes.c_double), v.size, backend)
    return v


def dst3(v, backend=1):
    v = _d(v).copy()
    lib().orc_dst3(_p(v, ctypes.c_double), v.size, backend)
    return v


def wa_axis_value(coords, coeff):
    """wa_axis_value (solver/wa.rs:17-46)."""
    c = _d(coords)
    return lib().orc_wa_axis_value(_p(c, ctypes.c_double), c.size, coeff)


def wa_axis_grad(coords, coeff):
    """wa_axis_grad (solver/wa.rs:51-101)."""
    c = _d(coords)
    g = np.zeros_like(c)
    lib().orc_wa_axis_grad(_p(c, ctypes.c_double), c.size, coeff, _p(g, ctypes.c_double))
    return g


def wa_wirelength(positions, coeff):
    """wa_wirelength (solver/wa.rs:104-113)."""
    pos = np.asarray(positions, np.float64).reshape(-1, 2)
    if pos.shape[0] < 2:
        return 0.0
    return wa_axis_value(pos[:, 0], coeff) + wa_axis_value(pos[:, 1], coeff)


def overlap_of(d, capacity=1.0):
    """compute_overlap (density.rs:79-86)."""
    d = _d(d).ravel()
    return lib().orc_overlap(_p(d, ctypes.c_double), d.size, capacity)


def rng_sequence(seed, n):
    """DeterministicRng::next_u64 (context/rng.rs:19-31), seed.max(1)."""
    s = ctypes.c_uint64(max(seed, 1))
    return [lib().orc_rng_next(ctypes.byref(s)) for _ in range(n)]


def rng_shuffle(seed, values):
    """DeterministicRng::shuffle (context/rng.rs:52-61)."""
    s = ctypes.c_uint64(max(seed, 1))
    a = np.ascontiguousarray(values, np.int32).copy()
    lib().orc_rng_shuffle_i32(ctypes.byref(s), _p(a, ctypes.c_int32), a.size)
    return a


class NesterovSolver:
    """NesterovSolver (solver/nesterov.rs:12-224) backed by the C restatement."""

    def __init__(self, n, step_size):
        self.xbuf = np.zeros(n)
        self.xpbuf = np.zeros(n)
        self.s = _Nest()
        lib().orc_nesterov_init(ctypes.byref(self.s), _p(self.xbuf, ctypes.c_double),
                                _p(self.xpbuf, ctypes.c_double), n, step_size)

    def set_positions(self, v):
        v = _d(v)
        lib().orc_nesterov_set_positions(ctypes.byref(self.s), _p(v, ctypes.c_double))

    def look_ahead(self):
        y = np.zeros_like(self.xbuf)
        lib().orc_nesterov_look_ahead(ctypes.byref(self.s), _p(y, ctypes.c_double))
        return y

    def step(self, g):
        g = _d(g)
        return lib().orc_nesterov_step(ctypes.byref(self.s), _p(g, ctypes.c_double))

    def clamp_positions_range(self, lo, hi):
        lib().orc_nesterov_clamp(ctypes.byref(self.s), lo, hi)

    def adaptive_restart(self, g):
        g = _d(g)
        lib().orc_nesterov_adaptive_restart(ctypes.byref(self.s), _p(g, ctypes.c_double))

    def lipschitz_step_size(self, pg, cg):
        pg, cg = _d(pg), _d(cg)
        return lib().orc_nesterov_lipschitz(ctypes.byref(self.s), _p(pg, ctypes.c_double), _p(cg, ctypes.c_double))

    def bb_step_size(self, pg, cg):
        pg, cg = _d(pg), _d(cg)
        out = ctypes.c_double()
        ok = lib().orc_nesterov_bb(ctypes.byref(self.s), _p(pg, ctypes.c_double), _p(cg, ctypes.c_double),
                                   ctypes.byref(out))
        return out.value if ok else None

    def positions(self):
        return self.xbuf.copy()

    @property
    def x_prev(self):
        return self.xpbuf.copy()

    @property
    def iter_count(self):
        return int(self.s.iter)

    @property
    def fista_param(self):
        return float(self.s.a)

    @property
    def step_size(self):
        return float(self.s.step_size)


def fista_sequence(k):
    """a_k of the FISTA sequence a_0 = 1, a_{j+1} = (1 + sqrt(1 + 4 a_j^2)) / 2."""
    a = 1.0
    for _ in range(k):
        a = (1.0 + np.sqrt(1.0 + 4.0 * a * a)) / 2.0
    return a


class Oracle:
    """The CPU restatement bound to one problem (netlist + chip)."""

    def __init__(self, netlist, chip):
        self.nl = netlist
        self.chip = chip
        L = lib()
        self._L = L
        p = _Problem()
        p.width, p.height = chip.width, chip.height
        p.bins_x = chip.bins_x or chip.width
        p.bins_y = chip.bins_y or chip.height
        p.num_cells = netlist.num_cells
        p.num_fixed = netlist.num_fixed
        p.num_nets = netlist.num_nets
        self._keep = [netlist.cell_w, netlist.cell_h, netlist.cell_init_x, netlist.cell_init_y, netlist.fixed_x,
                      netlist.fixed_y, netlist.fixed_on_logic, netlist.net_offsets, netlist.pin_cell,
                      netlist.net_has_driver]
        p.cell_w = _p(netlist.cell_w, ctypes.c_uint8)
        p.cell_h = _p(netlist.cell_h, ctypes.c_uint8)
        p.cell_init_x = _p(netlist.cell_init_x, ctypes.c_int32)
        p.cell_init_y = _p(netlist.cell_init_y, ctypes.c_int32)
        p.fixed_x = _p(netlist.fixed_x, ctypes.c_int32)
        p.fixed_y = _p(netlist.fixed_y, ctypes.c_int32)
        p.fixed_on_logic = _p(netlist.fixed_on_logic, ctypes.c_uint8)
        p.net_offsets = _p(netlist.net_offsets, ctypes.c_uint32)
        p.pin_cell = _p(netlist.pin_cell, ctypes.c_uint32)
        p.net_has_driver = _p(netlist.net_has_driver, ctypes.c_uint8)
        self.p = p
        self.bx, self.by = p.bins_x, p.bins_y
        self.n = netlist.num_cells

    @property
    def capacity(self):
        return float((self.chip.width // self.bx) * (self.chip.height // self.by))

    def initial_placement(self, seed):
        """initial_placement (placer/common.rs:27-117)."""
        sx = np.zeros(self.n, np.int32)
        sy = np.zeros(self.n, np.int32)
        st = self._L.orc_initial_placement(ctypes.byref(self.p), seed, _p(sx, ctypes.c_int32), _p(sy, ctypes.c_int32))
        return st, sx, sy

    def pin_weights(self):
        """compute_pin_weights (placer/common.rs:381-407)."""
        w = np.zeros(self.n, np.float64)
        self._L.orc_pin_weights(ctypes.byref(self.p), _p(w, ctypes.c_double))
        return w

    def wa_gradient(self, x, y, coeff=0.5, wa_mode=0):
        """add_wa_wirelength_gradient (placer/common.rs:205-291).  wa_mode 1
        shifts the exponents by the per-net max / min instead of the mean
        (extension: same function, no FP64 overflow on wide nets)."""
        x, y = _d(x), _d(y)
        gx, gy = np.zeros(self.n), np.zeros(self.n)
        self._L.orc_set_wa_mode(wa_mode)
        try:
            self._L.orc_wa_gradient(ctypes.byref(self.p), _p(x, ctypes.c_double), _p(y, ctypes.c_double), coeff,
                                    _p(gx, ctypes.c_double), _p(gy, ctypes.c_double))
        finally:
            self._L.orc_set_wa_mode(0)
        return gx, gy

    def density(self, x, y):
        """compute_concrete_density (density.rs:54-74)."""
        x, y = _d(x), _d(y)
        d = np.zeros((self.by, self.bx))
        self._L.orc_density(ctypes.byref(self.p), _p(x, ctypes.c_double), _p(y, ctypes.c_double),
                            _p(d, ctypes.c_double))
        return d

    def overlap(self, d):
        return overlap_of(d, self.capacity)

    def field(self, d, target_density=1.0, backend=1, want_phi=False, field_mode=0):
        """compute_density_field (density.rs:96-166).  field_mode 1 is the
        potential-gradient extension (not reference behaviour)."""
        d = _d(d).reshape(self.by, self.bx)
        ex, ey = np.zeros_like(d), np.zeros_like(d)
        phi = np.zeros_like(d) if want_phi else None
        self._L.orc_set_field_mode(field_mode)
        try:
            st = self._L.orc_field(_p(d, ctypes.c_double), self.bx, self.by, target_density, backend,
                                   _p(ex, ctypes.c_double), _p(ey, ctypes.c_double), _p(phi, ctypes.c_double))
        finally:
            self._L.orc_set_field_mode(0)
        assert st == 0
        return (ex, ey, phi) if want_phi else (ex, ey)

    def potential(self, phi_hat, backend=1):
        ph = _d(phi_hat).reshape(self.by, self.bx)
        out = np.zeros_like(ph)
        self._L.orc_potential(_p(ph, ctypes.c_double), self.bx, self.by, backend, _p(out, ctypes.c_double))
        return out

    def gather(self, x, y, ex, ey):
        """compute_density_gradient (density.rs:171-206)."""
        x, y, ex, ey = _d(x), _d(y), _d(ex), _d(ey)
        gx, gy = np.zeros(self.n), np.zeros(self.n)
        self._L.orc_gather(ctypes.byref(self.p), _p(x, ctypes.c_double), _p(y, ctypes.c_double),
                           _p(ex, ctypes.c_double), _p(ey, ctypes.c_double), _p(gx, ctypes.c_double),
                           _p(gy, ctypes.c_double))
        return gx, gy

    def legalize(self, x, y, method=1):
        """legalize_electro (electro_place/mod.rs:206-255); method 0 is the
        reference's exhaustive scan, 1 the ring search."""
        x, y = _d(x), _d(y)
        sx, sy = np.zeros(self.n, np.int32), np.zeros(self.n, np.int32)
        disp = ctypes.c_double()
        st = self._L.orc_legalize(ctypes.byref(self.p), _p(x, ctypes.c_double), _p(y, ctypes.c_double), method,
                                  _p(sx, ctypes.c_int32), _p(sy, ctypes.c_int32), ctypes.byref(disp))
        return st, sx, sy, disp.value

    def hpwl(self, sx, sy):
        """total_hpwl (metrics/wirelength.rs:46-51)."""
        sx, sy = np.ascontiguousarray(sx, np.int32), np.ascontiguousarray(sy, np.int32)
        return int(self._L.orc_hpwl(ctypes.byref(self.p), _p(sx, ctypes.c_int32), _p(sy, ctypes.c_int32)))

    def step(self, it, state, gwl_x, gwl_y, gden_x, gden_y, pw=None):
        """Loop body (f)-(i) of electro_place/mod.rs:131-173 on given state.
        state: dict with x, y, x_prev, y_prev, gprev_x, gprev_y (arrays),
        step_x, step_y, density_penalty, initialized, and the solver's FISTA
        position (iteration index `it`).  Returns (state', step norms)."""
        n = self.n
        L = self._L
        xs = [_d(state["x"]).copy(), _d(state["y"]).copy()]
        xps = [_d(state["x_prev"]).copy(), _d(state["y_prev"]).copy()]
        S = _State()
        for k, nm in enumerate(("sx", "sy")):
            ns = getattr(S, nm)
            ns.x = _p(xs[k], ctypes.c_double)
            ns.x_prev = _p(xps[k], ctypes.c_double)
            ns.n = n
            ns.step_size = state["step_x" if k == 0 else "step_y"]
            ns.iter = it
            ns.a = fista_sequence(it)
        prev = np.concatenate([_d(state["gprev_x"]), _d(state["gprev_y"])])
        S.prev_grad = _p(prev, ctypes.c_double)
        S.density_penalty = state["density_penalty"]
        S.density_initialized = int(state["initialized"])
        g = np.concatenate([_d(gwl_x), _d(gwl_y)])
        gd = np.concatenate([_d(gden_x), _d(gden_y)])
        pw = self.pin_weights() if pw is None else _d(pw)
        norms = np.zeros(2)
        L.orc_step(ctypes.byref(self.p), ctypes.byref(S), it, _p(g, ctypes.c_double), _p(gd, ctypes.c_double),
                   _p(pw, ctypes.c_double), float(self.chip.width - 1), float(self.chip.height - 1),
                   _p(norms, ctypes.c_double))
        out = dict(x=xs[0], y=xs[1], x_prev=xps[0], y_prev=xps[1], gprev_x=prev[:n].copy(), gprev_y=prev[n:].copy(),
                   step_x=S.sx.step_size, step_y=S.sy.step_size, density_penalty=S.density_penalty,
                   initialized=bool(S.density_initialized), a=S.sx.a, solver_iter=int(S.sx.iter))
        # next iteration's look-ahead, clamped (mod.rs:105-107)
        la = []
        for k, nm in enumerate(("sx", "sy")):
            y = np.zeros(n)
            L.orc_nesterov_look_ahead(ctypes.byref(getattr(S, nm)), _p(y, ctypes.c_double))
            la.append(np.clip(y, 0.0, float((self.chip.width if k == 0 else self.chip.height) - 1)))
        out["look_x"], out["look_y"] = la
        return out, norms

    def place(self, cfg, dct_backend=1, legal_method=1, want_trace=False, field_mode=0, wa_mode=0):
        """place_electro (electro_place/mod.rs:65-204).  cfg: any object with
        the nine ElectroPlaceCfg fields.  field_mode 1 is the
        potential-gradient extension, wa_mode 1 the overflow-free WA shift
        (both extensions).  Returns (status, dict)."""
        c = _Cfg()
        for name, _ in _Cfg._fields_:
            setattr(c, name, getattr(cfg, name))
        n = self.n
        sx, sy = np.zeros(n, np.int32), np.zeros(n, np.int32)
        bx, by = np.zeros(n), np.zeros(n)
        cap = int(cfg.max_iters // max(1, cfg.legalize_interval) + 2)
        traj = (_Traj * cap)()
        r = _Result()
        r.site_x, r.site_y = _p(sx, ctypes.c_int32), _p(sy, ctypes.c_int32)
        r.best_x, r.best_y = _p(bx, ctypes.c_double), _p(by, ctypes.c_double)
        r.traj = ctypes.cast(traj, P(_Traj))
        r.traj_capacity = cap
        trace = np.zeros(max(1, int(cfg.max_iters))) if want_trace else None
        self._L.orc_set_field_mode(field_mode)
        self._L.orc_set_wa_mode(wa_mode)
        try:
            st = self._L.orc_place(ctypes.byref(self.p), ctypes.byref(c), dct_backend, legal_method,
                                   ctypes.byref(r), _p(trace, ctypes.c_double))
        finally:
            self._L.orc_set_field_mode(0)
            self._L.orc_set_wa_mode(0)
        out = dict(
            site_x=sx, site_y=sy, best_x=bx, best_y=by, hpwl=int(r.hpwl), iters=int(r.iters),
            best_iter=int(r.best_iter), converged=bool(r.converged), final_overlap=r.final_overlap,
            first_nonfinite_grad_iter=int(r.first_nonfinite_grad_iter),
            trajectory=[dict(iter=traj[k].iter, hpwl=traj[k].hpwl, disp=traj[k].displacement,
                             step_x=traj[k].step_x, step_y=traj[k].step_y,
                             density_penalty=traj[k].density_penalty, overlap=traj[k].overlap)
                        for k in range(r.traj_len)],
        )
        if want_trace:
            out["overlap_trace"] = trace[: r.iters]
        return st, out
