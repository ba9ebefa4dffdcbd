"""ctypes mirror of include/eplace.h and the loader of libeplace.so.

The shared library is the product: if it is missing or fails to load, every
entry point raises -- there is no Python or CPU fallback.
"""

import ctypes
import os

import numpy as np

# The library runs long legalisation kernels and several jobs on separate
# streams.  With the driver's default of 8 hardware work queues, streams
# share queues and a short kernel can wait behind a long one of another
# stream; 32 queues keep them independent.  Read once, when the process
# creates its CUDA context, so it must be set before any CUDA use.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libeplace.so")

EPLACE_OK = 0
EPLACE_ERR_NO_BELS = 1
EPLACE_ERR_PLACEMENT_FAILED = 2
EPLACE_ERR_INITIAL_PLACEMENT = 3
EPLACE_ERR_INVALID = 4
EPLACE_ERR_OOM = 5
EPLACE_ERR_CUDA = 6
EPLACE_ERR_TIMEOUT = 7
EPLACE_ERR_NO_DEVICE = 8
EPLACE_PENDING = 9

EPLACE_DCT_FP32_SIMT = 0
EPLACE_DCT_BF16X3_TC = 1
EPLACE_DCT_FP32_FFT = 2

EPLACE_FIELD_REFERENCE = 0
EPLACE_FIELD_POTENTIAL_GRADIENT = 1
EPLACE_LEGAL_HOST = 0
EPLACE_LEGAL_GPU = 1

P = ctypes.POINTER
c_u8p = P(ctypes.c_uint8)
c_i32p = P(ctypes.c_int32)
c_u32p = P(ctypes.c_uint32)
c_f32p = P(ctypes.c_float)
c_f64p = P(ctypes.c_double)
c_i64p = P(ctypes.c_int64)


class Cfg(ctypes.Structure):
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


class Opts(ctypes.Structure):
    _fields_ = [
        ("dct_mode", ctypes.c_int32),
        ("legal_threads", ctypes.c_int32),
        ("use_graphs", ctypes.c_int32),
        ("verbose", ctypes.c_int32),
        ("max_inflight", ctypes.c_int32),
        ("field_mode", ctypes.c_int32),
        ("legal_mode", ctypes.c_int32),
        ("wait_limit_us", ctypes.c_int32),
    ]


class Chip(ctypes.Structure):
    _fields_ = [
        ("width", ctypes.c_int32),
        ("height", ctypes.c_int32),
        ("bins_x", ctypes.c_int32),
        ("bins_y", ctypes.c_int32),
    ]


class Netlist(ctypes.Structure):
    _fields_ = [
        ("num_cells", ctypes.c_uint32),
        ("num_fixed", ctypes.c_uint32),
        ("num_nets", ctypes.c_uint32),
        ("cell_w", c_u8p),
        ("cell_h", c_u8p),
        ("cell_init_x", c_i32p),
        ("cell_init_y", c_i32p),
        ("fixed_x", c_i32p),
        ("fixed_y", c_i32p),
        ("fixed_on_logic", c_u8p),
        ("net_offsets", c_u32p),
        ("pin_cell", c_u32p),
        ("net_has_driver", c_u8p),
    ]


class TrajEntry(ctypes.Structure):
    _fields_ = [
        ("iter", ctypes.c_int32),
        ("pad_", ctypes.c_int32),
        ("hpwl", ctypes.c_double),
        ("displacement", ctypes.c_double),
        ("step_x", ctypes.c_double),
        ("step_y", ctypes.c_double),
        ("density_penalty", ctypes.c_double),
        ("overlap", ctypes.c_double),
    ]


class Result(ctypes.Structure):
    _fields_ = [
        ("bel_tile", c_i32p),
        ("bel_index", c_i32p),
        ("x", c_f32p),
        ("y", c_f32p),
        ("traj", P(TrajEntry)),
        ("traj_capacity", ctypes.c_uint32),
        ("traj_len", ctypes.c_uint32),
        ("hpwl", ctypes.c_int64),
        ("overlap", ctypes.c_double),
        ("iters", ctypes.c_uint32),
        ("best_iter", ctypes.c_int32),
        ("converged", ctypes.c_uint8),
        ("gpu_seconds", ctypes.c_double),
        ("total_seconds", ctypes.c_double),
        ("gpu_launches", ctypes.c_uint64),
        ("h2d_bytes", ctypes.c_uint64),
        ("d2h_bytes", ctypes.c_uint64),
    ]


class SynthSpec(ctypes.Structure):
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


class SynthInfo(ctypes.Structure):
    _fields_ = [("num_pins", ctypes.c_uint32), ("max_degree", ctypes.c_uint32)]


class ServerCfg(ctypes.Structure):
    _fields_ = [
        ("device", ctypes.c_int32),
        ("max_jobs", ctypes.c_int32),
        ("hbm_budget", ctypes.c_uint64),
        ("legal_threads", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("opts", Opts),
    ]


class JobInfo(ctypes.Structure):
    _fields_ = [
        ("queued_seconds", ctypes.c_double),
        ("run_seconds", ctypes.c_double),
        ("latency_seconds", ctypes.c_double),
        ("footprint_bytes", ctypes.c_uint64),
    ]


class ServerStats(ctypes.Structure):
    _fields_ = [
        ("submitted", ctypes.c_uint64),
        ("finished", ctypes.c_uint64),
        ("running", ctypes.c_uint64),
        ("queued", ctypes.c_uint64),
        ("contexts", ctypes.c_uint64),
        ("device_bytes", ctypes.c_uint64),
        ("admit_seconds", ctypes.c_double),
        ("pump_seconds", ctypes.c_double),
        ("idle_seconds", ctypes.c_double),
    ]


# Every exported symbol of the C ABI with its prototype.
PROTOTYPES = {
    "eplace_abi_version": (ctypes.c_int32, []),
    "eplace_cfg_default": (None, [P(Cfg)]),
    "eplace_opts_default": (None, [P(Opts)]),
    "eplace_ctx_create": (ctypes.c_int, [P(Netlist), P(Chip), ctypes.c_int32, P(ctypes.c_void_p)]),
    "eplace_ctx_destroy": (None, [ctypes.c_void_p]),
    "eplace_run": (ctypes.c_int, [ctypes.c_void_p, P(Cfg), P(Opts), P(Result)]),
    "eplace_place": (ctypes.c_int, [P(Netlist), P(Chip), P(Cfg), P(Opts), ctypes.c_int32, P(Result)]),
    "eplace_last_error": (ctypes.c_size_t, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]),
    "eplace_stage_wa_grad": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, c_f32p, c_f32p, c_f32p, c_f32p]),
    "eplace_stage_density": (ctypes.c_int, [ctypes.c_void_p, c_f32p, c_f32p, c_f64p, c_f64p]),
    "eplace_stage_field": (ctypes.c_int, [ctypes.c_void_p, c_f64p, ctypes.c_int32, ctypes.c_int32, c_f32p, c_f32p, c_f32p]),
    "eplace_stage_gather": (ctypes.c_int, [ctypes.c_void_p, c_f32p, c_f32p, c_f32p, c_f32p, c_f32p, c_f32p]),
    "eplace_stage_step": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_uint64] + [c_f32p] * 6 + [c_f32p] * 6 + [c_f64p, c_f64p, c_f32p, c_f32p],
    ),
    "eplace_stage_hpwl": (ctypes.c_int, [ctypes.c_void_p, c_i32p, c_i32p, c_i64p]),
    "eplace_stage_barrier_timeout": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_uint32]),
    "eplace_legalize": (ctypes.c_int, [ctypes.c_void_p, c_f32p, c_f32p, c_i32p, c_i32p, c_f64p]),
    "eplace_ctx_load": (ctypes.c_int, [ctypes.c_void_p, P(Netlist), P(Chip)]),
    "eplace_stage_legalize": (ctypes.c_int, [ctypes.c_void_p, c_f32p, c_f32p, c_i32p, c_i32p, c_f64p, c_i64p]),
    "eplace_profile_stages": (ctypes.c_int, [ctypes.c_void_p, P(Cfg), P(Opts), ctypes.c_uint32, c_f64p]),
    "eplace_legalize_host": (ctypes.c_int, [P(Netlist), P(Chip), c_f32p, c_f32p, c_i32p, c_i32p, c_f64p]),
    "eplace_hpwl_host": (ctypes.c_int, [P(Netlist), P(Chip), c_i32p, c_i32p, c_i64p]),
    "eplace_initial_placement_host": (ctypes.c_int, [P(Netlist), P(Chip), ctypes.c_uint64, c_i32p, c_i32p]),
    "eplace_pin_weights": (ctypes.c_int, [P(Netlist), P(Chip), ctypes.POINTER(ctypes.c_double)]),
    "eplace_stage_initial_placement": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, c_i32p, c_i32p, c_i32p]),
    "eplace_density_noalloc": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
         ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
    ),
    "eplace_server_cfg_default": (None, [P(ServerCfg)]),
    "eplace_server_create": (ctypes.c_int, [P(ServerCfg), P(ctypes.c_void_p)]),
    "eplace_server_destroy": (None, [ctypes.c_void_p]),
    "eplace_server_submit": (ctypes.c_int, [ctypes.c_void_p, P(Netlist), P(Chip), P(Cfg), P(ctypes.c_uint64)]),
    "eplace_server_wait": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int32, P(Result), P(JobInfo)]),
    "eplace_server_stats_get": (ctypes.c_int, [ctypes.c_void_p, P(ServerStats)]),
    "eplace_footprint": (ctypes.c_uint64, [P(Netlist), P(Chip)]),
    "eplace_synth_size": (ctypes.c_int, [P(SynthSpec), P(SynthInfo)]),
    "eplace_synth_fill": (ctypes.c_int, [P(SynthSpec), c_u8p, c_u8p, c_i32p, c_i32p, c_u32p, c_u32p]),
}

_lib = None


def lib():
    """Loads libeplace.so once.  Raises if it is missing: no fallback."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                "libeplace.so is not built (%s); run `python -m eisenjoch_b200.build`" % LIB_PATH
            )
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in PROTOTYPES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def ptr(a, ctype):
    """Pointer to a contiguous numpy array (None passes NULL)."""
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "array must be C-contiguous"
    return a.ctypes.data_as(P(ctype))


def f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def last_error(ctx=None):
    L = lib()
    buf = ctypes.create_string_buffer(1024)
    L.eplace_last_error(ctx, buf, 1024)
    return buf.value.decode(errors="replace")
