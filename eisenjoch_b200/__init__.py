"""B200-native (sm_100a) ElectroPlace hot path.

The computation lives in libeplace.so (CUDA kernels + C ABI, include/eplace.h);
this package is the host-side mirror of the reference placer interface.
"""

from . import frontend  # noqa: F401
from ._abi import LIB_PATH, lib  # noqa: F401
from .placer import (  # noqa: F401
    WORKLOADS,
    Chip,
    ElectroPlaceCfg,
    EplaceError,
    InitialPlacementFailed,
    JobInfo,
    JobServer,
    Netlist,
    NoBelsAvailable,
    PlacementContext,
    PlacementFailed,
    PlacementResult,
    PlacerElectro,
    PlacerError,
    RunOptions,
    SynthSpec,
    batched_specs,
    footprint,
    hpwl_host,
    pin_weights,
    initial_placement_host,
    legalize_host,
    lock_others,
    mixed_job_spec,
    mixed_job_specs,
    place,
    place_electro,
    served_stream,
    synth_netlist,
    workload,
)
