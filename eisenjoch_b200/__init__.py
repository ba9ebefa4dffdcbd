"""B200-native (sm_100a) ElectroPlace hot path.

The computation lives in libeplace.so (CUDA kernels + C ABI, include/eplace.h);
this package is the host-side mirror of the reference placer interface.
"""

from ._abi import LIB_PATH, lib  # noqa: F401
from .placer import (  # noqa: F401
    WORKLOADS,
    Chip,
    ElectroPlaceCfg,
    EplaceError,
    InitialPlacementFailed,
    Netlist,
    NoBelsAvailable,
    PlacementContext,
    PlacementFailed,
    PlacementResult,
    PlacerElectro,
    PlacerError,
    RunOptions,
    SynthSpec,
    lock_others,
    place,
    place_electro,
    synth_netlist,
    workload,
)
