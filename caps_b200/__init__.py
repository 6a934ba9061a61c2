"""caps_b200: CAPS's MD force-and-integrate step on one NVIDIA B200.

The product is the C ABI library caps_b200/libcaps_b200.so (include/caps_gpu.h) with hand-written sm_100a kernels;
this package binds it with the reference's own names: Evaluator, EnergyOptions, DynamicsOptions, run_dynamics.
"""
from .engine import (DeviceError, DynamicsCancelled, DynamicsInterrupted, DynamicsOptions, EnergyOptions, Evaluator,  # noqa: F401
                     FieldError, cell_array, request_stop, run_batch, run_dynamics, stop_requested)
from .forcefield import ForceField, read_capsff  # noqa: F401
from .cooling import CoolingOptions, run_cooling  # noqa: F401
from .minimise import MinimiseOptions, minimise  # noqa: F401
from .relax import RelaxOptions, relax  # noqa: F401
from .equilibrate import EquilibrateOptions, ProtocolParams, Stage, equilibrate, parse_protocol, protocol_by_name  # noqa: F401
from .trajectory import TrajectoryWriter, write_trajectory  # noqa: F401

__all__ = ["Evaluator", "EnergyOptions", "DynamicsOptions", "run_dynamics", "run_batch", "ForceField", "read_capsff", "FieldError",
           "DynamicsCancelled", "DeviceError", "cell_array", "CoolingOptions", "run_cooling", "EquilibrateOptions",
           "ProtocolParams", "Stage", "equilibrate", "parse_protocol", "protocol_by_name", "MinimiseOptions",
           "minimise", "DynamicsInterrupted", "request_stop", "stop_requested", "TrajectoryWriter", "write_trajectory", "RelaxOptions", "relax"]
