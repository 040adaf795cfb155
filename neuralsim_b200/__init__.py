"""neuralsim_b200 — B200 step backend for NeuralSim's per-timestep hot path.

The compute path is libneuralsim.so (hand-written sm_100a CUDA behind the C
ABI in include/neuralsim.h); this package is the Python host mirror of the
reference crate's engine API on top of it.
"""
from . import _abi
from ._abi import NsError
from .engine import Drive, Network, SimConfig, SimulationEngine, StepResult, device_count

__all__ = ["Drive", "Network", "SimConfig", "SimulationEngine", "StepResult", "NsError",
           "device_count", "load_library"]


def load_library():
    """Loads libneuralsim.so (raises ImportError if it was not built)."""
    return _abi.load()
