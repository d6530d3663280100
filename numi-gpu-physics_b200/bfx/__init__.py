"""bfx: B200-native D3Q19 moving-boundary lattice-Boltzmann step.

Host-side mirror of BirdFlowMetal's solver interface over the CUDA library
libbfx.so (include/bfx.h).  There is no CPU execution path: every simulation
runs through the library, and constructing one without the built library or
without a CUDA device raises ``BirdFlowError``.
"""
from . import _lib as lib
from .config import (BirdBodyState, BirdFlowConfigurationError, BirdParameters, GridSize, LatticeScaling,
                     SimulationConfiguration, WingInertialProperties, WingKinematics)
from .simulation import AdvanceResult, BirdFlowError, BirdFlowSimulation, Lattice, default_config

__all__ = [
    "lib", "BirdBodyState", "BirdFlowConfigurationError", "BirdParameters", "GridSize", "LatticeScaling",
    "SimulationConfiguration", "WingInertialProperties", "WingKinematics", "AdvanceResult", "BirdFlowError",
    "BirdFlowSimulation", "Lattice", "default_config",
]
