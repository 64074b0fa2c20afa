"""B200-native Lagrangian-remap timestep of Lare3d (sm_100a CUDA behind a C ABI)."""
from .abi import (BC_OPEN, BC_PERIODIC, BC_USER, LareError, LareParams, LareScalars,  # noqa: F401
                  Simulation, State, default_params)
