"""B200-native (sm_100a) implementation of CRUNA's direct and adjoint compressible Navier-Stokes
time step behind a C ABI (include/cruna_b200.h, libcruna_b200.so)."""
from .cruna import Cruna, CrunaError, Settings, load_library  # noqa: F401

__all__ = ["Cruna", "CrunaError", "Settings", "load_library"]
