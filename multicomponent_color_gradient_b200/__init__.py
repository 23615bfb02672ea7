"""B200-native D3Q27 colour-gradient lattice Boltzmann step (drop-in for the
per-step path of Felipe-Aristi/Multicomponent_Color_Gradient).

The compute path is libmcg.so (hand-written sm_100a CUDA behind the C ABI in
include/mcg.h); this package is the Python host mirror of the reference's
launch interface.
"""
from .cases import CASES, derive, get_case  # noqa: F401
from .solver import Q, CX, CY, CZ, Solver, device_count, params_struct, write_constants_header  # noqa: F401
from ._lib import McgError, load as load_library  # noqa: F401

__all__ = ["CASES", "derive", "get_case", "Solver", "Q", "CX", "CY", "CZ", "device_count", "params_struct",
           "write_constants_header", "McgError", "load_library"]
