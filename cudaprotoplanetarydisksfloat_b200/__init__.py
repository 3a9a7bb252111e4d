"""B200-native FARGO / FARGO_ADSG disk-hydro timestep (drop-in for the hot path of
MatiasFloresS/CudaProtoplanetaryDisksFloat).  The computation lives in
libfargo_b200.so (hand-written sm_100a kernels behind the C ABI of
include/fargo_b200.h); importing this package loads it and fails loudly if it
is missing."""
from . import _abi  # noqa: F401  (loads libfargo_b200.so)
from .disk import Batch, Disk, grid_radii, planets_dict, read_params, read_planets  # noqa: F401

__all__ = ["Disk", "Batch", "read_params", "read_planets", "grid_radii", "planets_dict"]
