"""B200-native FP64 CUDA implementation of BOXZYHYDRO's hydrodynamic step."""
from .params import HydroParams, read_namelist  # noqa: F401
