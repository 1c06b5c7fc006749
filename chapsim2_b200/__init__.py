"""B200-native CHAPSim2 per-timestep DNS hot path.

The product is the C-ABI library ``libchapsim_gpu.so`` (sm_100a CUDA kernels
behind the entry points declared in include/chapsim_gpu.h).  This package is
the Python host side: configuration, initial fields and a ctypes binding whose
calls mirror the reference's Fortran interface.
"""
from . import config, initial  # noqa: F401
