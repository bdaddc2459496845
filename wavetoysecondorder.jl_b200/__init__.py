"""wavetoy_b200 -- B200 (sm_100a) implementation of WaveToySecondOrder.jl's 3D
SBP-SAT right-hand side and RK4 time step.

The numerics live in libwavetoy_b200.so (CUDA kernels behind the C ABI of
include/wavetoy_b200.h); this package is the Python mirror of the reference's
Julia API (wavetoy.py), the seeded workloads (workloads.py), the serving loop
over batched solves (serve.py), one solve split into z-slabs with halo
exchanges (slabs.py) and the build step (build.py).  The directory name
contains a dot, so load it with importlib under the module name
"wavetoy_b200" (see tests/conftest.py).
"""
from .wavetoy import *  # noqa: F401,F403
from .wavetoy import library, LIB_PATH  # noqa: F401
from . import workloads  # noqa: F401
from . import build  # noqa: F401
from . import serve  # noqa: F401
from . import slabs  # noqa: F401
