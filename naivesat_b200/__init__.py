"""naivesat_b200: exhaustive Gate-circuit search (SAT, QSAT, SATOSTOP) on B200.

The solver itself is the C ABI in include/nsat.h (libnsat.so, sm_100a kernels
specialised per circuit by NVRTC).  `api` is its ctypes binding and
`workloads` builds the seeded benchmark circuits.
"""
from . import api, workloads  # noqa: F401
