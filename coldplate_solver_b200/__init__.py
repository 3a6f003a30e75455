"""B200-native (sm_100a) implementation of one SIMPLE outer iteration of the
coldplate-solver reference: U/V momentum assembly with FOU/SOU deferred
correction, Brinkman penalisation and the 2.5-D model, implicit Jacobi
momentum sweeps, a matrix-free Jacobi-PCG pressure correction, and the
pressure/velocity correction with inlet/outlet/wall boundary conditions.

The compute path is libcps.so (CUDA, C ABI in include/cps.h); this package
holds the ctypes binding (:mod:`.cps`), the seeded geometry generators
(:mod:`.geometry`) and the build recipe (:mod:`.build`).
"""
from .geometry import Design  # noqa: F401

__version__ = "0.1.0"
