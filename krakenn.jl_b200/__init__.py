"""krakenn.jl_b200 -- the B200 backend of Kraken.jl's stream-collide path.

Hand-written sm_100a CUDA kernels behind a C ABI (include/krakenb200.h,
libkrakenb200.so in this directory), with this Python layer mirroring the
reference's kernel wrappers (`ops`) and step-loop drivers (`drivers`).
The directory name is not a Python identifier; load it with
`__graft_entry__.load_package()` (registered as module `krakenn_b200`).
"""
from . import _lib, batch, checkpoint, drivers, krk, lattice, libb, ops, output, sharding, slab, surrogate  # noqa: F401
from ._lib import KrakenArgumentError, KrakenError, version  # noqa: F401
from .drivers import (LBMConfig, initialize_2d, initialize_3d, omega, reynolds,  # noqa: F401
                      run_cavity_2d, run_cavity_3d, run_natural_convection_2d,
                      run_couette_2d, run_natural_convection_3d, run_poiseuille_2d,
                      run_rayleigh_benard_2d,
                      run_taylor_green_2d, run_taylor_green_3d)
from .batch import CavityBatch, Graph, sweep_cases  # noqa: F401
from .ops import *  # noqa: F401,F403
