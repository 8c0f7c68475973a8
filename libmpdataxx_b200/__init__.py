"""libmpdataxx_b200: libmpdata++'s MPDATA advection step and the pressure solve
it feeds, as hand-written sm_100a CUDA kernels behind the reference's API.

    from libmpdataxx_b200 import opts, solvers, concurr, bcond
"""
from . import bcond, opts, solvers  # noqa: F401
from . import concurr  # noqa: F401
