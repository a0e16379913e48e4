"""bhgpu -- B200 (sm_100a) GRMHD block update for black-hole-simulator.

Hand-written CUDA kernels (libbhgpu.so, C ABI in include/bhgpu.h) behind a
Python API named after the reference solver's C++ entry points.
"""
from ._lib import lib, LIB_PATH, BhError  # noqa: F401  (raises if the CUDA library is missing)
from .mesh import Quilt, BLOCK, GHOST, CPN, NC, NF, NE  # noqa: F401
from .solver import (Metric, State, Conserved, hlld, AmrTree, RK2Integrator, StepGraph, DomainError,  # noqa: F401
                     BH_MINMOD, BH_VANLEER, BH_MC)
from .pipeline import HostPipeline  # noqa: F401
from .analysis import Analyser  # noqa: F401
from .c2p_guess import C2PGuess, wait_selftest  # noqa: F401
from . import configs  # noqa: F401
from . import tune  # noqa: F401
from . import snapshot  # noqa: F401

__version__ = "0.1.0"
