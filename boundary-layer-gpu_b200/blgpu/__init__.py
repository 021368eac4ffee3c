"""blgpu -- B200 step path of the boundary-layer DNS solver (host side).

Solver      the reference's step-path subroutines over the C ABI
Ensemble    independent boxes advanced by one graph launch per step
WallNet     the learned wall-stress network (tensor-core training and inference)
cases       grids, Blasius/turbulent inflow and synthetic initial fields
files       .turbb parameters, snapshots and Lund means in the reference's formats
"""
from ._lib import FP64, MIXED, POISSON_NATIVE, POISSON_CUFFT, BlgpuError, load  # noqa: F401
from .solver import Solver  # noqa: F401
from .ensemble import Ensemble  # noqa: F401
from .mlp import WallNet  # noqa: F401
from . import cases  # noqa: F401
from . import files  # noqa: F401
