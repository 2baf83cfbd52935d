"""B200-native distributed 3D FFT execute path (slab / pencil topologies).

Python mirror of the reference's ``KokkosFFT::Distributed`` plan interface on
top of the C ABI of ``libdfft.so`` (include/dfft.h)."""
from ._lib import LIB_PATH, lib  # noqa: F401  (loads libdfft.so or raises)
from . import exchange  # noqa: F401
from .distributed import DistributedPlan  # noqa: F401
from .navier_stokes import NavierStokes, step_graph  # noqa: F401
from .plan import (  # noqa: F401
    Batch,
    Direction,
    DistributedFFTError,
    ExecMode,
    Graph,
    Normalization,
    Plan,
    Status,
    all_topologies,
    execute,
    execute_adjoint,
    gather_blocks,
    scatter_blocks,
)

__version__ = lib.dfft_version().decode()
