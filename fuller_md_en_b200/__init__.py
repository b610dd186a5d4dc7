"""fuller_md on B200: hand-written sm_100a CUDA kernels for the per-step
force-and-integrate path of fuller_md (focusnishikawa/fuller_md_en), behind a
C-ABI (include/fullermd.h, libfullermd_cuda.so), with C++ drop-in drivers
(fuller_*_gpu) and this Python mirror of the reference routines.
"""
from ._lib import FmdError, load, LIB_PATH  # noqa: F401
from .api import Batch, Context, System, Topology, RunConfig, mm_replica  # noqa: F401
from .rebo2 import Rebo2Knots  # noqa: F401

__all__ = ["Batch", "Context", "System", "Topology", "RunConfig", "mm_replica", "Rebo2Knots", "FmdError", "load",
           "LIB_PATH"]
