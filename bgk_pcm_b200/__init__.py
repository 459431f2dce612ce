"""bgk_pcm_b200 -- B200 (sm_100a) implementation of the BGK_PCM time step.

The compute path is libbgkpcm.so (hand-written CUDA, C ABI in
include/bgk_pcm.h).  This package holds its ctypes binding (`capi`), a host
mirror of the reference's subroutine interface (`Solver`), the y-slab
decomposition over several contexts or ranks (`SlabRun`), the input.dat
reader/writer and workload mapping (`inputs`), and the build recipe.
"""
from .capi import BGKError, Params, load, read_input  # noqa: F401
from .slab import SlabRun  # noqa: F401
from .solver import Solver  # noqa: F401

__all__ = ["BGKError", "Params", "SlabRun", "Solver", "load", "read_input"]
