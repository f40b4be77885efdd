"""B200-native implementation of the BGK3D_HIT time-step hot path.

The compute path is the CUDA library ``libbgk3d.so`` (sm_100a) behind the
C-ABI of ``include/bgk3d.h``; this package holds its ctypes bindings, a host
mirror of the reference's subroutine interface (``BGK3D``) and the seeded
HIT initial-condition generator.
"""
from ._abi import BgkError, load  # noqa: F401
from .solver import BGK3D, read_namelist, run_loop  # noqa: F401
from .hit import hit_velocity  # noqa: F401

__all__ = ["BGK3D", "BgkError", "load", "read_namelist", "run_loop", "hit_velocity"]
