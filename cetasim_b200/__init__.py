"""cetasim_b200: sm_100a implementation of CETASim's multi-particle tracking
path behind a C ABI (include/cetasim_gpu.h, libcetagpu.so).

The Python layer is a thin host API; all tracking runs in the CUDA kernels of
libcetagpu.so and importing a stage fails loudly when the library is absent.
"""
from . import _abi
from .configs import Workload, make

__all__ = ["_abi", "Workload", "make", "MPBeam"]


def __getattr__(name):
    if name == "MPBeam":
        from .beam import MPBeam
        return MPBeam
    raise AttributeError(name)
