"""B200-native (sm_100a) leap-frog pseudo-spectral Schroedinger-Poisson step of
IFDM_Code, behind the reference's run interface.

The compute lives in ``libifdm_b200.so`` (hand-written CUDA, C ABI in
``include/ifdm.h``); this package is a thin ctypes layer over it.
"""

from ._lib import EXPORTS, IfdmError, LIB_PATH, BIN_PATH, load_library  # noqa: F401
from .simulation import Batch, Simulation, fft3d_, supported_res  # noqa: F401

__all__ = ["Simulation", "Batch", "fft3d_", "supported_res", "IfdmError", "load_library", "LIB_PATH", "BIN_PATH"]
