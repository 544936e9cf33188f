"""B200-native (sm_100a) LBM per-timestep path behind the reference's subroutine interfaces.

The compute path is the CUDA library ``liblbmb200.so`` (C ABI in
``include/lbm_b200.h``); this package binds it with ctypes and drives it with
torch CUDA tensors.  There is no CPU fallback.
"""
from .api import Ensemble, Lbm, LbmError, Params  # noqa: F401
from .solver import Solver  # noqa: F401
from . import workloads  # noqa: F401

__all__ = ["Ensemble", "Lbm", "LbmError", "Params", "Solver", "workloads"]
