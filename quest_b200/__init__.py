"""B200-native (sm_100a) implementation of QuEST's O(N^2) retarded-interaction
time step.

The compute path is the CUDA library quest_b200/libquest_gpu.so behind the C
ABI in include/quest_gpu.h; quest_b200.capi binds it from Python.  There is
no CPU fallback.
"""
from . import inputs  # noqa: F401

__all__ = ["capi", "inputs"]
