"""B200-native finite-difference wave propagation behind RockSeis's driver API.

The compute path is librsgpu.so (hand-written sm_100a CUDA behind the C ABI of
include/rsgpu.h).  Importing this package loads it and raises if it is missing:
there is no CPU fallback.
"""
from . import abi  # noqa: F401  (loads librsgpu.so or raises)
from .rockseis import (Data2D, ModelAcoustic2D, ModelElastic2D, ModellingAcoustic2D,  # noqa: F401
                       ModellingElastic2D, Plan, modelling_batch)

__all__ = ["abi", "Data2D", "ModelAcoustic2D", "ModelElastic2D", "ModellingAcoustic2D", "ModellingElastic2D",
           "Plan", "modelling_batch"]
