"""B200-native finite-difference wave propagation behind RockSeis's driver API.

The compute path is librsgpu.so (hand-written sm_100a CUDA behind the C ABI of
include/rsgpu.h).  The first use of any public name loads it and raises if it
is missing or stale: there is no CPU fallback.  (The build module itself,
rockseis_b200.build, does not load the library.)
"""
import importlib

__all__ = ["abi", "Data2D", "ModelAcoustic2D", "ModelElastic2D", "ModellingAcoustic2D", "ModellingElastic2D",
           "Plan", "modelling_batch"]

_FROM_ROCKSEIS = {"Data2D", "ModelAcoustic2D", "ModelElastic2D", "ModellingAcoustic2D", "ModellingElastic2D",
                  "Plan", "modelling_batch"}


def __getattr__(name):
    if name == "abi":
        return importlib.import_module(".abi", __name__)
    if name in _FROM_ROCKSEIS:
        return getattr(importlib.import_module(".rockseis", __name__), name)
    raise AttributeError(name)
