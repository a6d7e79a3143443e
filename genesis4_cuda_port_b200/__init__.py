"""B200-native GENESIS 1.3 v4 time-stepping core.

The compute lives in ``lib/libg4b200.so`` (hand-written sm_100a CUDA behind
the C ABI of ``include/g4b.h``); this package holds its sources (``csrc/``),
the build recipe and a thin Python mirror of the reference's device-state and
solver classes.
"""
from ._lib import G4BError, G4B_FP64, G4B_MIXED, Step  # noqa: F401

__all__ = ["G4BError", "G4B_FP64", "G4B_MIXED", "Step"]
