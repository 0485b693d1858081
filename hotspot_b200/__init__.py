"""hotspot_b200 -- HotSpot's grid thermal model on NVIDIA B200 (sm_100a).

The product is ``libhotspot_b200.so`` (C host code + CUDA kernels, C-ABI in
``include/``).  This package holds its ctypes bindings (:mod:`._abi`), a
Python mirror of the reference's model API (:mod:`.model`), seeded
benchmark inputs in the reference's file formats (:mod:`.workloads`), and the
batch and serving layers.
"""
from . import _abi  # noqa: F401
from ._abi import (FORM_FAST, FORM_FAST_BLOCKED, FORM_FAST_PASSES, FORM_FAST_STAGES, FORM_FP64_BLOCKED, FORM_PARITY, STEADY_AUTO, STEADY_BICGSTAB,  # noqa: F401
                   STEADY_GS_REPLAY, STEADY_MG, HotspotError, lib)

__all__ = ["lib", "FORM_PARITY", "FORM_FAST", "FORM_FAST_STAGES", "FORM_FAST_PASSES", "FORM_FP64_BLOCKED", "FORM_FAST_BLOCKED", "STEADY_AUTO", "STEADY_GS_REPLAY",
           "STEADY_MG", "STEADY_BICGSTAB", "HotspotError"]
