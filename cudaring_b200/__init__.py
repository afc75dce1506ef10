"""cudaRing hot path on B200 (sm_100a): deformable / rigid ring polymers in 2-D.

``DPM2D`` mirrors the reference's model class over the C ABI of
``libcudaring.so`` (include/cudaring.h); ``synth`` builds seeded inputs with
the reference's conventions.
"""
from ._lib import CudaRingError, declared_symbols, lib
from .dpm2d import DPM2D, simControl

__all__ = ["DPM2D", "simControl", "CudaRingError", "lib", "declared_symbols"]
