"""B200 (sm_100a) gravity hot path of the NEXT N-body code.

The compute path is libnext_b200.so (hand-written CUDA, C ABI in
include/next_gpu.h); :mod:`next_b200.native` binds it, :mod:`next_b200.ic`
makes seeded initial conditions, and :mod:`next_b200.particle` mirrors the
reference's Particle / Step / computeAdaptiveDt interface.
"""
__all__ = ["ic", "native"]
