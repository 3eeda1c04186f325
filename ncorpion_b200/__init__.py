"""B200-native engine for NcorpiON's mutual-interaction hot path.

The compute path is ``libncgpu.so``: hand-written sm_100a CUDA kernels behind
the C ABI of ``include/ncgpu.h`` (brute-force gravity in exact-FP64, tiled
FP64 and mixed FP32/FP64 modes, the leapfrog kick/drift, collision search and
resolution).  ``ncorpion_b200.api`` binds that ABI with ctypes.
"""
import os

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "libncgpu.so")

__all__ = ["PKG_DIR", "LIB_PATH"]
