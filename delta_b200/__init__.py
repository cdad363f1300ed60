"""delta_b200 -- B200-native contact pipeline for triangulated DEM particles.

Broadphase, triangle-triangle narrowphase (bf / penalty / hybrid / GJK), penalty
forces and explicit rigid-body integration, after KonstantinosKr/delta's
delta/contact and delta/dynamics.  The compute runs in libdelta_b200.so (CUDA,
sm_100a) behind the C ABI in include/delta_b200.h.
"""
from ._lib import DeltaError, LIB_PATH, header_functions, lib  # noqa: F401

__version__ = "0.1.0"
