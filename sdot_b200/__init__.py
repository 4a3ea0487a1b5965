"""sdot_b200: B200-native power-diagram / semi-discrete optimal transport hot path.

The compute path is libsdot_b200.so (hand-written CUDA for sm_100a behind the
C ABI of include/sdot_gpu.h).  Importing the package does not touch the GPU;
creating a PowerDiagram loads the library and fails loudly if it is missing.
"""
from .power_diagram import PowerDiagram  # noqa: F401

__all__ = ["PowerDiagram"]
