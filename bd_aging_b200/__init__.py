"""bd_aging_b200: B200-native Brownian-dynamics engine for aging studies of a
bidisperse WCA mixture, a drop-in for the Ramborquito/bd_aging hot path.

The compute path is libbd_aging_b200.so (hand-written sm_100a CUDA behind the
C ABI of include/bd_aging.h); this package loads it with ctypes and mirrors
the reference's entry points.  Importing the package does not load the
library; the first call into it does, and fails loudly if it is missing.
"""
__all__ = ["configs", "lib"]
