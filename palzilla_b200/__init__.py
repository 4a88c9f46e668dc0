"""palzilla_b200 -- B200-native (sm_100a) caustics hot path of the Palzilla renderer.

The compute path lives in libpalzilla_b200.so (hand-written CUDA kernels behind the
C ABI declared in include/palzilla_b200.h); this package holds its build recipe,
the ctypes binding, Python mirrors of the reference's host classes and the
synthetic scene generators.
"""
__all__ = ["scenes", "build", "api"]
