"""alluvion_b200: a B200-native (sm_100a) engine for alluvion's SPH fluid-step path.

The engine is the native library liballuvion_b200.so behind the C ABI of
include/alluvion_b200.h.  `_capi` is its ctypes binding; `scenes` builds
constants, bodies and seeded scenes and steps them on a CUDA device.
"""
__all__ = ["_capi", "scenes", "build"]
