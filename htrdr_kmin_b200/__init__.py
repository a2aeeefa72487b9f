"""B200-native (sm_100a) drop-in for the htrdr-atmosphere null-collision path tracer.

* :mod:`htrdr_kmin_b200.scene` -- seeded synthetic scenes and requests.
* :mod:`htrdr_kmin_b200.api` -- ctypes mirror of the C ABI in include/htrdr_gpu.h.
* :mod:`htrdr_kmin_b200.build` -- builds lib/libhtrdr_gpu.so with nvcc.
"""
from . import scene  # noqa: F401

__all__ = ["scene"]
