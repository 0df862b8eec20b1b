"""B200-native PyroWave: the encode/decode hot path of Themaister/pyrowave as
hand-written sm_100a CUDA kernels behind the reference's C API.

The product is the C-ABI library ``libpyrowave-shared.so.0`` built from
``csrc/`` (see ``include/pyrowave.h`` and ``include/pyrowave_cuda.h``).
``capi`` is its ctypes binding; ``synth`` generates the seeded synthetic frames.
"""
from . import capi  # noqa: F401
