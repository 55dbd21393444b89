"""orot_b200 -- a B200-native DEFLATE compression engine.

The product is liborot_b200.so: CUDA kernels for sm_100a behind the C ABI of
include/orot_b200.h, a drop-in for orot's DEFLATE compress API.  This package
holds its sources (csrc/), the build recipe (build.py), a ctypes mirror of the
reference's C++ wrapper (deflate.py) and the synthetic-input generator used by
tests and benchmarks (synth.py).
"""
from . import deflate  # noqa: F401
from .deflate import Format, Level, Error, ParallelCompressor, DeviceBatch, compress, adler32, crc32  # noqa: F401
