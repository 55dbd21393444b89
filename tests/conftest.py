"""Shared fixtures.  GPU tests are marked `gpu`; everything else runs on CPU.

The oracle (oracle/liborot_oracle.so, a CPU restatement of the reference) and,
where it was built, the reference itself (oracle/_ref/liborot_ref.so) are
loaded here as checkers only.
"""
import ctypes
import json
import os
import subprocess
import sys
import zlib

import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
sys.path.insert(0, ROOT)

ORACLE_SO = os.path.join(ROOT, "oracle", "liborot_oracle.so")
REF_SO = os.path.join(ROOT, "oracle", "_ref", "liborot_ref.so")
GOLDEN = os.path.join(ROOT, "tests", "golden", "reference_vectors.json")
WBITS = {0: -15, 1: 15, 2: 31}


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def build_oracle():
    src = os.path.join(ROOT, "oracle", "orot_oracle.cpp")
    if not os.path.exists(ORACLE_SO) or os.path.getmtime(ORACLE_SO) < os.path.getmtime(src):
        subprocess.check_call(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-o", ORACLE_SO, src])


class Oracle:
    def __init__(self, path):
        c = ctypes
        L = c.CDLL(path)
        L.oracle_crc32.restype = c.c_uint32
        L.oracle_crc32.argtypes = [c.c_uint32, c.c_void_p, c.c_size_t]
        L.oracle_adler32.restype = c.c_uint32
        L.oracle_adler32.argtypes = [c.c_uint32, c.c_void_p, c.c_size_t]
        L.oracle_compress_bound.restype = c.c_size_t
        L.oracle_compress_bound.argtypes = [c.c_size_t, c.c_int]
        L.oracle_compress.restype = c.c_size_t
        L.oracle_compress.argtypes = [c.c_void_p, c.c_size_t, c.c_void_p, c.c_size_t, c.c_int, c.c_int]
        L.oracle_parallel_compress.restype = c.c_size_t
        L.oracle_parallel_compress.argtypes = [c.c_void_p, c.c_size_t, c.c_void_p, c.c_size_t, c.c_int, c.c_int,
                                               c.c_size_t]
        L.oracle_lz77.restype = c.c_size_t
        L.oracle_lz77.argtypes = [c.c_void_p, c.c_size_t, c.c_int, c.c_void_p]
        L.oracle_huffman_lengths.argtypes = [c.c_void_p, c.c_int, c.c_void_p, c.c_int]
        L.oracle_set_mode.argtypes = [c.c_int]
        L.oracle_limiter_events.restype = c.c_long
        L.oracle_block_types.restype = c.c_long
        L.oracle_block_types.argtypes = [c.c_void_p, c.c_size_t, c.c_void_p, c.c_long]
        self.L = L

    def compress(self, data: bytes, level: int, fmt: int) -> bytes:
        n = len(data)
        cap = self.L.oracle_compress_bound(n, fmt)
        out = ctypes.create_string_buffer(cap)
        r = self.L.oracle_compress(data, n, out, cap, level, fmt)
        return out.raw[:r]

    def parallel(self, data: bytes, level: int, fmt: int, block: int = 0) -> bytes:
        n = len(data)
        cap = 2 * n + 1024
        out = ctypes.create_string_buffer(cap)
        r = self.L.oracle_parallel_compress(data, n, out, cap, level, fmt, block)
        return out.raw[:r]

    def crc32(self, data: bytes, init: int = 0) -> int:
        return self.L.oracle_crc32(init, data, len(data))

    def adler32(self, data: bytes, init: int = 1) -> int:
        return self.L.oracle_adler32(init, data, len(data))

    def block_types(self, raw: bytes) -> list:
        """Types (0 stored, 1 fixed, 2 dynamic) of the blocks of a raw
        DEFLATE stream; raises on a malformed stream."""
        cap = 1 << 16
        while True:
            t = ctypes.create_string_buffer(cap)
            k = self.L.oracle_block_types(raw, len(raw), t, cap)
            if k < 0:
                raise ValueError("malformed DEFLATE stream")
            if k <= cap:
                return list(t.raw[:k])
            cap = k

    def tokens(self, data: bytes, level: int):
        import numpy as np
        t = np.zeros(max(len(data), 1), np.uint32)
        k = self.L.oracle_lz77(data, len(data), level, t.ctypes.data)
        return t[:k]


@pytest.fixture(scope="session")
def oracle():
    build_oracle()
    return Oracle(ORACLE_SO)


@pytest.fixture(scope="session")
def golden():
    with open(GOLDEN) as f:
        return json.load(f)


def inflate(blob: bytes, fmt: int) -> bytes:
    return zlib.decompress(blob, WBITS[fmt])


def cuda_available() -> bool:
    """True when the CUDA driver reports at least one device."""
    try:
        cu = ctypes.CDLL("libcuda.so.1")
    except OSError:
        return False
    if cu.cuInit(0) != 0:
        return False
    n = ctypes.c_int(0)
    return cu.cuDeviceGetCount(ctypes.byref(n)) == 0 and n.value > 0


@pytest.fixture(scope="session")
def gpu():
    """The engine's Python mirror; fails loudly if the library is missing."""
    if not cuda_available():
        pytest.skip("no CUDA device")
    from orot_b200 import deflate
    deflate.lib()
    return deflate
