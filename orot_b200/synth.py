"""Seeded synthetic inputs (ctypes over libsynth.so, built from csrc/synth.cpp).

Kinds: 0 Zipf text, 1 u32 sorted deltas, 2 zeros, 3 random, 4 mixed 1 MiB
rotation of 0-3, 5 8-byte periodic with 1% flips.  Deterministic in
(kind, n, seed).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

TEXT, INTS, ZEROS, RANDOM, MIXED, PERIODIC = range(6)
_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libsynth.so")
_lib = None


def _L():
    global _lib
    if _lib is None:
        if not os.path.exists(_PATH):
            from . import build
            build.build_synth()
        L = ctypes.CDLL(_PATH)
        L.synth_fill.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_uint64]
        L.synth_loguniform_sizes.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint64, ctypes.c_uint64,
                                             ctypes.c_uint64]
        _lib = L
    return _lib


def fill(out: np.ndarray, kind: int, seed: int) -> np.ndarray:
    assert out.dtype == np.uint8 and out.flags.c_contiguous
    _L().synth_fill(out.ctypes.data, out.size, int(kind), int(seed) & 0xFFFFFFFFFFFFFFFF)
    return out


def gen(n: int, kind: int, seed: int) -> bytes:
    return array(n, kind, seed).tobytes()


def array(n: int, kind: int, seed: int) -> np.ndarray:
    a = np.empty(n, np.uint8)
    if n:
        fill(a, kind, seed)
    return a


def loguniform_sizes(count: int, lo: int, hi: int, seed: int) -> np.ndarray:
    out = np.empty(count, np.uint64)
    _L().synth_loguniform_sizes(out.ctypes.data, count, lo, hi, seed)
    return out
