"""Python mirror of orot's DEFLATE compress API over liborot_b200.so.

Names, defaults and error behaviour follow the reference's C++ wrapper
(include/orot/deflate.h:184-389 in daramkun/orot): `compress` raises `Error`
with DEFLATE_BUF_ERROR when the C call returns 0, `ParallelCompressor`
defaults to gzip, `adler32` / `crc32` take the initial value last.  Every call
goes through the C ABI of include/orot_b200.h into the CUDA kernels; there is
no host fallback, and importing this module without the built library or
without a CUDA device raises.
"""
from __future__ import annotations

import ctypes
import enum
import os
from typing import Sequence

_LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "liborot_b200.so")
_lib = None

DEFLATE_OK = 0
DEFLATE_MEM_ERROR = -2
DEFLATE_BUF_ERROR = -3
DEFLATE_PARAM_ERROR = -5


class Format(enum.IntEnum):
    Raw = 0
    Zlib = 1
    Gzip = 2


class Level:
    Store = 0
    Fast = 1
    Default = 6
    Better = 9
    Max = 12


class Error(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(msg)
        self.code = code


def lib() -> ctypes.CDLL:
    """Loads liborot_b200.so once; raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        raise ImportError(f"{_LIB_PATH} is not built; run `python -m orot_b200.build`")
    L = ctypes.CDLL(_LIB_PATH)
    c = ctypes
    L.deflate_compress_bound.restype = c.c_size_t
    L.deflate_compress_bound.argtypes = [c.c_size_t, c.c_int]
    L.deflate_compress.restype = c.c_size_t
    L.deflate_compress.argtypes = [c.c_void_p, c.c_size_t, c.c_void_p, c.c_size_t, c.c_int, c.c_int]
    L.deflate_parallel_new.restype = c.c_void_p
    L.deflate_parallel_new.argtypes = [c.c_int, c.c_int, c.c_int, c.c_size_t]
    L.deflate_parallel_free.argtypes = [c.c_void_p]
    L.deflate_parallel_compress.restype = c.c_size_t
    L.deflate_parallel_compress.argtypes = [c.c_void_p, c.c_void_p, c.c_size_t, c.c_void_p, c.c_size_t]
    L.deflate_crc32.restype = c.c_uint32
    L.deflate_crc32.argtypes = [c.c_uint32, c.c_void_p, c.c_size_t]
    L.deflate_adler32.restype = c.c_uint32
    L.deflate_adler32.argtypes = [c.c_uint32, c.c_void_p, c.c_size_t]
    L.orot_b200_last_error.restype = c.c_char_p
    L.orot_b200_geometry_source.restype = c.c_char_p
    L.orot_b200_geometry_tile.restype = c.c_uint32
    L.orot_b200_geometry_tile.argtypes = [c.c_uint64, c.c_int, c.c_int]
    L.deflate_gpu_batch_new.restype = c.c_void_p
    L.deflate_gpu_batch_free.argtypes = [c.c_void_p]
    L.deflate_gpu_batch_load.restype = c.c_int
    L.deflate_gpu_batch_load.argtypes = [c.c_void_p, c.c_void_p, c.POINTER(c.c_size_t), c.c_size_t, c.c_int,
                                         c.c_int, c.c_int, c.c_size_t]
    L.deflate_gpu_batch_run.restype = c.c_int
    L.deflate_gpu_batch_run.argtypes = [c.c_void_p, c.c_void_p, c.c_int]
    L.deflate_gpu_batch_sizes.restype = c.c_int
    L.deflate_gpu_batch_sizes.argtypes = [c.c_void_p, c.POINTER(c.c_size_t)]
    L.deflate_gpu_batch_output.restype = c.c_size_t
    L.deflate_gpu_batch_output.argtypes = [c.c_void_p, c.c_size_t, c.c_void_p, c.c_size_t]
    L.deflate_gpu_batch_launches.restype = c.c_int
    L.deflate_gpu_batch_launches.argtypes = [c.c_void_p]
    L.deflate_gpu_compress_batch.restype = c.c_size_t
    L.deflate_gpu_compress_batch.argtypes = [c.POINTER(c.c_void_p), c.POINTER(c.c_size_t), c.POINTER(c.c_void_p),
                                             c.POINTER(c.c_size_t), c.POINTER(c.c_size_t), c.c_size_t, c.c_int,
                                             c.c_int]
    L.deflate_gpu_compress_packed.restype = c.c_size_t
    L.deflate_gpu_compress_packed.argtypes = [c.c_void_p, c.POINTER(c.c_size_t), c.c_size_t, c.c_int, c.c_int,
                                              c.c_void_p, c.c_size_t, c.POINTER(c.c_uint64), c.POINTER(c.c_size_t)]
    L.deflate_gpu_packed_bound.restype = c.c_size_t
    L.deflate_gpu_packed_bound.argtypes = [c.POINTER(c.c_size_t), c.c_size_t, c.c_int]
    L.deflate_gpu_batch_profile.restype = c.c_int
    L.deflate_gpu_batch_profile.argtypes = [c.c_void_p, c.c_int]
    L.deflate_gpu_batch_phase_ms.restype = c.c_int
    L.deflate_gpu_batch_phase_ms.argtypes = [c.c_void_p, c.POINTER(c.c_float), c.c_int]
    L.deflate_gpu_phase_name.restype = c.c_char_p
    L.deflate_gpu_phase_name.argtypes = [c.c_int]
    L.deflate_gpu_compress_pipelined.restype = c.c_size_t
    L.deflate_gpu_compress_pipelined.argtypes = [c.c_void_p, c.POINTER(c.c_size_t), c.c_size_t, c.c_int, c.c_int,
                                                 c.c_void_p, c.c_size_t, c.POINTER(c.c_uint64),
                                                 c.POINTER(c.c_size_t), c.c_size_t, c.c_int]
    L.deflate_gpu_server_new.restype = c.c_void_p
    L.deflate_gpu_server_new.argtypes = [c.c_size_t, c.c_int]
    L.deflate_gpu_server_free.argtypes = [c.c_void_p]
    L.deflate_gpu_server_submit.restype = c.c_uint64
    L.deflate_gpu_server_submit.argtypes = [c.c_void_p, c.c_void_p, c.c_size_t, c.c_void_p, c.c_size_t, c.c_int,
                                            c.c_int]
    L.deflate_gpu_server_wait.restype = c.c_int
    L.deflate_gpu_server_wait.argtypes = [c.c_void_p, c.c_uint64, c.POINTER(c.c_size_t), c.POINTER(c.c_double),
                                          c.c_double]
    L.deflate_gpu_server_stats.restype = c.c_int
    L.deflate_gpu_server_stats.argtypes = [c.c_void_p, c.POINTER(c.c_uint64), c.POINTER(c.c_uint64)]
    L.deflate_decompress.restype = c.c_int
    L.deflate_decompress.argtypes = [c.c_void_p, c.c_size_t, c.c_void_p, c.c_size_t, c.POINTER(c.c_size_t), c.c_int]
    L.deflate_stream_new.restype = c.c_void_p
    L.deflate_stream_new.argtypes = [c.c_int, c.c_int]
    L.deflate_stream_free.argtypes = [c.c_void_p]
    L.deflate_stream_compress.restype = c.c_int
    L.deflate_stream_compress.argtypes = [c.c_void_p, c.POINTER(c.c_void_p), c.POINTER(c.c_size_t),
                                          c.POINTER(c.c_void_p), c.POINTER(c.c_size_t), c.c_int]
    L.deflate_gzip_members_bound.restype = c.c_size_t
    L.deflate_gzip_members_bound.argtypes = [c.c_size_t, c.c_size_t]
    L.deflate_gpu_compress_gzip_members.restype = c.c_size_t
    L.deflate_gpu_compress_gzip_members.argtypes = [c.c_void_p, c.c_size_t, c.c_int, c.c_size_t, c.c_void_p, c.c_size_t]
    L.deflate_gpu_batch_verify.restype = c.c_int
    L.deflate_gpu_batch_verify.argtypes = [c.c_void_p, c.POINTER(c.c_int)]
    L.deflate_gpu_parallel_shard.restype = c.c_int
    L.deflate_gpu_parallel_shard.argtypes = [c.c_void_p, c.c_size_t, c.c_int, c.c_int, c.c_size_t, c.c_int, c.c_void_p,
                                             c.c_size_t, c.POINTER(c.c_size_t), c.POINTER(c.c_uint32)]
    L.deflate_crc32_combine.restype = c.c_uint32
    L.deflate_crc32_combine.argtypes = [c.c_uint32, c.c_uint32, c.c_uint64]
    L.deflate_adler32_combine.restype = c.c_uint32
    L.deflate_adler32_combine.argtypes = [c.c_uint32, c.c_uint32, c.c_uint64]
    _lib = L
    return L


def last_error() -> str:
    return lib().orot_b200_last_error().decode()


def geometry_source() -> str:
    """Where the library's pass geometry table came from (the autotuner's run)."""
    return lib().orot_b200_geometry_source().decode()


def geometry_tile(pass_bytes: int, sms: int = 148, hash_bits: int = 12) -> int:
    """Tile bytes the planner uses at levels 1-3 for a pass of `pass_bytes`
    on a device of `sms` SMs (hash_bits 12: level 1, 14: levels 2-3)."""
    return int(lib().orot_b200_geometry_tile(int(pass_bytes), int(sms), int(hash_bits)))


def _ptr(buf) -> tuple[int, int, object]:
    """(address, length, keepalive) of a bytes-like or numpy buffer."""
    try:
        import numpy as np
        if isinstance(buf, np.ndarray):
            a = np.ascontiguousarray(buf).view(np.uint8).reshape(-1)
            return a.ctypes.data, a.size, a
    except ImportError:  # pragma: no cover
        pass
    mv = memoryview(buf).cast("B")
    if mv.readonly:
        b = ctypes.create_string_buffer(bytes(mv), len(mv))
        return ctypes.addressof(b), len(mv), b
    arr = (ctypes.c_char * len(mv)).from_buffer(mv)
    return ctypes.addressof(arr), len(mv), (arr, mv)


def compress_bound(n: int, format: Format = Format.Zlib) -> int:
    return lib().deflate_compress_bound(n, int(format))


def compress(data, level: int = Level.Default, format: Format = Format.Zlib) -> bytes:
    """deflate_compress over the whole input (include/orot/deflate.h:219-235)."""
    L = lib()
    addr, n, keep = _ptr(data)
    bound = L.deflate_compress_bound(n, int(format))
    out = ctypes.create_string_buffer(bound)
    r = L.deflate_compress(addr if n else None, n, out, bound, int(level), int(format))
    del keep
    if r == 0:
        raise Error(DEFLATE_BUF_ERROR, "deflate::compress: output buffer overflow " + last_error())
    return out.raw[:r]


def decompress(data, format: Format = Format.Zlib, max_output: int = 256 << 20) -> bytes:
    """deflate_decompress into a buffer of max_output bytes, decoded on the GPU
    (include/orot/deflate.h:238-255); raises Error on failure."""
    L = lib()
    addr, n, keep = _ptr(data)
    out = ctypes.create_string_buffer(max(max_output, 1))
    actual = ctypes.c_size_t(0)
    r = L.deflate_decompress(addr if n else None, n, out, max_output, ctypes.byref(actual), int(format))
    del keep
    if r != DEFLATE_OK:
        raise Error(r, "deflate::decompress failed " + last_error())
    return out.raw[:actual.value]


def compress_gzip_members(data, level: int = Level.Default, member_size: int = 1 << 20) -> bytes:
    """One gzip file of independent members of member_size input bytes
    (deflate_gpu_compress_gzip_members)."""
    L = lib()
    addr, n, keep = _ptr(data)
    cap = L.deflate_gzip_members_bound(n, member_size)
    out = ctypes.create_string_buffer(max(cap, 1))
    r = L.deflate_gpu_compress_gzip_members(addr if n else None, n, int(level), member_size, out, cap)
    del keep
    if r == 0:
        raise Error(DEFLATE_BUF_ERROR, "compress_gzip_members failed " + last_error())
    return out.raw[:r]


NO_FLUSH, SYNC_FLUSH, FULL_FLUSH, FINISH = 0, 1, 2, 3
DEFLATE_STREAM_END, DEFLATE_NEED_OUTPUT = 1, 3


class Compressor:
    """Streaming compressor over deflate_stream_* (the reference's RAII
    Compressor, include/orot/deflate.h:260-301): feed() takes input and returns
    whatever compressed bytes are ready, flush() and finish() force output."""

    def __init__(self, level: int = Level.Default, fmt: Format = Format.Zlib):
        self._s = lib().deflate_stream_new(int(level), int(fmt))
        if not self._s:
            raise Error(DEFLATE_MEM_ERROR, "Compressor: allocation failed")

    def _run(self, data, mode: int) -> bytes:
        L = lib()
        addr, n, keep = _ptr(data) if data is not None and len(data) else (0, 0, None)
        nin = ctypes.c_void_p(addr or None)
        ain = ctypes.c_size_t(n)
        chunks = []
        while True:
            cap = 1 << 20
            buf = ctypes.create_string_buffer(cap)
            nout = ctypes.c_void_p(ctypes.addressof(buf))
            aout = ctypes.c_size_t(cap)
            r = L.deflate_stream_compress(self._s, ctypes.byref(nin), ctypes.byref(ain), ctypes.byref(nout),
                                          ctypes.byref(aout), mode)
            if r < 0:
                raise Error(r, "Compressor failed " + last_error())
            chunks.append(buf.raw[:cap - aout.value])
            if r == DEFLATE_NEED_OUTPUT or (r == DEFLATE_OK and ain.value):
                continue
            del keep
            return b"".join(chunks)

    def feed(self, data) -> bytes:
        return self._run(data, NO_FLUSH)

    def flush(self, full: bool = False) -> bytes:
        return self._run(None, FULL_FLUSH if full else SYNC_FLUSH)

    def finish(self) -> bytes:
        return self._run(None, FINISH)

    def close(self) -> None:
        if self._s:
            lib().deflate_stream_free(self._s)
            self._s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ParallelCompressor:
    """pigz-style compressor (include/orot/deflate.h:351-376)."""

    def __init__(self, level: int = Level.Default, fmt: Format = Format.Gzip, threads: int = 0, block_size: int = 0):
        self._ctx = lib().deflate_parallel_new(int(level), int(fmt), int(threads), int(block_size))
        if not self._ctx:
            raise Error(DEFLATE_MEM_ERROR, "ParallelCompressor: allocation failed")
        self.level, self.fmt, self.block_size = level, fmt, block_size

    def compress(self, data) -> bytes:
        L = lib()
        addr, n, keep = _ptr(data)
        bound = L.deflate_compress_bound(n, int(Format.Gzip))
        out = ctypes.create_string_buffer(bound)
        r = L.deflate_parallel_compress(self._ctx, addr if n else None, n, out, bound)
        del keep
        if r == 0:
            raise Error(DEFLATE_BUF_ERROR, "ParallelCompressor::compress: buffer overflow " + last_error())
        return out.raw[:r]

    def close(self) -> None:
        if self._ctx:
            lib().deflate_parallel_free(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # pragma: no cover
            pass


def adler32(data, init: int = 1) -> int:
    addr, n, keep = _ptr(data)
    r = lib().deflate_adler32(init, addr if n else None, n)
    del keep
    return r


def crc32(data, init: int = 0) -> int:
    addr, n, keep = _ptr(data)
    r = lib().deflate_crc32(init, addr if n else None, n)
    del keep
    return r


def compress_packed(concat, sizes: Sequence[int], level: int, format: Format, out) -> tuple[int, list, list]:
    """deflate_gpu_compress_packed: one H2D of `concat`, one D2H into `out`
    (a writable buffer of at least packed_bound(sizes) bytes).  Returns
    (packed_total, offsets, sizes)."""
    L = lib()
    addr, n, keep = _ptr(concat)
    oaddr, on, okeep = _ptr(out)
    cnt = len(sizes)
    arr = (ctypes.c_size_t * cnt)(*sizes)
    offs = (ctypes.c_uint64 * (cnt + 1))()
    szs = (ctypes.c_size_t * cnt)()
    r = L.deflate_gpu_compress_packed(addr if n else None, arr, cnt, int(level), int(format), oaddr, on, offs, szs)
    del keep, okeep
    if r == 0:
        raise Error(DEFLATE_BUF_ERROR, "compress_packed: " + last_error())
    return r, list(offs), list(szs)


def compress_pipelined(concat, sizes, level: int, format: Format, out, group_bytes: int = 0,
                       lanes: int = 0) -> tuple:
    """deflate_gpu_compress_pipelined; `out` needs packed_bound(sizes) bytes.
    `sizes` is a sequence of ints or a uint64 numpy array (passed without a
    copy); returns (end, offsets, sizes) with the stream offsets (count + 1
    entries) and sizes in `out` as uint64 numpy arrays."""
    import numpy as np
    L = lib()
    addr, n, keep = _ptr(concat)
    oaddr, on, okeep = _ptr(out)
    sz = np.ascontiguousarray(sizes, dtype=np.uint64)
    cnt = len(sz)
    offs = np.empty(cnt + 1, np.uint64)
    szs = np.empty(cnt, np.uint64)
    p_size = ctypes.POINTER(ctypes.c_size_t)
    r = L.deflate_gpu_compress_pipelined(addr if n else None, sz.ctypes.data_as(p_size), cnt, int(level), int(format),
                                         oaddr, on, offs.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
                                         szs.ctypes.data_as(p_size), int(group_bytes), int(lanes))
    del keep, okeep
    if r == 0:
        raise Error(DEFLATE_BUF_ERROR, "compress_pipelined: " + last_error())
    return r, offs, szs


class Server:
    """Continuous-batching compression server (deflate_gpu_server_*).

    submit() returns a ticket; the input and output buffers must stay alive
    until wait() returns for that ticket."""

    def __init__(self, device_budget: int = 0, lanes: int = 0):
        self._s = lib().deflate_gpu_server_new(int(device_budget), int(lanes))
        if not self._s:
            raise Error(DEFLATE_MEM_ERROR, "server: " + last_error())
        self._keep = {}

    def submit(self, data, level: int, format: Format, out=None, out_capacity: int | None = None) -> int:
        addr, n, keep = _ptr(data)
        if out is None:
            cap = compress_bound(n, format) if out_capacity is None else out_capacity
            out = ctypes.create_string_buffer(max(cap, 1))
        else:
            cap = len(out) if out_capacity is None else out_capacity
        oaddr, _, okeep = _ptr(out)
        t = lib().deflate_gpu_server_submit(self._s, addr if n else None, n, oaddr, cap, int(level), int(format))
        if t == 0:
            raise Error(DEFLATE_PARAM_ERROR, "server submit: " + last_error())
        self._keep[t] = (keep, okeep, out)
        return t

    def wait(self, ticket: int, timeout: float = 0.0):
        """(bytes or None on failure, latency seconds); raises TimeoutError."""
        sz = ctypes.c_size_t(0)
        lat = ctypes.c_double(0)
        r = lib().deflate_gpu_server_wait(self._s, ticket, ctypes.byref(sz), ctypes.byref(lat), float(timeout))
        if r == 1:
            raise TimeoutError(f"ticket {ticket}")
        keep = self._keep.pop(ticket, None)
        if r == -1:
            raise Error(DEFLATE_PARAM_ERROR, f"unknown ticket {ticket}")
        if r != 0:
            return None, lat.value
        out = keep[2]
        buf = bytes(memoryview(out).cast("B")[:sz.value])
        return buf, lat.value

    def stats(self) -> tuple[int, int]:
        a, b = ctypes.c_uint64(0), ctypes.c_uint64(0)
        lib().deflate_gpu_server_stats(self._s, ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value

    def close(self) -> None:
        if self._s:
            lib().deflate_gpu_server_free(self._s)
            self._s = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # pragma: no cover
            pass


def packed_bound(sizes: Sequence[int], format: Format) -> int:
    arr = (ctypes.c_size_t * len(sizes))(*sizes)
    return lib().deflate_gpu_packed_bound(arr, len(sizes), int(format))


class DeviceBatch:
    """Buffers kept on the device and compressed by one pass of kernels."""

    def __init__(self):
        self._b = lib().deflate_gpu_batch_new()
        if not self._b:
            raise Error(DEFLATE_MEM_ERROR, "batch: " + last_error())
        self.count = 0

    def load(self, concat, sizes: Sequence[int], level: int, format: Format, parallel: bool = False,
             block_size: int = 0) -> None:
        addr, n, keep = _ptr(concat)
        arr = (ctypes.c_size_t * len(sizes))(*sizes)
        r = lib().deflate_gpu_batch_load(self._b, addr, arr, len(sizes), int(level), int(format), int(parallel),
                                         int(block_size))
        del keep
        if r != 0:
            raise Error(DEFLATE_PARAM_ERROR, "batch load: " + last_error())
        self.count = len(sizes)

    def run(self, stream: int = 0, graph: bool = False) -> None:
        r = lib().deflate_gpu_batch_run(self._b, ctypes.c_void_p(stream or None), int(graph))
        if r != 0:
            raise Error(DEFLATE_PARAM_ERROR, "batch run: " + last_error())

    def sizes(self) -> list[int]:
        arr = (ctypes.c_size_t * self.count)()
        if lib().deflate_gpu_batch_sizes(self._b, arr) != 0:
            raise Error(DEFLATE_PARAM_ERROR, "batch sizes: " + last_error())
        return list(arr)

    def output(self, i: int, size: int) -> bytes:
        buf = ctypes.create_string_buffer(max(size, 1))
        r = lib().deflate_gpu_batch_output(self._b, i, buf, size)
        return buf.raw[:r]

    def launches(self) -> int:
        return lib().deflate_gpu_batch_launches(self._b)

    def verify(self) -> list[bool]:
        """Decodes every stream of the last run on the device and compares it
        with its input (deflate_gpu_batch_verify); True per stream that
        round-trips with the right framing and trailer."""
        ok = (ctypes.c_int * self.count)()
        if lib().deflate_gpu_batch_verify(self._b, ok) < 0:
            raise Error(DEFLATE_PARAM_ERROR, "batch verify: " + last_error())
        return [bool(x) for x in ok]

    def profile(self, on: bool) -> None:
        lib().deflate_gpu_batch_profile(self._b, int(on))

    def phase_ms(self) -> dict:
        arr = (ctypes.c_float * 16)()
        n = lib().deflate_gpu_batch_phase_ms(self._b, arr, 16)
        if n < 0:
            raise Error(DEFLATE_PARAM_ERROR, "phase_ms: " + last_error())
        return {lib().deflate_gpu_phase_name(i).decode(): float(arr[i]) for i in range(n)}

    def close(self) -> None:
        if self._b:
            lib().deflate_gpu_batch_free(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # pragma: no cover
            pass
