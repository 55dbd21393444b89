"""CPU tests of the C ABI boundary: the library loads, exports every entry
point include/orot_b200.h declares, and the host-side argument checks behave
like the reference (no device work is issued by these calls)."""
import ctypes
import os
import re

import pytest

from conftest import ROOT

LIB = os.path.join(ROOT, "orot_b200", "liborot_b200.so")
HDR = os.path.join(ROOT, "include", "orot_b200.h")


def declared_functions():
    src = open(HDR).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^[A-Za-z_][\w\s\*]*?\b(\w+)\s*\(", src, flags=re.M)
    return sorted(set(n for n in names if n not in ("defined",)))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(LIB):
        from orot_b200 import build
        build.build_all()
    return ctypes.CDLL(LIB)


def test_exports_every_declared_symbol(lib):
    names = declared_functions()
    assert "deflate_compress" in names and "deflate_parallel_compress" in names
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n


def test_reference_symbols_present(lib):
    # the orot entry points a caller of the reference binds (include/orot/deflate.h:61-150)
    for n in ["deflate_set_allocator", "deflate_compress_bound", "deflate_compress", "deflate_parallel_new",
              "deflate_parallel_free", "deflate_parallel_compress", "deflate_crc32", "deflate_adler32"]:
        assert hasattr(lib, n)


def test_bound_matches_reference_formula(lib, oracle):
    lib.deflate_compress_bound.restype = ctypes.c_size_t
    lib.deflate_compress_bound.argtypes = [ctypes.c_size_t, ctypes.c_int]
    for n in [0, 1, 100, 4095, 4096, 65536, 1 << 25, (1 << 33) + 7]:
        for f in (0, 1, 2):
            assert lib.deflate_compress_bound(n, f) == oracle.L.oracle_compress_bound(n, f)
    assert lib.deflate_compress_bound(0, 0) == 13


def test_host_side_rejections(lib):
    c = ctypes
    lib.deflate_compress.restype = c.c_size_t
    lib.deflate_compress.argtypes = [c.c_void_p, c.c_size_t, c.c_void_p, c.c_size_t, c.c_int, c.c_int]
    out = c.create_string_buffer(64)
    # capacity below the bound returns 0 (src/formats/raw_deflate.cpp:20)
    assert lib.deflate_compress(b"abc", 3, out, 5, 1, 0) == 0
    assert lib.deflate_compress(b"abc", 3, out, 15, 1, 0) == 0
    # unknown format returns 0 (src/api/deflate_api.cpp:127-135 has no default)
    assert lib.deflate_compress(b"abc", 3, out, 64, 1, 7) == 0
    lib.deflate_parallel_compress.restype = c.c_size_t
    lib.deflate_parallel_compress.argtypes = [c.c_void_p, c.c_void_p, c.c_size_t, c.c_void_p, c.c_size_t]
    assert lib.deflate_parallel_compress(None, b"abc", 3, out, 64) == 0
    lib.deflate_parallel_new.restype = c.c_void_p
    lib.deflate_parallel_new.argtypes = [c.c_int, c.c_int, c.c_int, c.c_size_t]
    lib.deflate_parallel_free.argtypes = [c.c_void_p]
    ctx = lib.deflate_parallel_new(6, 2, 4, 0)
    assert ctx
    lib.deflate_parallel_free(ctx)
    assert not lib.deflate_parallel_new(6, 9, 4, 0)
    lib.deflate_crc32.restype = c.c_uint32
    lib.deflate_crc32.argtypes = [c.c_uint32, c.c_void_p, c.c_size_t]
    lib.deflate_adler32.restype = c.c_uint32
    lib.deflate_adler32.argtypes = [c.c_uint32, c.c_void_p, c.c_size_t]
    # empty input returns the initial value (test_deflate_simd.cpp:41-42,83)
    assert lib.deflate_crc32(0x1234, None, 0) == 0x1234
    assert lib.deflate_adler32(1, None, 0) == 1


def test_more_host_side_rejections(lib):
    """Argument checks of the other entry points, all answered on the host
    before any device work (the reference's DEFLATE_PARAM_ERROR, -5, where it
    has the call; the documented codes of the GPU-only calls otherwise)."""
    c = ctypes
    PARAM = -5
    lib.deflate_decompress.restype = c.c_int
    lib.deflate_decompress.argtypes = [c.c_void_p, c.c_size_t, c.c_void_p, c.c_size_t, c.POINTER(c.c_size_t), c.c_int]
    out = c.create_string_buffer(64)
    n = c.c_size_t(0)
    assert lib.deflate_decompress(b"x", 1, out, 64, c.byref(n), 7) == PARAM    # unknown format
    assert lib.deflate_decompress(None, 5, out, 64, c.byref(n), 0) == PARAM    # input pointer missing
    assert lib.deflate_decompress(b"x", 1, None, 64, c.byref(n), 0) == PARAM   # output pointer missing

    lib.deflate_stream_new.restype = c.c_void_p
    lib.deflate_stream_new.argtypes = [c.c_int, c.c_int]
    lib.deflate_stream_free.argtypes = [c.c_void_p]
    lib.deflate_stream_compress.restype = c.c_int
    lib.deflate_stream_compress.argtypes = [c.c_void_p, c.POINTER(c.c_void_p), c.POINTER(c.c_size_t),
                                            c.POINTER(c.c_void_p), c.POINTER(c.c_size_t), c.c_int]
    assert not lib.deflate_stream_new(6, 9)
    s = lib.deflate_stream_new(6, 1)
    assert s
    nin, ain = c.c_void_p(None), c.c_size_t(0)
    nout, aout = c.c_void_p(c.addressof(out)), c.c_size_t(64)
    assert lib.deflate_stream_compress(None, c.byref(nin), c.byref(ain), c.byref(nout), c.byref(aout), 0) == PARAM
    assert lib.deflate_stream_compress(s, None, c.byref(ain), c.byref(nout), c.byref(aout), 0) == PARAM
    assert lib.deflate_stream_compress(s, c.byref(nin), c.byref(ain), c.byref(nout), c.byref(aout), 9) == PARAM
    ain.value = 10  # input announced without a pointer
    assert lib.deflate_stream_compress(s, c.byref(nin), c.byref(ain), c.byref(nout), c.byref(aout), 0) == PARAM
    lib.deflate_stream_free(s)
    lib.deflate_stream_free(None)

    lib.deflate_gpu_compress_noalloc.restype = c.c_int
    lib.deflate_gpu_compress_noalloc.argtypes = [c.c_void_p, c.c_size_t, c.c_void_p, c.c_size_t, c.c_int, c.c_int,
                                                 c.c_void_p, c.c_void_p]
    fake = 4096  # never dereferenced: every case below is rejected first
    assert lib.deflate_gpu_compress_noalloc(fake, 10, None, 64, 1, 0, fake, None) == -1          # no output
    assert lib.deflate_gpu_compress_noalloc(fake, 10, fake, 64, 1, 5, fake, None) == -1          # format
    assert lib.deflate_gpu_compress_noalloc(fake, (1 << 20) + 1, fake, 1 << 22, 1, 0, fake, None) == -2
    assert lib.deflate_gpu_compress_noalloc(fake, 10, fake, 64, 6, 0, fake, None) == -3          # level
    assert lib.deflate_gpu_compress_noalloc(fake, 1000, fake, 1000, 1, 0, fake, None) == -4      # capacity

    lib.deflate_gpu_parallel_shard.restype = c.c_int
    lib.deflate_gpu_parallel_shard.argtypes = [c.c_void_p, c.c_size_t, c.c_int, c.c_int, c.c_size_t, c.c_int,
                                               c.c_void_p, c.c_size_t, c.POINTER(c.c_size_t), c.POINTER(c.c_uint32)]
    ck = c.c_uint32(0)
    assert lib.deflate_gpu_parallel_shard(b"abc", 3, 6, 0, 0, 1, None, 64, c.byref(n), c.byref(ck)) == -1
    assert lib.deflate_gpu_parallel_shard(b"abc", 3, 6, 4, 0, 1, out, 64, c.byref(n), c.byref(ck)) == -1

    lib.deflate_gpu_batch_load.restype = c.c_int
    lib.deflate_gpu_batch_load.argtypes = [c.c_void_p, c.c_void_p, c.POINTER(c.c_size_t), c.c_size_t, c.c_int, c.c_int,
                                           c.c_int, c.c_size_t]
    lib.deflate_gpu_batch_run.restype = c.c_int
    lib.deflate_gpu_batch_run.argtypes = [c.c_void_p, c.c_void_p, c.c_int]
    assert lib.deflate_gpu_batch_load(None, b"abc", None, 0, 1, 0, 0, 0) == -1
    assert lib.deflate_gpu_batch_run(None, None, 0) == -1

    lib.deflate_gpu_server_submit.restype = c.c_uint64
    lib.deflate_gpu_server_submit.argtypes = [c.c_void_p, c.c_void_p, c.c_size_t, c.c_void_p, c.c_size_t, c.c_int,
                                              c.c_int]
    lib.deflate_gpu_server_wait.restype = c.c_int
    lib.deflate_gpu_server_wait.argtypes = [c.c_void_p, c.c_uint64, c.POINTER(c.c_size_t), c.POINTER(c.c_double),
                                            c.c_double]
    assert lib.deflate_gpu_server_submit(None, b"abc", 3, out, 64, 1, 0) == 0
    assert lib.deflate_gpu_server_wait(None, 1, None, None, 0.0) == -1


def test_reference_unit_tests_link_the_engine():
    """The reference's unit tests (built by oracle/Makefile.ref) resolve their
    deflate_* calls to liborot_b200.so, not to the reference's archive linked
    after it (no execution here: that is a GPU test)."""
    import subprocess
    unit = os.path.join(ROOT, "oracle", "_ref", "unit")
    if not os.path.isdir(unit):
        pytest.skip("reference unit tests not built on this machine")
    for name in ["test_deflate_roundtrip", "test_deflate_levels", "test_deflate_formats", "test_deflate_simd",
                 "test_deflate_parallel"]:
        exe = os.path.join(unit, name)
        undefined = subprocess.run(["nm", "-u", exe], capture_output=True, text=True).stdout
        defined = subprocess.run(["nm", "--defined-only", exe], capture_output=True, text=True).stdout
        assert " deflate_" not in defined, name          # nothing taken from the archive
        assert "deflate_compress" in undefined or "deflate_crc32" in undefined or "deflate_parallel" in undefined
        ldd = subprocess.run(["ldd", exe], capture_output=True, text=True).stdout
        assert "liborot_b200.so" in ldd and "not found" not in ldd.split("liborot_b200.so")[1].split("\n")[0]
