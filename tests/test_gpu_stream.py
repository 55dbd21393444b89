"""Streaming compression (deflate_stream_*, the reference's streaming API,
include/orot/deflate.h:92-108) over the GPU engine: any split of the input,
any output buffer size and any flush pattern give a stream that inflates to
the input, flushes make all input so far decodable, and the trailer is
right."""
import ctypes
import zlib

import pytest

from orot_b200 import deflate, synth

pytestmark = pytest.mark.gpu

WBITS = {0: -15, 1: 15, 2: 31}


@pytest.mark.parametrize("fmt", [0, 1, 2])
@pytest.mark.parametrize("level", [0, 1, 6])
def test_pieces_round_trip(gpu, fmt, level):
    d = synth.gen((3 << 20) + 12345, synth.MIXED, 5 + level)
    c = deflate.Compressor(level, deflate.Format(fmt))
    out, pos, step = [], 0, 1
    while pos < len(d):
        out.append(c.feed(d[pos:pos + step]))
        pos += step
        step = step * 7 + 3
    out.append(c.finish())
    c.close()
    assert zlib.decompress(b"".join(out), WBITS[fmt]) == d


def test_sync_flush_makes_input_decodable(gpu):
    d = synth.gen(3 << 20, synth.TEXT, 8)
    c = deflate.Compressor(6, deflate.Format.Zlib)
    dobj = zlib.decompressobj(15)
    got = b""
    for a, b in [(0, 1000), (1000, 1500000), (1500000, 2500000), (2500000, len(d))]:
        got += dobj.decompress(c.feed(d[a:b]) + c.flush(full=(a % 2 == 0)))
        assert got == d[:b]
    got += dobj.decompress(c.finish())
    assert got == d and dobj.eof


def test_small_output_buffer_and_errors(gpu):
    L = deflate.lib()
    d = synth.gen(2500000, synth.INTS, 2)
    s = L.deflate_stream_new(1, 2)
    src = ctypes.create_string_buffer(d, len(d))
    nin = ctypes.c_void_p(ctypes.addressof(src))
    ain = ctypes.c_size_t(len(d))
    out = b""
    while True:
        buf = ctypes.create_string_buffer(4093)
        nout = ctypes.c_void_p(ctypes.addressof(buf))
        aout = ctypes.c_size_t(4093)
        r = L.deflate_stream_compress(s, ctypes.byref(nin), ctypes.byref(ain), ctypes.byref(nout), ctypes.byref(aout), 3)
        out += buf.raw[:4093 - aout.value]
        assert r in (0, 1, 3)
        if r == 1:
            break
    assert zlib.decompress(out, 31) == d
    # input after the end is refused
    one = ctypes.create_string_buffer(b"x", 1)
    nin = ctypes.c_void_p(ctypes.addressof(one))
    ain = ctypes.c_size_t(1)
    buf = ctypes.create_string_buffer(64)
    nout = ctypes.c_void_p(ctypes.addressof(buf))
    aout = ctypes.c_size_t(64)
    assert L.deflate_stream_compress(s, ctypes.byref(nin), ctypes.byref(ain), ctypes.byref(nout), ctypes.byref(aout), 0) == -5
    L.deflate_stream_free(s)


@pytest.mark.parametrize("fmt", [0, 1, 2])
def test_empty_stream(gpu, fmt):
    c = deflate.Compressor(6, deflate.Format(fmt))
    assert zlib.decompress(c.finish(), WBITS[fmt]) == b""
