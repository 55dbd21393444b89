"""GPU inflate: deflate_decompress (the reference's whole-buffer decompress,
src/api/deflate_api.cpp:138-219 and src/formats/*) and on-device verification
of compressed batches.  Streams come from three encoders: this engine, the
oracle (the reference's encoder restated) and zlib; every decode must equal
the original bytes, and corrupt, truncated or oversized cases must fail the
way the reference fails (DEFLATE_DATA_ERROR)."""
import struct
import zlib

import pytest

from orot_b200 import deflate, synth

pytestmark = pytest.mark.gpu

DATA_ERROR = -1
WBITS = {0: -15, 1: 15, 2: 31}


def raw_call(blob, fmt, cap):
    import ctypes
    L = deflate.lib()
    out = ctypes.create_string_buffer(max(cap, 1))
    n = ctypes.c_size_t(0)
    r = L.deflate_decompress(blob, len(blob), out, cap, ctypes.byref(n), fmt)
    return r, out.raw[:n.value]


@pytest.mark.parametrize("fmt", [0, 1, 2])
@pytest.mark.parametrize("level", [0, 1, 3, 6, 9, 12])
def test_own_streams_round_trip(gpu, fmt, level):
    for kind, n in [(synth.MIXED, 3 << 20), (synth.TEXT, 100000), (synth.ZEROS, 70000), (synth.RANDOM, 5000),
                    (synth.PERIODIC, 1 << 20), (synth.INTS, 0)]:
        d = synth.gen(n, kind, level + kind)
        c = deflate.compress(d, level, deflate.Format(fmt))
        assert deflate.decompress(c, deflate.Format(fmt), n + 16) == d


@pytest.mark.parametrize("fmt", [0, 1, 2])
def test_oracle_and_zlib_streams(gpu, oracle, fmt):
    for kind in range(6):
        d = synth.gen(400000, kind, 30 + kind)
        for level in (1, 4, 6, 9):
            assert deflate.decompress(oracle.compress(d, level, fmt), deflate.Format(fmt), len(d)) == d
            assert deflate.decompress(oracle.parallel(d, level, fmt, 65536), deflate.Format(fmt), len(d)) == d
        for zl in (0, 1, 6, 9):
            c = zlib.compressobj(zl, zlib.DEFLATED, WBITS[fmt])
            z = c.compress(d) + c.flush()
            assert deflate.decompress(z, deflate.Format(fmt), len(d)) == d


def test_gzip_header_fields(gpu):
    d = synth.gen(50000, synth.TEXT, 5)
    c = zlib.compressobj(6, zlib.DEFLATED, -15)
    body = c.compress(d) + c.flush()
    extra = b"AB\x04\x00xyzw"
    hdr = bytes([0x1F, 0x8B, 8, 0x04 | 0x08 | 0x10 | 0x02, 0, 0, 0, 0, 0, 3])
    hdr += struct.pack("<H", len(extra)) + extra + b"name.txt\x00" + b"a comment\x00"
    hdr += struct.pack("<H", zlib.crc32(hdr) & 0xFFFF)
    blob = hdr + body + struct.pack("<II", zlib.crc32(d), len(d))
    assert deflate.decompress(blob, deflate.Format.Gzip, len(d)) == d


def test_errors_like_the_reference(gpu):
    d = synth.gen(200000, synth.MIXED, 9)
    for fmt in (1, 2):
        c = bytearray(deflate.compress(d, 6, deflate.Format(fmt)))
        r, _ = raw_call(bytes(c), fmt, len(d))
        assert r == 0
        bad = bytearray(c)
        bad[-2 if fmt == 1 else -6] ^= 0x40  # a byte of the Adler-32 / CRC-32 trailer
        assert raw_call(bytes(bad), fmt, len(d))[0] == DATA_ERROR
        assert raw_call(bytes(c[: len(c) // 2]), fmt, len(d))[0] == DATA_ERROR  # truncated
        assert raw_call(bytes(c), fmt, len(d) - 1)[0] == DATA_ERROR            # output too small
    assert raw_call(b"\x78\x9d" + b"\x00" * 10, 1, 100)[0] == DATA_ERROR      # FCHECK
    assert raw_call(b"\x1f\x8c" + b"\x00" * 20, 2, 100)[0] == DATA_ERROR      # magic
    assert raw_call(b"\x07\x00\x00", 0, 100)[0] == DATA_ERROR                 # block type 3
    assert raw_call(b"\x03\x00", 0, 0) == (0, b"")                           # empty fixed block
    r, out = raw_call(deflate.compress(b"", 6, deflate.Format.Gzip), 2, 0)
    assert r == 0 and out == b""
    # exactly full output is fine
    c = deflate.compress(d, 1, deflate.Format.Raw)
    assert raw_call(c, 0, len(d)) == (0, d)


@pytest.mark.parametrize("level", [1, 6])
def test_batch_verify_on_device(gpu, level):
    sizes = [int(x) for x in synth.loguniform_sizes(400, 1, 2 << 20, 3)] + [0, 1, 5]
    bufs = [synth.gen(n, i % 6, i) for i, n in enumerate(sizes)]
    for fmt in (deflate.Format.Zlib, deflate.Format.Gzip, deflate.Format.Raw):
        b = deflate.DeviceBatch()
        b.load(b"".join(bufs), sizes, level, fmt)
        b.run()
        assert all(b.verify())
        b.close()


@pytest.mark.parametrize("level", [1, 6, 9])
def test_gzip_members_compress_and_parallel_decode(gpu, oracle, level):
    """Independent members: any gzip reader (zlib with concatenated members)
    reads the whole file, every member is a complete gzip stream, and
    deflate_decompress decodes members in parallel (inputs >= 256 KiB)."""
    d = synth.array((6 << 20) + 777, synth.MIXED, level)
    blob = deflate.compress_gzip_members(d, level, 1 << 20)
    # zlib reads concatenated members one at a time
    out, rest, pos = b"", blob, 0
    while rest:
        dobj = zlib.decompressobj(31)
        out += dobj.decompress(rest)
        rest = dobj.unused_data
        pos += 1
    assert out == d.tobytes() and pos == 7
    assert deflate.decompress(blob, deflate.Format.Gzip, len(d)) == d.tobytes()
    # members of the reference's encoder decode the same way
    ref = b"".join(oracle.compress(d[i:i + (1 << 20)].tobytes(), level, 2) for i in range(0, len(d), 1 << 20))
    assert deflate.decompress(ref, deflate.Format.Gzip, len(d)) == d.tobytes()


def test_gzip_members_errors(gpu):
    d = synth.array(3 << 20, synth.TEXT, 4)
    blob = bytearray(deflate.compress_gzip_members(d, 6, 1 << 20))
    # output smaller than the members' total: MEM_ERROR, as the reference's parallel path
    assert raw_call(bytes(blob), 2, len(d) - 1)[0] == -2
    # a damaged member CRC fails the parallel path, and the one-stream fallback fails too
    first_end = len(deflate.compress_gzip_members(d[: 1 << 20], 6, 1 << 20))
    blob[first_end - 8] ^= 1
    assert raw_call(bytes(blob), 2, len(d))[0] == DATA_ERROR


def test_header_pattern_inside_member_data(gpu):
    """A gzip file of 256 KiB or more whose data holds a gzip-header-like
    pattern: the member scan splits on it, and the file must still decode
    (as one stream, or member after member)."""
    d = bytearray(synth.gen(400000, synth.RANDOM, 11))
    fake = bytes([0x1F, 0x8B, 8, 0, 1, 2, 3, 4, 0, 3]) + b"\xff" * 12
    d[1000:1000 + len(fake)] = fake
    d[300000:300000 + len(fake)] = fake
    d = bytes(d)
    for blob in (deflate.compress(d, 0, deflate.Format.Gzip),
                 deflate.compress(d[:200000], 0, deflate.Format.Gzip) + deflate.compress(d[200000:], 0, deflate.Format.Gzip)):
        assert raw_call(blob, 2, len(d)) == (0, d)
        assert raw_call(blob, 2, len(d) - 1)[0] in (DATA_ERROR, -2)


def _wrap(raw, data, fmt):
    if fmt == 0:
        return raw
    if fmt == 1:
        return b"\x78\x9c" + raw + zlib.adler32(data).to_bytes(4, "big")
    return bytes([0x1F, 0x8B, 8, 0, 0, 0, 0, 0, 0, 0xFF]) + raw + struct.pack("<II", zlib.crc32(data), len(data))


@pytest.mark.parametrize("fmt", [0, 1, 2])
def test_crafted_blocks_and_long_codes(gpu, fmt):
    """Stored (also empty), fixed and dynamic blocks back to back; dynamic
    codes of 1 to 15 bits (longer than the 9-bit lookup tables, for literals,
    lengths and distances) and a 1-bit literal code (64 tokens in a window,
    32 literals pending at once); every length and distance the history
    allows (tests/deflate_craft.py)."""
    from deflate_craft import crafted_stream
    for seed in range(6):
        raw, data = crafted_stream(seed)
        assert deflate.decompress(_wrap(raw, data, fmt), deflate.Format(fmt), len(data)) == data


def test_zlib_strategies_and_flushes(gpu):
    """zlib's filtered, Huffman-only, RLE and fixed strategies, with sync and
    full flushes (empty stored blocks, byte alignment) between chunks."""
    skew = bytes(synth.gen(300000, synth.RANDOM, 3)[i] if i % 97 == 0 else 65 for i in range(300000))
    for d in (synth.gen(300000, synth.MIXED, 12), synth.gen(200000, synth.TEXT, 13), skew):
        for strategy in (0, 1, 2, 3, 4):
            for flush in (zlib.Z_NO_FLUSH, zlib.Z_SYNC_FLUSH, zlib.Z_FULL_FLUSH):
                c = zlib.compressobj(6, zlib.DEFLATED, -15, 9, strategy)
                z = b""
                for i in range(0, len(d), 70001):
                    z += c.compress(d[i:i + 70001]) + (c.flush(flush) if flush != zlib.Z_NO_FLUSH else b"")
                z += c.flush()
                assert deflate.decompress(z, deflate.Format.Raw, len(d)) == d, (strategy, flush)


def test_truncated_at_every_byte(gpu):
    """Every proper prefix of a stream fails with DEFLATE_DATA_ERROR (the last
    block never ends, or the trailer is missing); the whole stream decodes."""
    from deflate_craft import crafted_stream
    raw, data = crafted_stream(7, tokens=120)
    for fmt in (0, 1):
        blob = _wrap(raw, data, fmt)
        assert raw_call(blob, fmt, len(data)) == (0, data)
        for k in range(len(blob)):
            assert raw_call(blob[:k], fmt, len(data))[0] == DATA_ERROR, (fmt, k)
