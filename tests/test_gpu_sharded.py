"""GPU parts of one stream compressed across ranks (deflate_gpu_parallel_shard),
run here as several parts on one GPU in rank order: the framed stream
inflates to the input, its checksum is exact, a single part gives exactly
the bytes of deflate_parallel_compress, and each rank boundary costs one
sync block (at most 5 bytes)."""
import zlib

import pytest

from orot_b200 import deflate, sharded, synth

pytestmark = pytest.mark.gpu

WBITS = {0: -15, 1: 15, 2: 31}


def run_parts(data, level, fmt, block, world):
    ranges = sharded.chunk_ranges(len(data), block, world)
    parts, cks, lens = [], [], []
    for s, e, final in ranges:
        if s == e and not final:
            parts.append(b"")
            cks.append(1 if fmt == deflate.Format.Zlib else 0)
        else:
            p, ck = sharded.compress_part(data[s:e], level, fmt, block, final)
            parts.append(p)
            cks.append(ck)
        lens.append(e - s)
    return sharded.frame(parts, cks, lens, fmt), parts


@pytest.mark.parametrize("level,fmt,block", [(1, 2, 131072), (6, 2, 131072), (6, 1, 65536), (9, 0, 262144),
                                             (0, 2, 100000), (3, 1, 50000)])
def test_one_part_is_the_parallel_stream(gpu, level, fmt, block):
    d = synth.array(3 << 20, synth.MIXED, level + 1)
    out, _ = run_parts(d, level, deflate.Format(fmt), block, 1)
    ref = deflate.ParallelCompressor(level, deflate.Format(fmt), 0, block).compress(d)
    assert out == ref


@pytest.mark.parametrize("world", [2, 3, 8])
@pytest.mark.parametrize("level,fmt", [(1, 2), (6, 1), (6, 0)])
def test_parts_across_ranks(gpu, world, level, fmt):
    block = 131072
    d = synth.array((5 << 20) + 12345, synth.MIXED, 7 * world)
    out, parts = run_parts(d, level, deflate.Format(fmt), block, world)
    assert zlib.decompress(out, WBITS[fmt]) == d.tobytes()
    if fmt == 2:
        assert int.from_bytes(out[-8:-4], "little") == zlib.crc32(d.tobytes())
    if fmt == 1:
        assert int.from_bytes(out[-4:], "big") == zlib.adler32(d.tobytes())
    one, _ = run_parts(d, level, deflate.Format(fmt), block, 1)
    boundaries = sum(1 for p in parts[:-1] if p)
    assert len(one) + 4 * boundaries <= len(out) <= len(one) + 5 * boundaries


def test_more_ranks_than_chunks_and_empty(gpu):
    d = synth.array(300000, synth.TEXT, 3)
    out, parts = run_parts(d, 6, deflate.Format.Gzip, 131072, 8)
    assert zlib.decompress(out, 31) == d.tobytes()
    assert sum(1 for p in parts if p) == 3
    out, _ = run_parts(b"", 6, deflate.Format.Gzip, 131072, 4)
    assert zlib.decompress(out, 31) == b""
