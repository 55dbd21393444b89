"""GPU parity on the full-size workloads the benchmarks are quoted on.

  16 MiB Zipf text, raw, level 1, whole buffer: byte-identical to the
      reference's deflate_compress (src/api/deflate_api.cpp:100-136).
  256 MiB mixed, gzip, level 6, 128 KiB chunks (pigz-style,
      src/parallel/parallel_compressor.cpp:36-150): inflates byte-exactly,
      CRC-32 and ISIZE exact, and the size of a 16 MiB prefix within 3% of
      the reference's parallel output (chunks are independent, so every
      prefix of whole chunks is compressed exactly as in the full run).
  1 GiB, raw, level 9, 256 KiB chunks, in three variants (random bytes,
      8-byte period with 1% flips, Zipf text): inflates byte-exactly; random
      input falls back to stored blocks; sizes of an 8 MiB prefix within 3%.
Full-size round trips are checked with zlib."""
import zlib

import numpy as np
import pytest

from orot_b200 import synth

pytestmark = pytest.mark.gpu

TOL = 1.03


def test_text_16mib_level1_identical(gpu, oracle):
    d = synth.array(16 << 20, synth.TEXT, 42)
    out = gpu.compress(d, 1, gpu.Format.Raw)
    assert out == oracle.compress(d.tobytes(), 1, 0)
    assert zlib.decompress(out, -15) == d.tobytes()


def test_mixed_256mib_gzip_level6_chunks(gpu, oracle):
    d = synth.array(256 << 20, synth.MIXED, 7)
    pc = gpu.ParallelCompressor(6, gpu.Format.Gzip, 0, 128 << 10)
    out = pc.compress(d)
    assert out[:3] == b"\x1f\x8b\x08" and out[8] == 0  # XFL 0 in the parallel path
    assert int.from_bytes(out[-8:-4], "little") == oracle.crc32(d.tobytes())
    assert int.from_bytes(out[-4:], "little") == (256 << 20) & 0xFFFFFFFF
    assert zlib.decompress(out, 31) == d.tobytes()
    head = d[:16 << 20]
    got = pc.compress(head)
    ref = oracle.parallel(head.tobytes(), 6, 2, 128 << 10)
    assert len(got) <= TOL * len(ref), (len(got), len(ref))


@pytest.mark.parametrize("kind,seed", [(synth.RANDOM, 99), (synth.PERIODIC, 98), (synth.TEXT, 97)])
def test_1gib_level9_chunks(gpu, oracle, kind, seed):
    n = 1 << 30
    d = synth.array(n, kind, seed)
    pc = gpu.ParallelCompressor(9, gpu.Format.Raw, 0, 256 << 10)
    out = pc.compress(d)
    assert len(out) <= gpu.compress_bound(n, gpu.Format.Raw)
    assert zlib.decompress(out, -15) == d.tobytes()
    if kind == synth.RANDOM:
        # stored fallback: 5 header bytes per block of at most 65535 bytes
        assert len(out) <= n + 5 * (n // 65535 + 4096 + 1)
    head = d[:8 << 20]
    got = pc.compress(head)
    ref = oracle.parallel(head.tobytes(), 9, 0, 256 << 10)
    assert len(got) <= TOL * len(ref) + 8, (len(got), len(ref))
