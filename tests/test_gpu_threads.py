"""Calls from many host threads at once.

The reference's deflate_compress keeps all its state per call, so a program
may call it from any number of threads (src/api/deflate_api.cpp:100-136).
The engine runs each such call on an engine of the calling thread's current
device, taken from a pool, so concurrent calls overlap on the GPU; their
bytes must be exactly those of the same calls made one after another.
ctypes releases the GIL during the foreign call, so these Python threads do
call the C ABI concurrently."""
import threading
import zlib
from concurrent.futures import ThreadPoolExecutor

import pytest

from conftest import inflate
from orot_b200 import synth

pytestmark = pytest.mark.gpu


def _cases():
    cases = []
    for i in range(48):
        n = [1000, 40000, 300000, 1 << 20, (2 << 20) + 7][i % 5]
        cases.append((synth.gen(n, i % 6, 1000 + i), [1, 3, 6, 9, 0][i % 5], i % 3))
    return cases


def test_concurrent_compress_equals_sequential(gpu):
    cases = _cases()
    seq = [gpu.compress(d, lv, gpu.Format(f)) for d, lv, f in cases]
    with ThreadPoolExecutor(16) as ex:
        for _ in range(2):
            par = list(ex.map(lambda c: gpu.compress(c[0], c[1], gpu.Format(c[2])), cases))
            assert par == seq
    for (d, lv, f), out in zip(cases, seq):
        assert inflate(out, f) == d


def test_concurrent_mixed_entry_points(gpu):
    """deflate_compress, deflate_parallel_compress, crc32/adler32 and
    deflate_decompress from different threads at the same time."""
    data = [synth.gen(200000 + 999 * i, i % 6, 77 + i) for i in range(24)]

    def work(i):
        d = data[i]
        a = gpu.compress(d, 1 + i % 3, gpu.Format.Gzip)
        b = gpu.ParallelCompressor(6, gpu.Format.Zlib, 0, 65536).compress(d)
        assert zlib.decompress(a, 31) == d and zlib.decompress(b) == d
        assert gpu.crc32(d) == zlib.crc32(d) and gpu.adler32(d) == zlib.adler32(d)
        assert gpu.decompress(a, gpu.Format.Gzip, len(d)) == d
        return len(a), len(b)

    with ThreadPoolExecutor(12) as ex:
        first = list(ex.map(work, range(len(data))))
    assert first == [work(i) for i in range(len(data))]


def test_fresh_thread_after_engine_exists(gpu):
    """A thread started after the first call (whose current device is the
    default one) reuses the device's engines and gets the same bytes."""
    d = synth.gen(700001, 0, 5)
    ref = gpu.compress(d, 1, gpu.Format.Zlib)
    got = {}

    def run():
        got["c"] = gpu.compress(d, 1, gpu.Format.Zlib)
        got["crc"] = gpu.crc32(d)
        got["d"] = gpu.decompress(ref, gpu.Format.Zlib, len(d))

    t = threading.Thread(target=run)
    t.start()
    t.join()
    assert got["c"] == ref
    assert got["crc"] == zlib.crc32(d)
    assert got["d"] == d
