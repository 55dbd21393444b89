"""GPU parity for levels 4-12 (hash chains + lazy evaluation, dynamic Huffman).

These levels are GPU-native (independent 4 KiB tiles whose 32 KiB window
slides across a run of tiles, an always-valid length limiter), so the bar is the one the
task sets: every stream inflates byte-exactly under zlib, checksums are
exact, and the compressed size is at most 3% above the reference's size at
the same level (one-sided).  Where the reference's own stream is invalid
(its over-subscribed Huffman codes and its level-10..12 tree matcher) the
size reference is the corrected oracle."""
import zlib

import pytest

from conftest import inflate
from orot_b200 import synth

pytestmark = pytest.mark.gpu

TOL = 1.03


def within(gpu_len, ref_len):
    return gpu_len <= TOL * ref_len + 8


def test_golden_lazy_levels(gpu, golden, oracle):
    cache = {}
    n = 0
    for c in golden["cases"]:
        if c["level"] < 4:
            continue
        key = (c["kind"], c["n"], c["seed"])
        if key not in cache:
            cache[key] = synth.gen(c["n"], c["kind"], c["seed"])
        d = cache[key]
        if c["path"] == "whole":
            out = gpu.compress(d, c["level"], gpu.Format(c["fmt"]))
            ref_ok = oracle.compress(d, c["level"], c["fmt"])
        else:
            out = gpu.ParallelCompressor(c["level"], gpu.Format(c["fmt"]), 0, c["block"]).compress(d)
            ref_ok = oracle.parallel(d, c["level"], c["fmt"], c["block"])
        assert inflate(out, c["fmt"]) == d, c
        ref_len = c["len"] if c["valid"] else len(ref_ok)
        assert within(len(out), ref_len), (c, len(out), ref_len)
        n += 1
    assert n > 1000


@pytest.mark.parametrize("level", [4, 6, 9, 12])
@pytest.mark.parametrize("kind", [0, 1, 2, 3, 4, 5])
def test_lazy_sizes_vs_oracle(gpu, oracle, level, kind):
    d = synth.gen(3 << 20, kind, 17 + kind)
    for fmt in (0, 1, 2):
        out = gpu.compress(d, level, gpu.Format(fmt))
        assert inflate(out, fmt) == d
        ref = oracle.compress(d, level, fmt)
        assert within(len(out), len(ref)), (fmt, len(out), len(ref))


@pytest.mark.parametrize("level", [6, 9])
def test_parallel_gzip_lazy(gpu, oracle, level):
    d = synth.array(12 << 20, synth.MIXED, level).tobytes()
    pc = gpu.ParallelCompressor(level, gpu.Format.Gzip, 0, 131072)
    out = pc.compress(d)
    assert zlib.decompress(out, 31) == d
    assert out[-8:-4] == oracle.crc32(d).to_bytes(4, "little")
    ref = oracle.parallel(d, level, 2, 131072)
    assert within(len(out), len(ref)), (len(out), len(ref))


def test_lazy_deterministic_and_batched(gpu):
    sizes = [1 << 20, 12345, 0, 777777, 3]
    bufs = [synth.gen(n, i, i) for i, n in enumerate(sizes)]
    singles = [gpu.compress(x, 6, gpu.Format.Zlib) for x in bufs]
    assert singles == [gpu.compress(x, 6, gpu.Format.Zlib) for x in bufs]
    b = gpu.DeviceBatch()
    b.load(b"".join(bufs), sizes, 6, gpu.Format.Zlib)
    b.run()
    got = b.sizes()
    for i, s in enumerate(singles):
        assert b.output(i, got[i]) == s
    b.close()


def test_incompressible_stays_within_bound(gpu):
    d = synth.gen(5 << 20, synth.RANDOM, 99)
    for level in (6, 9):
        out = gpu.compress(d, level, gpu.Format.Raw)
        assert len(out) <= gpu.compress_bound(len(d), gpu.Format.Raw)
        assert inflate(out, 0) == d


@pytest.mark.parametrize("level", [6, 9])
def test_lazy_window_runs_match_single_tiles(gpu, oracle, level, monkeypatch):
    """A CTA that slides its window over a run of tiles emits exactly the
    tokens of one CTA per tile (run length forced to 1), and both stay within
    the size bound of the reference."""
    sizes = [40 << 20, 5 << 20, 4128 * 16 + 1, 4128 * 17, 100, 3 << 20]
    kinds = [synth.MIXED, 1, 2, 3, 4, synth.PERIODIC]
    bufs = [synth.gen(n, kinds[i], 40 + i) for i, n in enumerate(sizes)]
    outs = {}
    for run in ("32", "16", "5", "1"):
        monkeypatch.setenv("OROT_B200_LAZY_RUN", run)
        b = gpu.DeviceBatch()
        b.load(b"".join(bufs), sizes, level, gpu.Format.Zlib)
        b.run()
        got = b.sizes()
        outs[run] = [b.output(i, got[i]) for i in range(len(sizes))]
        b.close()
    assert outs["32"] == outs["1"]
    assert outs["16"] == outs["1"]
    assert outs["5"] == outs["1"]
    for d, out in zip(bufs, outs["16"]):
        assert zlib.decompress(out) == d
    ref = oracle.compress(bufs[1], level, 1)
    assert within(len(outs["16"][1]), len(ref)), (len(outs["16"][1]), len(ref))
