"""The engine's streams through the reference's own inflate.

Every GPU stream must inflate byte-identically under zlib (the authoritative
check) and under orot's own deflate_decompress (src/api/deflate_api.cpp:
138-219, built from the reference's sources into oracle/_ref/liborot_ref.so).
orot's inflate runs in child processes (tests/orot_inflate.py) because it can
crash.  Where zlib accepts a stream and orot's inflate does not, the failure
must be one of the reference's two known inflate defects, identified here
from the stream itself:

  stored-after-huffman  a stored block that follows a Huffman-coded block in
                        the same stream.  The Huffman decoder refills its
                        64-bit bit buffer ahead of the symbol it decodes; the
                        stored-block path then reads LEN/NLEN from that buffer
                        but copies the payload from the input pointer
                        (src/decompress/decompressor.cpp:148-152, 254-300),
                        skipping the bytes still buffered, and the stream
                        ends in DATA_ERROR.  The reference's own parallel
                        output hits it whenever a chunk is stored after a
                        compressed one (mixed data), exactly as the engine's
                        identical bytes do.
  gzip-member-scan      gzip input of 256 KiB or more first goes to the
                        parallel member decoder, which splits the stream at
                        any byte pattern that looks like a gzip header
                        (src/decompress/parallel_decompress.cpp:53-63); a
                        false split gives MEM_ERROR or garbage sizes, and only
                        DATA_ERROR falls back to the sequential decoder
                        (src/api/deflate_api.cpp:207-216).

Every other stream must pass orot's inflate.  The counts are printed."""
import collections

import pytest

import orot_inflate
from conftest import inflate
from orot_b200 import synth

pytestmark = pytest.mark.gpu

HDR = {0: 0, 1: 2, 2: 10}
TRL = {0: 0, 1: 4, 2: 8}


def _raw(fmt, blob):
    return blob[HDR[fmt]:len(blob) - TRL[fmt]]


def _check(oracle, items, label):
    """items: (fmt, data, stream, name).  Asserts the rules above and returns
    the counts."""
    assert orot_inflate.available(), "oracle/_ref/liborot_ref.so is not built (python -c 'import __graft_entry__ as g; g.build()')"
    for fmt, d, blob, name in items:
        assert inflate(blob, fmt) == d, f"{label}: {name} does not round-trip under zlib"
    res = orot_inflate.inflate_many([(f, d, b) for f, d, b, _ in items])
    counts = collections.Counter()
    unexplained = []
    for (fmt, d, blob, name), (code, ok) in zip(items, res):
        if ok:
            counts["orot_ok"] += 1
            continue
        types = oracle.block_types(_raw(fmt, blob))
        huff = [i for i, t in enumerate(types) if t != 0]
        if huff and any(t == 0 for t in types[huff[0] + 1:]):
            counts["stored-after-huffman"] += 1
        elif fmt == 2 and len(blob) >= (256 << 10) and code in (-2, -1):
            counts["gzip-member-scan"] += 1
        else:
            unexplained.append((name, orot_inflate.NAMES.get(code, code), types[:8]))
    counts["zlib_ok"] = len(items)
    print(f"\n{label}: {len(items)} streams, zlib {counts['zlib_ok']}, orot {counts['orot_ok']}, "
          f"reference defects: stored-after-huffman {counts['stored-after-huffman']}, "
          f"gzip-member-scan {counts['gzip-member-scan']}")
    assert not unexplained, f"{label}: orot inflate rejects streams for no known reason: {unexplained[:5]}"
    return counts


def test_golden_cases_under_orot_inflate(gpu, golden, oracle):
    items, cache = [], {}
    for c in golden["cases"]:
        key = (c["kind"], c["n"], c["seed"])
        if key not in cache:
            cache[key] = synth.gen(c["n"], c["kind"], c["seed"])
        d = cache[key]
        if c["path"] == "whole":
            out = gpu.compress(d, c["level"], gpu.Format(c["fmt"]))
        else:
            out = gpu.ParallelCompressor(c["level"], gpu.Format(c["fmt"]), 0, c["block"]).compress(d)
        items.append((c["fmt"], d, out, f"{c['path']}/{c['kind']}/{c['n']}/L{c['level']}/f{c['fmt']}"))
    counts = _check(oracle, items, "golden cases")
    assert counts["orot_ok"] == len(items)  # no golden case holds the defect patterns


def test_config_workloads_under_orot_inflate(gpu, oracle):
    """The benchmark configurations at full size or a stated prefix."""
    items = []
    text = synth.gen(16 << 20, 0, 42)
    items.append((0, text, gpu.compress(text, 1, gpu.Format.Raw), "16 MiB Zipf text, raw L1, whole buffer"))
    mixed = synth.gen(16 << 20, synth.MIXED, 7)
    items.append((2, mixed, gpu.ParallelCompressor(6, gpu.Format.Gzip, 0, 128 << 10).compress(mixed),
                  "16 MiB prefix of the mixed buffer, gzip L6, 128 KiB chunks"))
    for kind, seed in ((3, 99), (5, 98), (0, 97)):
        d = synth.gen(8 << 20, kind, seed)
        items.append((0, d, gpu.ParallelCompressor(9, gpu.Format.Raw, 0, 256 << 10).compress(d),
                      f"8 MiB of generator {kind}, raw L9, 256 KiB chunks"))
    for lv in (1, 6):
        for f in (0, 1, 2):
            d = synth.gen(3 << 20, synth.MIXED, 11 + lv)
            items.append((f, d, gpu.compress(d, lv, gpu.Format(f)), f"3 MiB mixed, whole buffer, L{lv}, format {f}"))
    _check(oracle, items, "benchmark workloads")
