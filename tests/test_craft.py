"""The crafted DEFLATE streams used by the GPU inflate tests are valid: zlib
inflates them to the bytes the encoder applied, and they contain what they are
meant to exercise (codes longer than the decoder's 9-bit tables, 1-bit codes,
every block type)."""
import zlib

from deflate_craft import crafted_stream


def test_crafted_streams_inflate_under_zlib():
    for seed in range(4):
        used = {}
        raw, data = crafted_stream(seed, used=used)
        assert zlib.decompress(raw, -15) == data
        assert max(used["lit"]) > 9 and max(used["dist"]) > 9  # the decoder's slow path
        assert 1 in used["lit"]                                 # 1-bit codes: 64 tokens per window
        assert min(used["dist"]) <= 9


def test_small_crafted_stream():
    raw, data = crafted_stream(7, tokens=120)
    assert zlib.decompress(raw, -15) == data
    assert 300 < len(raw) < 4000


def test_block_walker_reads_block_types(oracle):
    """The oracle's block walker (used to explain the reference inflate's
    failures) reports the planned block types of the crafted streams, and
    zlib's own single dynamic block."""
    for seed in range(3):
        raw, _ = crafted_stream(seed, tokens=800)
        assert oracle.block_types(raw) == [2, 1, 0, 2, 2, 0, 2, 1]
    d = bytes(range(256)) * 300
    assert oracle.block_types(zlib.compress(d, 9)[2:-4]) == [2]
    assert oracle.block_types(zlib.compress(b"", 0)[2:-4]) in ([1], [0])
