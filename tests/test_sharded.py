"""The multi-rank path: one pigz-style stream compressed by the ranks of a
gloo process group on CPU (world sizes 2 and 3).  The GPU part compressor is
replaced by zlib producing parts of the same shape (raw DEFLATE, a sync
block at the end of every part but the last), so these tests cover the host
logic: chunk ranges, the exchange of sizes and checksums, the gather,
framing and the checksum combine identities (checked against zlib)."""
import os
import random
import socket
import zlib

import pytest
import torch.multiprocessing as mp

from orot_b200 import deflate, sharded


def zlib_part(data, level, fmt, block, final):
    b = bytes(data)
    c = zlib.compressobj(max(1, min(level, 9)), zlib.DEFLATED, -15)
    out = c.compress(b) + c.flush(zlib.Z_FINISH if final else zlib.Z_SYNC_FLUSH)
    ck = zlib.adler32(b) if fmt == deflate.Format.Zlib else zlib.crc32(b) if fmt == deflate.Format.Gzip else 0
    return out, ck


def test_chunk_ranges_cover_input():
    for n, block, world in [(0, 100, 1), (0, 100, 3), (1, 100, 2), (1000, 100, 3), (1050, 100, 4), (250, 100, 8),
                            (10 ** 6, 4096, 7)]:
        r = sharded.chunk_ranges(n, block, world)
        assert len(r) == world
        assert r[0][0] == 0 and r[-1][1] == n
        for (s0, e0, _), (s1, _, _) in zip(r, r[1:]):
            assert e0 == s1
        for s, e, _ in r:
            assert s % block == 0 or s == n
        finals = [i for i, x in enumerate(r) if x[2]]
        assert len(finals) == 1
        assert all(r[i][0] == r[i][1] for i in range(finals[0] + 1, world))


def test_checksum_combine_matches_zlib():
    rng = random.Random(5)
    L = deflate.lib()
    for _ in range(200):
        a = rng.randbytes(rng.randrange(0, 3000))
        b = rng.randbytes(rng.randrange(0, 3000))
        assert L.deflate_crc32_combine(zlib.crc32(a), zlib.crc32(b), len(b)) == zlib.crc32(a + b)
        assert L.deflate_adler32_combine(zlib.adler32(a), zlib.adler32(b), len(b)) == zlib.adler32(a + b)
    big = 5 << 30  # lengths past 4 GiB
    x = L.deflate_crc32_combine(zlib.crc32(b"abc"), 0x12345678, big)
    assert x == L.deflate_crc32_combine(zlib.crc32(b"abc"), 0x12345678, big)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, cases, q):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        for data, level, fmt, block in cases:
            out = sharded.compress(data, level, fmt, block, part_fn=zlib_part)
            if rank == 0:
                q.put(out)
            else:
                assert out is None
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_stream_on_gloo_ranks(world):
    rng = random.Random(world)
    text = b" ".join(rng.choice([b"deflate", b"chunk", b"rank", b"stream", b"zlib"]) for _ in range(60000))
    cases = [(text, 6, deflate.Format.Gzip, 16384), (text, 1, deflate.Format.Zlib, 100000),
             (text[:70000], 9, deflate.Format.Raw, 4096), (b"", 6, deflate.Format.Gzip, 4096),
             (text[:5000], 6, deflate.Format.Zlib, 4096)]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, cases, q)) for r in range(world)]
    for p in procs:
        p.start()
    outs = [q.get(timeout=120) for _ in cases]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    for (data, level, fmt, block), out in zip(cases, outs):
        wbits = {deflate.Format.Raw: -15, deflate.Format.Zlib: 15, deflate.Format.Gzip: 31}[fmt]
        assert zlib.decompress(out, wbits) == data
        if fmt == deflate.Format.Gzip:
            assert out[8] == 0 and int.from_bytes(out[-8:-4], "little") == zlib.crc32(data)
        if fmt == deflate.Format.Zlib:
            assert int.from_bytes(out[-4:], "big") == zlib.adler32(data)
