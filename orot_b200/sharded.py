"""One pigz-style DEFLATE stream compressed by the ranks of a process group.

orot's deflate_parallel_compress (include/orot/deflate.h:122-150,
src/parallel/parallel_compressor.cpp:36-150) cuts its input into chunks of
block_size bytes that are compressed independently.  Here the chunks are
split into contiguous ranges, one per rank (one GPU each): every rank
compresses its range with deflate_gpu_parallel_shard, the ranks exchange the
part sizes and range checksums (a few bytes each, all_gather over the group),
rank 0 gathers the parts and frames the stream: header, parts in rank order,
trailer with the combined checksum (deflate_crc32_combine /
deflate_adler32_combine).  Parts other than the last end with an empty stored
block, so they are whole bytes and concatenate as they are; the stream
therefore differs from a one-GPU deflate_parallel_compress only by those
sync blocks (5 bytes per rank boundary) and inflates to the same bytes.

    out = sharded.compress(data, level=6, fmt=Format.Gzip, block_size=128 << 10)
    # rank 0: the gzip stream; other ranks: None
"""
from __future__ import annotations

import ctypes
from typing import Callable, Optional, Sequence

from . import deflate


def default_block_size(level: int) -> int:
    """Chunk size the parallel path uses when block_size is 0
    (src/parallel/parallel_compressor.cpp:16-20)."""
    return 131072 if level <= 3 else 524288 if level <= 6 else 1048576


def chunk_ranges(n: int, block: int, world: int) -> list[tuple[int, int, bool]]:
    """(start, end, final) byte range of every rank: contiguous runs of whole
    chunks, as even as possible; `final` marks the rank holding the last
    chunk.  Ranks beyond the chunk count get empty, non-final ranges."""
    if block <= 0 or world <= 0:
        raise ValueError("block and world must be positive")
    nchunks = max(1, -(-n // block))
    out = []
    c = 0
    for r in range(world):
        k = nchunks // world + (1 if r < nchunks % world else 0)
        s, e = min(c * block, n), min((c + k) * block, n)
        out.append((s, e, k > 0 and c + k == nchunks))
        c += k
    return out


def compress_part(data, level: int, fmt: deflate.Format, block: int, final: bool) -> tuple[bytes, int]:
    """This rank's part on its GPU: (bytes, checksum of the range)."""
    L = deflate.lib()
    addr, n, keep = deflate._ptr(data)
    nchunk = max(1, -(-n // block))
    cap = max(deflate.compress_bound(n, deflate.Format.Raw), n + nchunk * (5 * -(-block // 65535) + 1) + 32) + 64
    out = ctypes.create_string_buffer(cap)
    size = ctypes.c_size_t(0)
    ck = ctypes.c_uint32(0)
    r = L.deflate_gpu_parallel_shard(addr if n else None, n, int(level), int(fmt), int(block), 1 if final else 0, out,
                                     cap, ctypes.byref(size), ctypes.byref(ck))
    del keep
    if r != 0:
        raise deflate.Error(deflate.DEFLATE_BUF_ERROR, f"deflate_gpu_parallel_shard failed ({r}): {deflate.last_error()}")
    return out.raw[:size.value], ck.value


def frame(parts: Sequence[bytes], checksums: Sequence[int], lengths: Sequence[int], fmt: deflate.Format) -> bytes:
    """Header + parts + trailer (zlib_wrapper.cpp:28-52, gzip_wrapper.cpp:21-74;
    the parallel path writes gzip XFL 0, parallel_compressor.cpp:96-98)."""
    L = deflate.lib()
    total = sum(lengths)
    body = b"".join(parts)
    if fmt == deflate.Format.Raw:
        return body
    if fmt == deflate.Format.Zlib:
        a = 1
        for ck, n in zip(checksums, lengths):
            a = L.deflate_adler32_combine(a, ck, n) if n else a
        return b"\x78\x9c" + body + a.to_bytes(4, "big")
    c = 0
    for ck, n in zip(checksums, lengths):
        c = L.deflate_crc32_combine(c, ck, n) if n else c
    hdr = bytes([0x1F, 0x8B, 8, 0, 0, 0, 0, 0, 0, 0xFF])
    return hdr + body + c.to_bytes(4, "little") + (total & 0xFFFFFFFF).to_bytes(4, "little")


def compress(data, level: int = 6, fmt: deflate.Format = deflate.Format.Gzip, block_size: int = 0, group=None,
             part_fn: Optional[Callable] = None) -> Optional[bytes]:
    """Compresses `data` (the whole input, present on every rank) as one
    stream across the ranks of `group` (torch.distributed; every rank calls
    this with the same arguments).  Returns the stream on rank 0, None on the
    others.  `part_fn(range_bytes, level, fmt, block, final) -> (bytes,
    checksum)` replaces the GPU part compressor (tests)."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    block = block_size or default_block_size(level)
    s, e, final = chunk_ranges(len(data), block, world)[rank]
    view = memoryview(data).cast("B")[s:e] if not hasattr(data, "dtype") else data[s:e]
    if s == e and not final:  # a rank beyond the last chunk adds nothing
        part, ck = b"", (1 if fmt == deflate.Format.Zlib else 0)
    else:
        part, ck = (part_fn or compress_part)(view, level, fmt, block, final)
    meta = [None] * world
    dist.all_gather_object(meta, (len(part), ck, e - s), group=group)
    parts = [None] * world if rank == 0 else None
    dst = 0 if group is None else dist.get_global_rank(group, 0)
    dist.gather_object(part, parts, dst=dst, group=group)
    if rank != 0:
        return None
    return frame(parts, [m[1] for m in meta], [m[2] for m in meta], fmt)
