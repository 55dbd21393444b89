"""GPU parity for levels 0-3 (stored + orot's greedy fast path).

These levels are token-exact restatements of the reference, so the CUDA
engine's bytes must equal the reference's: checked against the golden
SHA-256s produced by the reference itself and against the oracle on larger,
multi-tile inputs where the parse crosses tile boundaries.  Every call goes
through the C ABI (orot_b200.deflate -> liborot_b200.so)."""
import hashlib
import random
import zlib

import numpy as np
import pytest

from conftest import inflate
from orot_b200 import synth

pytestmark = pytest.mark.gpu


def sha(b):
    return hashlib.sha256(b).hexdigest()[:24]


def test_golden_fast_levels_byte_identical(gpu, golden):
    cache = {}
    checked = 0
    for c in golden["cases"]:
        if c["level"] > 3:
            continue
        key = (c["kind"], c["n"], c["seed"])
        if key not in cache:
            cache[key] = synth.gen(c["n"], c["kind"], c["seed"])
        d = cache[key]
        if c["path"] == "whole":
            out = gpu.compress(d, c["level"], gpu.Format(c["fmt"]))
        else:
            out = gpu.ParallelCompressor(c["level"], gpu.Format(c["fmt"]), 0, c["block"]).compress(d)
        assert (len(out), sha(out)) == (c["len"], c["sha256"]), c
        checked += 1
    assert checked > 1000


def test_checksums(gpu, golden, oracle):
    for k in golden["kats"]:
        d = bytes.fromhex(k["data_hex"])
        got = gpu.crc32(d, k["init"]) if k["fn"] == "crc32" else gpu.adler32(d, k["init"])
        assert got == k["value"], k
    for k in golden["gen_kats"]:
        d = synth.gen(k["n"], k["kind"], k["seed"])
        assert gpu.crc32(d, k["init"]) == k["crc32"]
        assert gpu.adler32(d, k["adler_init"]) == k["adler32"]
    rng = random.Random(3)
    for n in [1, 3, 4, 255, 256, 257, 1023, 65535, 65536, 65537, 200003, 3 << 20]:
        d = synth.gen(n, rng.randint(0, 5), n)
        init = rng.randint(0, 0xFFFFFFFF)
        assert gpu.crc32(d, init) == oracle.crc32(d, init) == zlib.crc32(d, init)
        a0 = rng.randint(0, 65520) | (rng.randint(0, 65520) << 16)
        assert gpu.adler32(d, a0) == oracle.adler32(d, a0) == zlib.adler32(d, a0)
    # incremental == one shot (test_deflate_simd.cpp:45-56)
    d = synth.gen(300000, 0, 9)
    assert gpu.crc32(d[1000:], gpu.crc32(d[:1000])) == gpu.crc32(d)
    assert gpu.adler32(d[77777:], gpu.adler32(d[:77777])) == gpu.adler32(d)


@pytest.mark.parametrize("kind", [0, 1, 2, 3, 4, 5])
@pytest.mark.parametrize("level", [1, 2])
def test_multi_tile_whole_buffer_matches_oracle(gpu, oracle, kind, level):
    """Inputs spanning many tiles: carried hash tables and parse fix-up must
    reproduce the single sequential parse exactly."""
    for n in [16385, 70001, 1 << 20, (3 << 20) + 5]:
        d = synth.gen(n, kind, 31 * n + kind)
        for fmt in (0, 1, 2):
            out = gpu.compress(d, level, gpu.Format(fmt))
            ref = oracle.compress(d, level, fmt)
            assert out == ref, (n, kind, level, fmt, len(out), len(ref))
        assert inflate(out, 2) == d


def parallel_c(gpu, data, level, fmt, block, cap):
    """deflate_parallel_compress through the C ABI with an explicit capacity."""
    import ctypes
    L = gpu.lib()
    ctx = L.deflate_parallel_new(level, fmt, 8, block)
    out = ctypes.create_string_buffer(cap)
    r = L.deflate_parallel_compress(ctx, data, len(data), out, cap)
    L.deflate_parallel_free(ctx)
    return out.raw[:r]


@pytest.mark.parametrize("block", [0, 1000, 32768, 65537, 262144])
def test_parallel_fast_matches_oracle(gpu, oracle, block):
    for kind in (0, 2, 4, 5):
        d = synth.gen(900001, kind, block + kind)
        for level in (0, 1, 3):
            for fmt in (0, 1, 2):
                out = parallel_c(gpu, d, level, fmt, block, 2 * len(d) + 1024)
                ref = oracle.parallel(d, level, fmt, block)
                assert out == ref, (kind, level, fmt, block)
    assert inflate(out, 2) == d


def test_parallel_overflow_returns_zero(gpu, oracle):
    """Stored chunks of 1000 bytes cost 5 bytes each, so the pigz stream is
    larger than deflate_compress_bound(); the reference writes past such a
    buffer (src/parallel/parallel_compressor.cpp:108-120 never checks), the
    engine returns 0 instead."""
    import ctypes
    d = synth.gen(900001, 3, 1)
    L = gpu.lib()
    bound = L.deflate_compress_bound(len(d), 2)
    assert len(oracle.parallel(d, 0, 2, 1000)) > bound
    assert parallel_c(gpu, d, 0, 2, 1000, bound) == b""


def test_empty_and_tiny_inputs(gpu, oracle):
    for n in range(0, 12):
        d = bytes(range(n))
        for level in (0, 1, 2, 3):
            for fmt in (0, 1, 2):
                assert gpu.compress(d, level, gpu.Format(fmt)) == oracle.compress(d, level, fmt)
    # the reference's empty raw stream: final empty stored block
    assert gpu.compress(b"", 1, gpu.Format.Raw) == bytes.fromhex("010000ffff")
    assert gpu.ParallelCompressor(1, gpu.Format.Raw).compress(b"") == oracle.parallel(b"", 1, 0)


def test_level_clamp(gpu, oracle):
    d = synth.gen(5000, 0, 1)
    assert gpu.compress(d, -5, gpu.Format.Gzip) == oracle.compress(d, -5, 2)


def test_capacity_rules(gpu):
    import ctypes
    L = gpu.lib()
    d = synth.gen(10000, 3, 5)
    bound = L.deflate_compress_bound(len(d), 1)
    out = ctypes.create_string_buffer(bound)
    assert L.deflate_compress(d, len(d), out, bound, 1, 1) > 0
    assert L.deflate_compress(d, len(d), out, bound - 1, 1, 1) == 0
    ctx = L.deflate_parallel_new(1, 1, 0, 0)
    small = ctypes.create_string_buffer(100)
    assert L.deflate_parallel_compress(ctx, d, len(d), small, 100) == 0
    L.deflate_parallel_free(ctx)


def test_large_mixed_roundtrip(gpu, oracle):
    d = synth.array(64 << 20, synth.MIXED, 77).tobytes()
    out = gpu.compress(d, 1, gpu.Format.Zlib)
    assert zlib.decompress(out) == d
    assert out == oracle.compress(d, 1, 1)


def test_device_batch_equals_single_calls(gpu):
    rng = np.random.default_rng(5)
    sizes = [int(x) for x in synth.loguniform_sizes(60, 1, 1 << 20, 4)] + [0, 1, 2]
    bufs = [synth.gen(n, i % 4, i) for i, n in enumerate(sizes)]
    b = gpu.DeviceBatch()
    b.load(b"".join(bufs), sizes, 1, gpu.Format.Zlib)
    for graph in (False, True, True):
        b.run(graph=graph)
        got = b.sizes()
        for i, d in enumerate(bufs):
            single = gpu.compress(d, 1, gpu.Format.Zlib)
            assert got[i] == len(single)
            assert b.output(i, got[i]) == single
    assert b.launches() > 0
    b.close()


def test_launch_count_matches_the_kernels_of_a_pass(gpu):
    """deflate_gpu_batch_launches counts every kernel of a pass: at level 1
    with a multi-tile buffer and zlib framing that is k_lastocc, k_carry_scan,
    k_cand_parse (the candidate pass and the parse in one kernel), k_fix1,
    k_fix2, k_plan_seg, k_plan_stream, k_plan_pieces, k_zero, k_join,
    k_ck_block, k_ck_fold and k_frame (13); raw output drops the two checksum
    kernels."""
    d = synth.gen(3 << 20, synth.MIXED, 2)
    for fmt, want in ((gpu.Format.Zlib, 13), (gpu.Format.Raw, 11)):
        b = gpu.DeviceBatch()
        b.load(d, [len(d)], 1, fmt)
        b.run()
        assert b.launches() == want
        b.close()


_FUSED_CASES = "[(k, n, lv) for k, n in ((0, 3 << 20), (2, 1 << 20), (4, 5 << 20), (5, 700001), (1, 2 << 20)) for lv in (1, 2, 3)]"
_FUSED_SCRIPT = """
import hashlib, sys
sys.path.insert(0, {root!r})
from orot_b200 import deflate, synth
for k, n, lv in {cases}:
    print(hashlib.sha256(deflate.compress(synth.gen(n, k, 31 + k), lv, deflate.Format.Raw)).hexdigest())
"""


def test_fused_and_separate_kernels_same_bytes(gpu):
    """The candidate pass and the parse run as one kernel (k_cand_parse) by
    default; OROT_B200_FUSED=0 runs them as k_cand then k_parse.  Both give
    the same bytes at every fast level, multi-tile buffers included."""
    import hashlib
    import os
    import subprocess
    import sys
    cases = eval(_FUSED_CASES)
    fused = [hashlib.sha256(gpu.compress(synth.gen(n, k, 31 + k), lv, gpu.Format.Raw)).hexdigest()
             for k, n, lv in cases]
    root = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
    env = dict(os.environ, OROT_B200_FUSED="0")
    p = subprocess.run([sys.executable, "-c", _FUSED_SCRIPT.format(root=root, cases=_FUSED_CASES)], env=env,
                       capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    assert p.stdout.split() == fused
