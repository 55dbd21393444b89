"""CPU tests of the oracle: the C restatement against the reference's own
golden outputs and known answers, and the corrected Huffman limiter."""
import hashlib
import os
import random
import zlib

import numpy as np
import pytest

from conftest import REF_SO, inflate
from orot_b200 import synth


def test_checksum_kats(oracle, golden):
    for k in golden["kats"]:
        d = bytes.fromhex(k["data_hex"])
        got = oracle.crc32(d, k["init"]) if k["fn"] == "crc32" else oracle.adler32(d, k["init"])
        assert got == k["value"], k
    assert oracle.crc32(b"123456789") == 0xCBF43926
    assert oracle.adler32(b"Wikipedia") == 0x11E60398


def test_checksum_generated_vectors(oracle, golden):
    for k in golden["gen_kats"]:
        d = synth.gen(k["n"], k["kind"], k["seed"])
        assert oracle.crc32(d, k["init"]) == k["crc32"]
        assert oracle.adler32(d, k["adler_init"]) == k["adler32"]
        assert zlib.crc32(d, k["init"]) == k["crc32"]
        assert zlib.adler32(d, k["adler_init"]) == k["adler32"]


def _golden_inputs(golden):
    cache = {}
    for c in golden["cases"]:
        key = (c["kind"], c["n"], c["seed"])
        if key not in cache:
            cache[key] = synth.gen(c["n"], c["kind"], c["seed"])
        yield c, cache[key]


def test_oracle_reproduces_reference_bytes(oracle, golden):
    """With the reference's clamping limiter the restatement is byte-identical
    to every golden output of the reference."""
    oracle.L.oracle_set_mode(0)
    try:
        for c, d in _golden_inputs(golden):
            if c["path"] == "whole":
                out = oracle.compress(d, c["level"], c["fmt"])
            else:
                out = oracle.parallel(d, c["level"], c["fmt"], c["block"])
            assert len(out) == c["len"], c
            assert hashlib.sha256(out).hexdigest()[:24] == c["sha256"], c
    finally:
        oracle.L.oracle_set_mode(1)


def test_corrected_oracle_is_valid_and_close(oracle, golden):
    """The corrected oracle always inflates.  Levels 0-9 without a limiter
    event are byte-identical to the reference; where the reference's stream
    is valid the corrected one is at most 3% larger."""
    oracle.L.oracle_set_mode(1)
    for c, d in _golden_inputs(golden):
        before = oracle.L.oracle_limiter_events()
        if c["path"] == "whole":
            out = oracle.compress(d, c["level"], c["fmt"])
        else:
            out = oracle.parallel(d, c["level"], c["fmt"], c["block"])
        fired = oracle.L.oracle_limiter_events() != before
        assert inflate(out, c["fmt"]) == d, c
        if not fired and c["level"] <= 9:
            assert hashlib.sha256(out).hexdigest()[:24] == c["sha256"], c
        if c["valid"]:
            assert len(out) <= 1.03 * c["len"] + 8, c


def _kraft(lens, limit):
    return sum(2 ** (limit - l) for l in lens if l)


@pytest.mark.parametrize("nsym,limit", [(288, 15), (32, 15), (19, 7)])
def test_huffman_limiter(oracle, nsym, limit):
    rng = random.Random(nsym)
    fib = [1, 1]
    while len(fib) < nsym:
        fib.append(fib[-1] + fib[-2])
    cases = [fib[:nsym], [rng.randint(0, 5) for _ in range(nsym)], [1] * nsym, [0] * (nsym - 1) + [9],
             [rng.choice([0, 1, 1000000]) for _ in range(nsym)], [2 ** min(i, 30) for i in range(nsym)]]
    for f in cases:
        freq = np.array([min(x, 2 ** 31) for x in f], np.uint32)
        lens = np.zeros(nsym, np.uint8)
        oracle.L.oracle_huffman_lengths(freq.ctypes.data, nsym, lens.ctypes.data, limit)
        used = int((freq > 0).sum())
        assert all((lens > 0) == (freq > 0))
        assert lens.max(initial=0) <= limit
        if used >= 2:
            assert _kraft(lens.tolist(), limit) == 2 ** limit
        elif used == 1:
            assert lens.max() == 1


@pytest.mark.skipif(not os.path.exists(REF_SO), reason="reference not built here")
def test_oracle_matches_reference_library_randomized(oracle):
    """Differential run against the compiled reference on fresh random cases."""
    import ctypes
    c = ctypes
    R = c.CDLL(REF_SO)
    R.deflate_compress.restype = c.c_size_t
    R.deflate_compress.argtypes = [c.c_void_p, c.c_size_t, c.c_void_p, c.c_size_t, c.c_int, c.c_int]
    rng = random.Random(7)
    oracle.L.oracle_set_mode(0)
    try:
        for _ in range(60):
            n = rng.choice([rng.randint(0, 64), rng.randint(64, 5000), rng.randint(5000, 200000)])
            kind = rng.randint(0, 5)
            d = synth.gen(n, kind, rng.randint(0, 1 << 30))
            lvl, fmt = rng.randint(0, 12), rng.randint(0, 2)
            cap = 2 * n + 256
            buf = c.create_string_buffer(cap)
            r = R.deflate_compress(d, n, buf, cap, lvl, fmt)
            assert oracle.compress(d, lvl, fmt) == buf.raw[:r], (n, kind, lvl, fmt)
    finally:
        oracle.L.oracle_set_mode(1)
