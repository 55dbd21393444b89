"""Generates tests/golden/reference_vectors.json from the reference itself.

Run where the daramkun/orot sources are, after building the reference from
them (REF names the source tree):

    make -f oracle/Makefile.ref REF=<reference tree>   # oracle/_ref/liborot_ref.so
    python tests/golden/make_golden.py

For every case (input kind/size/seed from orot_b200.synth, level, format,
whole-buffer or parallel path) the file records the length and SHA-256 of
the reference's compressed output and whether zlib inflates it back to the
input.  Inputs are regenerated at test time from the seeded generator, so the
fixture stays small.  Checksum known answers are the reference's own KATs
(tests/unit/test_deflate_formats.cpp:74-88) plus the reference's values over
generated inputs.
"""
import ctypes
import hashlib
import json
import os
import sys
import zlib

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)
from orot_b200 import synth  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref", "liborot_ref.so")

SIZES = [0, 1, 2, 3, 4, 5, 31, 32, 33, 257, 258, 259, 1000, 4097, 32767, 32768, 32769, 65537, 140000]
KINDS = [0, 1, 2, 3, 5]
LEVELS = [0, 1, 2, 3, 4, 6, 9, 12]
WBITS = {0: -15, 1: 15, 2: 31}


def load_ref():
    L = ctypes.CDLL(REF)
    c = ctypes
    L.deflate_compress.restype = c.c_size_t
    L.deflate_compress.argtypes = [c.c_void_p, c.c_size_t, c.c_void_p, c.c_size_t, c.c_int, c.c_int]
    L.deflate_parallel_new.restype = c.c_void_p
    L.deflate_parallel_new.argtypes = [c.c_int, c.c_int, c.c_int, c.c_size_t]
    L.deflate_parallel_compress.restype = c.c_size_t
    L.deflate_parallel_compress.argtypes = [c.c_void_p, c.c_void_p, c.c_size_t, c.c_void_p, c.c_size_t]
    L.deflate_parallel_free.argtypes = [c.c_void_p]
    L.deflate_crc32.restype = c.c_uint32
    L.deflate_crc32.argtypes = [c.c_uint32, c.c_void_p, c.c_size_t]
    L.deflate_adler32.restype = c.c_uint32
    L.deflate_adler32.argtypes = [c.c_uint32, c.c_void_p, c.c_size_t]
    return L


def inflates(blob, fmt, data):
    try:
        return zlib.decompress(blob, WBITS[fmt]) == data
    except zlib.error:
        return False


def main():
    L = load_ref()
    cases = []
    for n in SIZES:
        for kind in KINDS:
            seed = 1000 * kind + n
            data = synth.gen(n, kind, seed)
            cap = 2 * n + 256
            out = ctypes.create_string_buffer(cap)
            for lvl in LEVELS:
                for fmt in (0, 1, 2):
                    r = L.deflate_compress(data, n, out, cap, lvl, fmt)
                    blob = out.raw[:r]
                    cases.append(dict(kind=kind, n=n, seed=seed, level=lvl, fmt=fmt, path="whole", block=0,
                                      len=r, sha256=hashlib.sha256(blob).hexdigest()[:24], valid=inflates(blob, fmt, data)))
                if n >= 1000 and lvl in (1, 6, 9):
                    for block in (0, 32768):
                        ctx = L.deflate_parallel_new(lvl, 2, 2, block)
                        r = L.deflate_parallel_compress(ctx, data, n, out, cap)
                        L.deflate_parallel_free(ctx)
                        blob = out.raw[:r]
                        cases.append(dict(kind=kind, n=n, seed=seed, level=lvl, fmt=2, path="parallel", block=block,
                                          len=r, sha256=hashlib.sha256(blob).hexdigest()[:24],
                                          valid=inflates(blob, 2, data)))
    kats = [
        dict(fn="crc32", init=0, data_hex=b"123456789".hex(), value=L.deflate_crc32(0, b"123456789", 9)),
        dict(fn="adler32", init=1, data_hex=b"Wikipedia".hex(), value=L.deflate_adler32(1, b"Wikipedia", 9)),
        dict(fn="crc32", init=0, data_hex="", value=L.deflate_crc32(0, b"", 0)),
        dict(fn="adler32", init=1, data_hex="", value=L.deflate_adler32(1, b"", 0)),
    ]
    gen_kats = []
    for n, kind, seed in [(1, 3, 1), (100, 0, 2), (65536, 3, 3), (65537, 0, 4), (300000, 4, 5), (1 << 20, 1, 6)]:
        d = synth.gen(n, kind, seed)
        for init in (0, 1, 0xDEADBEEF):
            gen_kats.append(dict(kind=kind, n=n, seed=seed, init=init, crc32=L.deflate_crc32(init, d, n),
                                 adler32=L.deflate_adler32(init if init != 0xDEADBEEF else 0x12345, d, n),
                                 adler_init=init if init != 0xDEADBEEF else 0x12345))
    doc = dict(source="daramkun/orot built by oracle/Makefile.ref (no system backends, scalar CRC-32)",
               generator="tests/golden/make_golden.py", cases=cases, kats=kats, gen_kats=gen_kats)
    with open(os.path.join(HERE, "reference_vectors.json"), "w") as f:
        json.dump(doc, f, separators=(",", ":"))
    bad = sum(1 for c in cases if not c["valid"])
    print(f"{len(cases)} cases ({bad} not inflatable by zlib), {len(kats) + len(gen_kats)} checksum vectors")


if __name__ == "__main__":
    main()
