"""The reference's own inflate (orot's deflate_decompress) as a secondary
round-trip check, run in child processes.

orot's inflate can crash on some inputs and rejects some valid streams, so it
never runs inside the test process: a child loads oracle/_ref/liborot_ref.so
(the reference built from its sources by oracle/Makefile.ref), decodes the
streams of a record file one by one and prints one result line per stream.
When the child dies, the stream it was decoding is recorded as a crash and a
new child resumes after it.  Test infrastructure only.

Record file: per stream, a 17-byte header (format u8, expected length u64 LE,
stream length u64 LE) and the stream bytes.
Result codes: the deflate_result the reference returned, and `ok` = 1 when it
returned DEFLATE_OK with exactly the expected bytes.
"""
from __future__ import annotations

import os
import struct
import subprocess
import sys
import tempfile

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
REF_SO = os.path.join(ROOT, "oracle", "_ref", "liborot_ref.so")
CRASH = -100  # result code recorded for a stream the child died on

# deflate_result values (include/orot/deflate.h:15-25 of the reference)
NAMES = {0: "OK", 1: "STREAM_END", 2: "NEED_INPUT", 3: "NEED_OUTPUT", -1: "DATA_ERROR", -2: "MEM_ERROR",
         -3: "BUF_ERROR", -4: "VERSION_ERROR", -5: "PARAM_ERROR", CRASH: "CRASH"}


def available() -> bool:
    return os.path.exists(REF_SO)


def _child(path: str, start: int, expected_path: str) -> None:
    """Runs in the child: decodes records start.. of `path`."""
    import ctypes
    import hashlib
    L = ctypes.CDLL(REF_SO)
    L.deflate_decompress.restype = ctypes.c_int
    L.deflate_decompress.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t,
                                     ctypes.POINTER(ctypes.c_size_t), ctypes.c_int]
    with open(expected_path) as f:
        digests = f.read().split()
    out = sys.stdout
    with open(path, "rb") as f:
        i = 0
        while True:
            h = f.read(17)
            if len(h) < 17:
                break
            fmt, n_exp, n_blob = struct.unpack("<BQQ", h)
            blob = f.read(n_blob)
            if i >= start:
                out.write(f"start {i}\n")
                out.flush()
                cap = n_exp + 1024
                buf = ctypes.create_string_buffer(cap)
                got = ctypes.c_size_t(0)
                r = L.deflate_decompress(blob, len(blob), buf, cap, ctypes.byref(got), fmt)
                ok = int(r == 0 and got.value == n_exp and hashlib.sha256(buf.raw[:n_exp]).hexdigest() == digests[i])
                out.write(f"done {i} {r} {ok}\n")
                out.flush()
            i += 1


def inflate_many(items, timeout: float = 600.0):
    """items: list of (format, original bytes, stream bytes).  Returns a list
    of (result code, ok) in the same order."""
    import hashlib
    n = len(items)
    res = [None] * n
    with tempfile.TemporaryDirectory() as td:
        rec = os.path.join(td, "streams.bin")
        exp = os.path.join(td, "expected.txt")
        with open(rec, "wb") as f:
            for fmt, orig, blob in items:
                f.write(struct.pack("<BQQ", int(fmt), len(orig), len(blob)))
                f.write(blob)
        with open(exp, "w") as f:
            f.write("\n".join(hashlib.sha256(orig).hexdigest() for _, orig, _ in items))
        start = 0
        while start < n:
            try:
                p = subprocess.run([sys.executable, os.path.abspath(__file__), rec, str(start), exp],
                                   capture_output=True, text=True, timeout=timeout)
                stdout, rc, err = p.stdout, p.returncode, p.stderr
            except subprocess.TimeoutExpired as e:  # a stream the reference never finishes decoding
                stdout = e.stdout.decode() if isinstance(e.stdout, bytes) else (e.stdout or "")
                rc, err = -9, "timeout"
            current = None
            for line in stdout.splitlines():
                parts = line.split()
                if parts[0] == "start":
                    current = int(parts[1])
                elif parts[0] == "done":
                    res[int(parts[1])] = (int(parts[2]), int(parts[3]))
                    current = None
            if current is not None:       # the child died while decoding `current`
                res[current] = (CRASH, 0)
                start = current + 1
            elif rc != 0 and res[start] is None:
                raise RuntimeError(f"orot inflate child failed to start: {err[-2000:]}")
            else:
                start = n
    return res


if __name__ == "__main__":
    _child(sys.argv[1], int(sys.argv[2]), sys.argv[3])
