"""The reference's own unit tests for this path, run against the engine.

orot's tests/unit/test_deflate_{roundtrip,levels,formats,simd,parallel}.cpp
call only the public C API (include/orot/deflate.h).  oracle/Makefile.ref
compiles them unchanged from the reference's sources and links them the way
a program switching to the GPU engine links: liborot_b200.so first, the
reference's own static library after it, so every deflate_* symbol they call
(compress, parallel compress, decompress, crc32, adler32, bound) resolves to
the engine.  Each binary must exit 0 with no FAIL line.  The binaries are
built where the reference's sources are, and travel prebuilt."""
import os
import subprocess

import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
UNIT = os.path.join(ROOT, "oracle", "_ref", "unit")
TESTS = ["test_deflate_roundtrip", "test_deflate_levels", "test_deflate_formats", "test_deflate_simd",
         "test_deflate_parallel"]

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", TESTS)
def test_reference_unit_test_passes_on_engine(gpu, name):
    exe = os.path.join(UNIT, name)
    assert os.path.exists(exe), f"{exe} is not built (make -f oracle/Makefile.ref REF=<reference tree> unit)"
    # the binary resolves its deflate_* symbols to the engine's library
    nm = subprocess.run(["nm", "-u", exe], capture_output=True, text=True).stdout
    assert "deflate_compress" in nm or "deflate_parallel_compress" in nm or "deflate_crc32" in nm
    p = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert p.returncode == 0 and "FAIL" not in p.stdout + p.stderr, (p.returncode, p.stdout[-3000:], p.stderr[-3000:])
    assert "PASS" in p.stdout
