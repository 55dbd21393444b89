"""GPU test of deflate_gpu_compress_noalloc, the entry point for callers that
cannot let a library allocate device memory (they own all of it, e.g. through
a host framework's pool or a fixed budget).  It must produce exactly the bytes
of deflate_compress, on two calls in a row that share its static scratch
array, and reject inputs above its stated maximum.  Collected last so that a
run stopping at the first failure has already run every other test."""
import ctypes

import pytest

from orot_b200 import synth

pytestmark = pytest.mark.gpu


def _bind(L):
    c = ctypes
    L.deflate_gpu_compress_noalloc.restype = c.c_int
    L.deflate_gpu_compress_noalloc.argtypes = [c.c_void_p, c.c_size_t, c.c_void_p, c.c_size_t, c.c_int, c.c_int,
                                               c.c_void_p, c.c_void_p]
    return L


def test_noalloc_equals_deflate_compress(gpu):
    import torch
    L = _bind(gpu.lib())
    # two calls in a row; the second is smaller, so stale scratch from the
    # first would show up if the kernel read anything it did not write
    cases = [(700001, synth.TEXT, 1, 1), (3001, synth.ZEROS, 1, 2), (65536, synth.MIXED, 2, 0),
             (1 << 20, synth.RANDOM, 3, 1), (0, synth.TEXT, 1, 0), (100, synth.TEXT, 0, 2)]
    for n, kind, level, fmt in cases:
        data = synth.gen(n, kind, 7 * n + 1)
        ref = gpu.compress(data, level, gpu.Format(fmt))
        d_in = torch.tensor(list(data) or [0], dtype=torch.uint8, device="cuda")
        cap = L.deflate_compress_bound(n, fmt)
        d_out = torch.zeros(cap, dtype=torch.uint8, device="cuda")
        d_size = torch.zeros(1, dtype=torch.int64, device="cuda")
        torch.cuda.synchronize()
        rc = L.deflate_gpu_compress_noalloc(d_in.data_ptr(), n, d_out.data_ptr(), cap, level, fmt,
                                            d_size.data_ptr(), None)
        assert rc == 0, gpu.last_error()
        torch.cuda.synchronize()
        size = int(d_size.item())
        assert size == len(ref), (n, kind, level, fmt)
        assert d_out[:size].cpu().numpy().tobytes() == ref, (n, kind, level, fmt)


def test_noalloc_rejects_what_it_cannot_do(gpu):
    import torch
    L = _bind(gpu.lib())
    big = 1 << 20
    d = torch.zeros(big + 1, dtype=torch.uint8, device="cuda")
    o = torch.zeros(2 * big, dtype=torch.uint8, device="cuda")
    s = torch.zeros(1, dtype=torch.int64, device="cuda")
    assert L.deflate_gpu_compress_noalloc(d.data_ptr(), big + 1, o.data_ptr(), 2 * big, 1, 0, s.data_ptr(), None) == -2
    assert L.deflate_gpu_compress_noalloc(d.data_ptr(), 10, o.data_ptr(), 2 * big, 6, 0, s.data_ptr(), None) == -3
    assert L.deflate_gpu_compress_noalloc(d.data_ptr(), 100, o.data_ptr(), 50, 1, 0, s.data_ptr(), None) == -4
    assert "larger" in gpu.last_error() or "capacity" in gpu.last_error()
