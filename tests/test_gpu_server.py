"""GPU tests of the continuous-batching server and the pipelined batch.

The server admits requests that arrive while other passes run into the next
pass; each request is its own stream, so its bytes must be identical alone
(deflate_compress) and in any mix, and a request whose output does not fit
must fail alone without disturbing the requests batched with it."""
import random
import threading
import time

import numpy as np
import pytest

from orot_b200 import synth

pytestmark = pytest.mark.gpu


def _requests(count, seed, max_size=2 << 20):
    rng = random.Random(seed)
    out = []
    for i in range(count):
        n = int(np.exp(rng.uniform(np.log(1), np.log(max_size))))
        kind = rng.randint(0, 5)
        level = rng.choice([0, 1, 1, 1, 2, 3, 6, 6, 9])
        fmt = rng.randint(0, 2)
        out.append((synth.gen(n, kind, seed * 1000 + i), level, fmt))
    return out


def test_server_alone_equals_mix(gpu):
    reqs = _requests(80, 1)
    singles = [gpu.compress(d, lv, gpu.Format(f)) for d, lv, f in reqs]
    srv = gpu.Server(device_budget=4 << 30, lanes=3)
    tickets = [srv.submit(d, lv, gpu.Format(f)) for d, lv, f in reqs]
    for t, ref in zip(tickets, singles):
        out, lat = srv.wait(t, timeout=120)
        assert out == ref
        assert lat >= 0
    passes, _ = srv.stats()
    assert passes >= 1
    srv.close()


def test_server_large_requests_alone_equal_mix(gpu):
    """The serving workload's largest class (4-16 MiB, levels 1 and 6) mixed
    with small requests and submitted while earlier passes run: each result
    equals its single deflate_compress call byte for byte."""
    rng = random.Random(5)
    reqs = []
    for i in range(36):
        if i % 3 == 0:
            n = int(np.exp(rng.uniform(np.log(4 << 20), np.log(16 << 20))))
        else:
            n = int(np.exp(rng.uniform(np.log(4 << 10), np.log(4 << 20))))
        reqs.append((synth.gen(n, synth.MIXED if i % 2 else rng.randint(0, 5), 500 + i), rng.choice([1, 1, 6]), 0))
    singles = [gpu.compress(d, lv, gpu.Format(f)) for d, lv, f in reqs]
    srv = gpu.Server(device_budget=16 << 30, lanes=3)
    tickets = []
    for k, (d, lv, f) in enumerate(reqs):
        tickets.append(srv.submit(d, lv, gpu.Format(f)))
        if k % 6 == 5:
            time.sleep(0.01)  # later requests arrive while earlier passes run
    for t, ref in zip(tickets, singles):
        out, _ = srv.wait(t, timeout=300)
        assert out == ref
    passes, _ = srv.stats()
    assert passes >= 2
    srv.close()


def test_server_poisoned_request_fails_alone(gpu):
    reqs = _requests(12, 2, max_size=1 << 20)
    srv = gpu.Server(lanes=2)
    tickets = []
    for i, (d, lv, f) in enumerate(reqs):
        cap = 8 if i == 5 else None  # far too small: this request must fail alone
        tickets.append(srv.submit(d, lv, gpu.Format(f), out_capacity=cap))
    for i, (t, (d, lv, f)) in enumerate(zip(tickets, reqs)):
        out, _ = srv.wait(t, timeout=120)
        if i == 5 and len(d) > 0:
            assert out is None
        else:
            assert out == gpu.compress(d, lv, gpu.Format(f))
    srv.close()


def test_server_arrivals_overlap_passes(gpu):
    """Requests submitted from another thread while passes run: several
    passes end up in flight together and every result stays exact."""
    reqs = _requests(150, 3, max_size=4 << 20)
    srv = gpu.Server(device_budget=1 << 30, lanes=3)
    tickets = [None] * len(reqs)

    def producer():
        for i, (d, lv, f) in enumerate(reqs):
            tickets[i] = srv.submit(d, lv, gpu.Format(f))
            time.sleep(0.0005)

    th = threading.Thread(target=producer)
    th.start()
    th.join()
    for t, (d, lv, f) in zip(tickets, reqs):
        out, _ = srv.wait(t, timeout=300)
        assert out == gpu.compress(d, lv, gpu.Format(f))
    passes, inflight = srv.stats()
    assert passes >= 2
    assert inflight >= 2
    srv.close()


def test_server_small_budget_still_completes(gpu):
    reqs = [(synth.gen(8 << 20, k, k), 1, 1) for k in range(4)]
    srv = gpu.Server(device_budget=96 << 20, lanes=2)
    ts = [srv.submit(d, lv, gpu.Format(f)) for d, lv, f in reqs]
    for t, (d, lv, f) in zip(ts, reqs):
        out, _ = srv.wait(t, timeout=120)
        assert out == gpu.compress(d, lv, gpu.Format(f))
    srv.close()


def test_pipelined_batch_equals_single_calls(gpu):
    sizes = [int(x) for x in synth.loguniform_sizes(200, 1024, 2 << 20, 7)]
    bufs = [synth.array(n, i % 4, i + 3) for i, n in enumerate(sizes)]
    concat = np.concatenate(bufs)
    out = np.zeros(gpu.packed_bound(sizes, gpu.Format.Zlib), np.uint8)
    end, offs, szs = gpu.compress_pipelined(concat, sizes, 1, gpu.Format.Zlib, out, group_bytes=16 << 20, lanes=3)
    assert end == offs[-1]
    for i, b in enumerate(bufs):
        ref = gpu.compress(b, 1, gpu.Format.Zlib)
        assert szs[i] == len(ref)
        assert out[offs[i]:offs[i] + szs[i]].tobytes() == ref


def test_pipelined_batch_pinned_equals_pageable(gpu):
    """Pageable caller memory is staged through the lanes' pinned buffers;
    pinned caller memory is read and written by DMA directly: same bytes."""
    import torch
    sizes = [int(x) for x in synth.loguniform_sizes(300, 1024, 4 << 20, 8)]
    concat = np.concatenate([synth.array(n, i % 4, i + 5) for i, n in enumerate(sizes)])
    bound = gpu.packed_bound(sizes, gpu.Format.Gzip)
    out_pageable = np.zeros(bound, np.uint8)
    r1 = gpu.compress_pipelined(concat, sizes, 1, gpu.Format.Gzip, out_pageable, group_bytes=32 << 20, lanes=3)
    pin_in = torch.from_numpy(concat).pin_memory().numpy()
    pin_out = torch.zeros(bound, dtype=torch.uint8).pin_memory().numpy()
    r2 = gpu.compress_pipelined(pin_in, sizes, 1, gpu.Format.Gzip, pin_out, group_bytes=32 << 20, lanes=3)
    assert r1[0] == r2[0]
    assert list(r1[1]) == list(r2[1]) and list(r1[2]) == list(r2[2])
    assert out_pageable[:r1[0]].tobytes() == pin_out[:r2[0]].tobytes()
