#!/usr/bin/env python3
"""Headline benchmark: batched DEFLATE compression on one (or N) B200s.

Workload: 10,000 independent zlib streams, buffer sizes drawn log-uniformly
from 1 KiB to 4 MiB (seed 11, 5.13 GB), buffer i filled by generator
i mod 4 (Zipf text, sorted u32 deltas, zeros, random bytes; see
orot_b200/synth.py), level 1, deflate_compress semantics per buffer (one
block per buffer, byte-identical to the reference).  All buffers are
compressed by one pass of kernels replayed from a CUDA graph.

Reported (one JSON line from rank 0):
  value      GB/s (decimal, input bytes / device time) with the inputs already
             in HBM, CUDA events on the launching stream, max over ranks;
  e2e        the same through deflate_gpu_compress_pipelined from pinned host
             memory: host->device copies, kernels, packing and the
             device->host copies of every compressed stream inside the timing
             (groups of buffers in flight so copies overlap kernels); and the
             same call from pageable host memory;
  plain      one pass per buffer on a sample (device-resident and through
             deflate_compress), the comparison the batch is measured against;
  roofline   the dominant kernel phase against the measured HBM copy peak and
             against the SM issue rate (its ncu instruction count);
  cpu_baseline  the reference's own deflate_compress (oracle/_ref) on the
             host cores over a bounded sample;
  threads16  deflate_compress called from 16 host threads at once on a 1 GiB
             random sample of the buffers, beside the reference's own
             deflate_compress on the same sample and thread count;
  configs    the other configurations, each with a device-resident value,
             an end-to-end value through orot's own C entry point from
             pageable host memory, its roofline and the reference's entry
             point on the host cores: 16 MiB Zipf text, raw, level 1, whole
             buffer (reference: deflate_compress, one thread); 256 MiB mixed
             data, gzip, level 6, 128 KiB chunks (reference:
             deflate_parallel_compress on all host threads); 1 GiB random,
             8-byte periodic with 1% flips and Zipf text, raw, level 9,
             256 KiB chunks (reference: deflate_parallel_compress on all host
             threads over the first 64 MiB);
  serving    20,000 requests with Poisson arrivals (2,000 requests/s, 4 KiB-
             16 MiB, 70% level 1 / 30% level 6, raw) through the
             continuous-batching server: p50/p99 latency and sustained GB/s,
             every result compared with its single deflate_compress output;
             then the server's capacity (the first 2,000 requests submitted at
             once; mixed, level 1 and level 6) beside the plain path on a
             random sample of 300 of them.
  device_verify  every stream of the batch decoded by the GPU inflate and
             compared with its input on the device (wall time of a second
             call, and of the first, which also allocates the decode arena;
             informational).
Inputs (5.1 GB) exceed the 126 MB L2, so no flush is needed between steps.

`--impl reference` times the reference's CPU implementation on the same
workload (bounded samples per step) and prints the same line.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time
import zlib

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
# Many host threads call the engine at once in some legs (each call on its own
# CUDA stream): let the device run that many streams' work side by side
# instead of the default 8 hardware queues.  Must be set before CUDA starts.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

METRIC = "deflate_compress_GBps_batched"
UNIT = "GB/s"
WORKLOAD = "10000 zlib buffers, log-uniform 1 KiB-4 MiB, mixed text/ints/zeros/random, level 1, one pass"
HBM_FALLBACK_GBS = 6650.0
# DRAM bytes (read + write) per input byte of the dominant kernel, from one
# ncu capture (dram__bytes_read.sum + dram__bytes_write.sum) on a slice of
# this workload; every term of that traffic is per byte or per tile, so it is
# scaled by the input size for the full launch (profiles/k_cand_parse_L1_mixed_300MB.md).
DRAM_BYTES_PER_INPUT_BYTE = {"candidates": (759.450e6 + 703.093e6) / 301540590,
                             "parse": (2088.913e6 + 1095.331e6) / 301540590}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--buffers", type=int, default=10000)
    ap.add_argument("--level", type=int, default=1)
    ap.add_argument("--plain-sample", type=int, default=300)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--serve-requests", type=int, default=20000)
    ap.add_argument("--serve-capacity-requests", type=int, default=2000)
    ap.add_argument("--no-configs", action="store_true", help="skip the whole-buffer, parallel and stress legs")
    ap.add_argument("--no-threads", action="store_true", help="skip the 16-thread deflate_compress leg")
    ap.add_argument("--serve-rate", type=float, default=2000.0)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    return ap.parse_args()


def make_workload(count: int, seed_base: int):
    from orot_b200 import synth
    sizes = [int(x) for x in synth.loguniform_sizes(count, 1024, 4 << 20, 11 + seed_base)]
    offs = np.zeros(count + 1, np.int64)
    offs[1:] = np.cumsum(sizes)
    return sizes, offs


def fill_workload(buf: np.ndarray, sizes, offs, seed_base: int):
    from orot_b200 import synth

    def job(i):
        if sizes[i]:
            synth.fill(buf[offs[i]:offs[i + 1]], i % 4, seed_base * 1000003 + i + 1)

    with cf.ThreadPoolExecutor(max(1, min(16, os.cpu_count() or 1))) as ex:
        list(ex.map(job, range(len(sizes))))


class ClockSampler:
    """nvidia-smi samples (SM clock, max clock, throttle reasons) while running."""

    FIELDS = ("clocks.sm,clocks.max.sm,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.index)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 7:
                continue
            try:
                sm.append(float(p[0]))
                mx.append(float(p[1]))
            except ValueError:
                continue
            for n, v in zip(names, p[3:7]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_hbm():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback"


# ---------------------------------------------------------------- CPU arms
def load_cpu_impl():
    """The reference built from its sources (oracle/_ref), else the oracle port."""
    ref = os.path.join(ROOT, "oracle", "_ref", "liborot_ref.so")
    if os.path.exists(ref):
        L = ctypes.CDLL(ref)
        fn, kind = L.deflate_compress, "reference"
    else:
        port = os.path.join(ROOT, "oracle", "liborot_oracle.so")
        L = ctypes.CDLL(port)
        fn, kind = L.oracle_compress, "port"
    fn.restype = ctypes.c_size_t
    fn.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_int]
    return fn, kind


def cpu_sample_rate(buf, sizes, offs, idx, level, threads):
    """Compresses buffers idx with deflate_compress on `threads` host threads;
    returns (GB/s, bytes, seconds, ratio)."""
    fn, kind = load_cpu_impl()
    base = buf.ctypes.data

    def one(i):
        n = sizes[i]
        cap = n + (n >> 12) + (n >> 14) + (n >> 25) + 13 + 6
        out = ctypes.create_string_buffer(cap)
        r = fn(base + int(offs[i]), n, out, cap, level, 1)
        return r

    t0 = time.perf_counter()
    with cf.ThreadPoolExecutor(threads) as ex:
        outs = list(ex.map(one, idx))
    dt = time.perf_counter() - t0
    nb = sum(sizes[i] for i in idx)
    return nb / dt / 1e9, nb, dt, (sum(outs) / nb if nb else 0.0), kind


def sample_indices(sizes, target_bytes, rng_seed=5):
    rng = np.random.default_rng(rng_seed)
    order = rng.permutation(len(sizes))
    idx, tot = [], 0
    for i in order:
        idx.append(int(i))
        tot += sizes[i]
        if tot >= target_bytes:
            break
    return idx


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    sizes, offs = make_workload(args.buffers, 0)
    buf = np.empty(int(offs[-1]) + 64, np.uint8)
    fill_workload(buf, sizes, offs, 0)
    threads = os.cpu_count() or 1
    per_step = 128 << 20  # bytes per timed step (bounded sample)
    rates, kind, nbytes = [], "reference", 0
    for s in range(args.warmup + args.steps):
        idx = sample_indices(sizes, per_step, 100 + s)
        r, nb, dt, ratio, kind = cpu_sample_rate(buf, sizes, offs, idx, args.level, threads)
        if s >= args.warmup:
            rates.append(r)
            nbytes = nb
    value = statistics.median(rates)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": nbytes / (value * 1e9) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": {"workload": WORKLOAD, "level": args.level, "format": "zlib", "buffers": args.buffers,
                   "step": f"{per_step >> 20} MiB random sample of the buffers per step"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                         "sample": f"{per_step >> 20} MiB of the workload per step, deflate_compress per buffer "
                                   f"on {threads} threads"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------- serving
class OutRing:
    """Output space for served requests, reused in submission order: a
    request's region is handed out only after every request that held it has
    been collected (collection runs in submission order too)."""

    def __init__(self, nbytes: int):
        self.buf = np.empty(nbytes, np.uint8)
        self.head = 0          # next free byte (monotonic)
        self.regions = []      # monotonic starts of the requests not yet collected, oldest first

    def take(self, n: int, collect_oldest):
        """Ring offsets [lo, hi) for n bytes; collects the oldest requests
        first while they still hold any of that space."""
        n = (n + 63) & ~63
        size = self.buf.size
        assert n <= size
        start = self.head  # monotonic byte position
        if start % size + n > size:  # does not fit before the ring's end: start over at its beginning
            start += size - start % size
        # the ring bytes of [start, start + n) were last handed out as
        # [start - size, start + n - size); every request starting there must be collected
        while self.regions and self.regions[0] < start + n - size:
            collect_oldest()
        self.head = start + n
        self.regions.append(start)
        o = start % size
        return o, o + n


def _serve(deflate, srv, buf, trace, gaps, ring, expect=None):
    """Submits the trace (arrival gaps in seconds, or None for all at once)
    while a collector thread waits for the results in submission order,
    frees their output space and, with `expect` (the CRC-32 and size of each
    request's single deflate_compress output), compares every result.
    Returns the latencies (s, submission to completion, timed by the server)
    and the makespan from the first submission to the last completion."""
    import queue
    L = deflate.lib()
    sizes, levels, starts = trace
    n = len(sizes)
    lat = np.zeros(n)
    sub_at = np.zeros(n)
    q = queue.Queue()
    cond = threading.Condition()
    errors = []
    base, rbase = buf.ctypes.data, ring.buf.ctypes.data

    def collector():
        for _ in range(n):
            i, t, lo = q.get()
            sz, lt = ctypes.c_size_t(0), ctypes.c_double(0)
            r = L.deflate_gpu_server_wait(srv._s, t, ctypes.byref(sz), ctypes.byref(lt), 600.0)
            lat[i] = lt.value
            if r != 0:
                errors.append(f"served request {i} failed ({r})")
            elif expect is not None and (zlib.crc32(ring.buf[lo:lo + sz.value]), int(sz.value)) != expect[i]:
                errors.append(f"served request {i} differs from its single deflate_compress call")
            with cond:
                ring.regions.pop(0)
                cond.notify_all()

    th = threading.Thread(target=collector, daemon=True)
    th.start()
    t0 = time.perf_counter()
    due = t0
    for i in range(n):
        if gaps is not None:
            due += gaps[i]
            now = time.perf_counter()
            if due > now:
                time.sleep(due - now)
        cap = deflate_bound(sizes[i])
        with cond:
            lo, hi = ring.take(cap, lambda: cond.wait(1.0))
        sub_at[i] = time.perf_counter()
        t = L.deflate_gpu_server_submit(srv._s, base + starts[i], sizes[i], rbase + lo, cap, levels[i], 0)
        if t == 0:
            raise SystemExit(f"submit {i} failed: {deflate.last_error()}")
        q.put((i, t, lo))
    th.join()
    if errors:
        raise SystemExit(errors[0])
    return lat, float(np.max(sub_at + lat)) - t0


def _single_outputs(L, buf, trace, idx, threads=16):
    """(CRC-32, size) of every request's single deflate_compress output, from
    `threads` host threads calling the C ABI at once."""
    sizes, levels, starts = trace
    base = buf.ctypes.data
    local = threading.local()

    def one(i):
        n = sizes[i]
        cap = n + (n >> 12) + (n >> 14) + (n >> 25) + 13
        o = getattr(local, "out", None)
        if o is None or o.size < cap:
            o = local.out = np.empty(max(cap, 16 << 20), np.uint8)
        r = L.deflate_compress(base + starts[i], n, o.ctypes.data, cap, levels[i], 0)
        if r == 0:
            raise SystemExit(f"deflate_compress failed on request {i}")
        return zlib.crc32(o[:r]), int(r)

    with cf.ThreadPoolExecutor(threads) as ex:
        return list(ex.map(one, idx))


def _plain(L, buf, trace, idx):
    """The requests idx through deflate_compress, one call after another on
    one thread (service time with no queueing)."""
    sizes, levels, starts = trace
    base = buf.ctypes.data
    out = np.empty(max(deflate_bound(max(sizes[i] for i in idx)), 16), np.uint8)
    pl = []
    tp = time.perf_counter()
    for i in idx:
        a = time.perf_counter()
        if L.deflate_compress(base + starts[i], sizes[i], out.ctypes.data, out.size, levels[i], 0) == 0:
            raise SystemExit("deflate_compress failed")
        pl.append(time.perf_counter() - a)
    tp = time.perf_counter() - tp
    nb = sum(sizes[i] for i in idx)
    return {"requests": len(idx), "GBps": nb / tp / 1e9, "p50_ms": float(np.percentile(np.array(pl) * 1e3, 50)),
            "p99_ms": float(np.percentile(np.array(pl) * 1e3, 99))}


def deflate_bound(n: int) -> int:
    return n + (n >> 12) + (n >> 14) + (n >> 25) + 13


def measure_serving(deflate, buf, total, count, rate, cap_count, seed=0):
    """Serving: raw DEFLATE requests, sizes log-uniform in 4 KiB-16 MiB, cut
    from the mixed workload buffer, through the continuous-batching server
    (16 GiB device budget).
      open_loop   `count` requests with Poisson arrivals at `rate` requests/s,
                  70% level 1 / 30% level 6: p50/p99 latency (submission to
                  completion, timed by the server) and sustained GB/s (bytes
                  over first submission to last completion; bounded by the
                  offered rate).  Every result is compared (CRC-32 and size)
                  with the same request's single deflate_compress output.
      capacity    the first `cap_count` requests of the trace submitted at
                  once (mixed, level-1-only and level-6-only): the sustained
                  GB/s the server reaches when requests queue, beside the
                  plain path (one deflate_compress after another) on a random
                  sample of 300 requests of the same trace."""
    from orot_b200 import synth
    L = deflate.lib()
    rng = np.random.default_rng(13 + seed)
    sizes = [int(x) for x in synth.loguniform_sizes(count, 4096, 16 << 20, 13 + seed)]
    mix = [1 if u < 0.7 else 6 for u in rng.random(count)]
    starts = [int(rng.integers(0, max(1, total - n))) for n in sizes]
    gaps = rng.exponential(1.0 / rate, count)
    nbytes = sum(sizes)
    trace = (sizes, mix, starts)
    t0 = time.perf_counter()
    expect = _single_outputs(L, buf, trace, range(count))
    single_s = time.perf_counter() - t0
    srv = deflate.Server(device_budget=16 << 30, lanes=3)
    ring = OutRing(6 << 30)
    res = {"requests": count, "rate_req_s": rate, "offered_GBps": nbytes / gaps.sum() / 1e9,
           "duration_s": float(gaps.sum()), "bytes": nbytes, "levels": "70% L1 / 30% L6", "format": "raw",
           "sizes": "log-uniform 4 KiB-16 MiB", "budget_GiB": 16}
    lat, span = _serve(deflate, srv, buf, trace, gaps, ring, expect)
    lat_ms = lat * 1e3
    res["open_loop"] = {"sustained_GBps": nbytes / span / 1e9, "p50_ms": float(np.percentile(lat_ms, 50)),
                        "p99_ms": float(np.percentile(lat_ms, 99)), "p999_ms": float(np.percentile(lat_ms, 99.9)),
                        "max_ms": float(lat_ms.max()), "verified": count,
                        "verify": "every result equals its single deflate_compress output (CRC-32 and size)"}
    cap = {}
    k = min(cap_count, count)
    sample = sorted(np.random.default_rng(77 + seed).choice(k, size=min(300, k), replace=False).tolist())
    for name, lv in (("mix", mix[:k]), ("L1", [1] * k), ("L6", [6] * k)):
        tr = (sizes[:k], lv, starts[:k])
        exp = expect[:k] if name == "mix" else None
        lat, span = _serve(deflate, srv, buf, tr, None, ring, exp)
        plain = _plain(L, buf, tr, sample)
        kb = sum(sizes[:k])
        cap[name] = {"requests": k, "GBps": kb / span / 1e9, "p50_ms": float(np.percentile(lat * 1e3, 50)),
                     "p99_ms": float(np.percentile(lat * 1e3, 99)), "plain": plain,
                     "vs_plain": kb / span / 1e9 / plain["GBps"]}
    passes, inflight = srv.stats()
    srv.close()
    res["capacity"] = cap
    res["passes"] = passes
    res["max_passes_in_flight"] = inflight
    res["plain_note"] = ("one deflate_compress per request, back to back on one thread, on a random sample of 300 "
                         f"of the first {k} requests")
    res["single_call_reference_s"] = single_s
    return res


# ---------------------------------------------------------------- the other configurations
# ncu figures of the dominant kernels (profiles/): warp instructions per
# input byte, for the issue-rate roofline (4 warp instructions per SM cycle).
# The "parse" phase is k_cand_parse, the candidate pass and the parse in one
# kernel (the "candidates" phase is empty then).
WARP_INST_PER_BYTE = {"candidates": 3.65, "parse": 12.07, "lazy_match": 77.4}
PHASE_KERNEL = {"candidates": "k_cand", "parse": "k_cand_parse",  "lazy_match": "k_lz", "lazy_encode": "k_enc", "lazy_huffman": "k_huff",
                "hash_carry": "k_lastocc + k_carry_scan", "fixup": "k_fix1 + k_fix2", "join": "k_join",
                "checksum": "k_ck_block + k_ck_fold", "plan": "k_plan + k_zero"}


def roofline_of(phases, nbytes, comp, sm_mhz, sms):
    """Dominant phase of a pass against the HBM copy peak and, where ncu gave
    its instruction count, against the SM issue rate."""
    dom = max(phases, key=phases.get)
    peak, kind = measured_hbm()
    ms = phases[dom]
    achieved = (nbytes + comp) / (ms / 1e3) / 1e9
    r = {"bound": "hbm", "kernel": PHASE_KERNEL.get(dom, dom), "dominant_phase": dom, "achieved": achieved,
         "peak": peak, "unit": UNIT, "frac": achieved / peak, "peak_source": kind,
         "phase_ms": {k: round(v, 3) for k, v in phases.items() if v > 0}}
    if dom in WARP_INST_PER_BYTE and sm_mhz:
        inst_rate = WARP_INST_PER_BYTE[dom] * nbytes / (ms / 1e3)      # warp instructions / s
        issue_peak = sms * 4 * sm_mhz * 1e6
        r["issue"] = {"warp_inst_per_input_byte": WARP_INST_PER_BYTE[dom], "achieved_warp_inst_per_s": inst_rate,
                      "peak_warp_inst_per_s": issue_peak, "frac": inst_rate / issue_peak,
                      "note": "instructions per byte from the kernel's ncu capture; peak = SMs x 4 x median SM clock"}
    return r


def load_reference():
    """The reference built from its sources (oracle/_ref), for the CPU arms."""
    path = os.path.join(ROOT, "oracle", "_ref", "liborot_ref.so")
    L = ctypes.CDLL(path)
    c = ctypes
    L.deflate_compress.restype = c.c_size_t
    L.deflate_compress.argtypes = [c.c_void_p, c.c_size_t, c.c_void_p, c.c_size_t, c.c_int, c.c_int]
    L.deflate_parallel_new.restype = c.c_void_p
    L.deflate_parallel_new.argtypes = [c.c_int, c.c_int, c.c_int, c.c_size_t]
    L.deflate_parallel_free.argtypes = [c.c_void_p]
    L.deflate_parallel_compress.restype = c.c_size_t
    L.deflate_parallel_compress.argtypes = [c.c_void_p, c.c_void_p, c.c_size_t, c.c_void_p, c.c_size_t]
    return L


def cpu_reference(data: np.ndarray, level, fmt, parallel, block, threads, reps=2):
    """The reference's own entry point on the host cores: deflate_compress on
    one thread (whole buffer) or deflate_parallel_compress with `threads`
    workers.  Returns (GB/s, compressed size) of the best of `reps` runs."""
    L = load_reference()
    n = data.size
    cap = 2 * n + (1 << 20)
    out = np.empty(cap, np.uint8)
    best, size = 1e30, 0
    for _ in range(reps):
        t0 = time.perf_counter()
        if parallel:
            ctx = L.deflate_parallel_new(level, fmt, threads, block)
            r = L.deflate_parallel_compress(ctx, data.ctypes.data, n, out.ctypes.data, cap)
            L.deflate_parallel_free(ctx)
        else:
            r = L.deflate_compress(data.ctypes.data, n, out.ctypes.data, cap, level, fmt)
        best = min(best, time.perf_counter() - t0)
        size = int(r)
    return n / best / 1e9, size


def measure_config(deflate, name, data: np.ndarray, level, fmt, parallel, block, stream, sh, steps, cpu_bytes,
                   cpu_threads, sm_mhz, sms):
    """One buffer compressed by deflate_compress (whole) or the pigz-style
    parallel path: device-resident passes (graph replay, CUDA events), the
    same call end to end through the C ABI from host memory, the on-chip
    roofline of its dominant kernel, a zlib round trip of the output, and the
    reference's own entry point on the host cores."""
    import torch
    L = deflate.lib()
    n = data.size
    b = deflate.DeviceBatch()
    b.load(data, [n], level, deflate.Format(fmt), parallel=parallel, block_size=block)
    for _ in range(2):
        b.run(stream=sh, graph=True)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        b.run(stream=sh, graph=True)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    comp = b.sizes()[0]
    out = b.output(0, comp)
    if zlib.decompress(out, {0: -15, 1: 15, 2: 31}[fmt]) != data.tobytes():
        raise SystemExit(f"{name}: output does not round-trip under zlib")
    b.profile(True)
    b.run(stream=sh)
    torch.cuda.synchronize()
    phases = b.phase_ms()
    b.profile(False)
    launches = b.launches()
    b.close()
    # end to end through the C ABI: pageable host input and output, the
    # library's own staging and copies inside the timing
    cap = 2 * n + (1 << 20)
    host_out = np.empty(cap, np.uint8)
    if parallel:
        ctx = L.deflate_parallel_new(level, fmt, 0, block)

        def call():
            return L.deflate_parallel_compress(ctx, data.ctypes.data, n, host_out.ctypes.data, cap)
    else:
        def call():
            return L.deflate_compress(data.ctypes.data, n, host_out.ctypes.data, cap, level, fmt)
    call()
    reps = 3
    t0 = time.perf_counter()
    for _ in range(reps):
        r = call()
    e2e_s = (time.perf_counter() - t0) / reps
    if parallel:
        L.deflate_parallel_free(ctx)
    if r != comp or host_out[:r].tobytes() != out:
        raise SystemExit(f"{name}: the C ABI call differs from the device-resident pass")
    res = {"value": n / (ms / 1e3) / 1e9, "unit": UNIT, "ms_per_step": ms, "bytes": n, "ratio": comp / n,
           "gpu_launches_per_step": launches,
           "e2e": {"value": n / e2e_s / 1e9, "unit": UNIT, "ms_per_step": e2e_s * 1e3, "h2d_bytes_per_step": n,
                   "d2h_bytes_per_step": int(comp),
                   "api": ("deflate_parallel_compress" if parallel else "deflate_compress") +
                          " (pageable host buffers)"},
           "roofline": roofline_of(phases, n, comp, sm_mhz, sms)}
    try:
        sample = data[:cpu_bytes] if cpu_bytes < n else data
        v, csize = cpu_reference(sample, level, fmt, parallel, block, cpu_threads)
        res["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": 1 if not parallel else cpu_threads,
                               "kind": "reference",
                               "sample": (f"first {sample.size >> 20} MiB of the input" if sample.size < n
                                          else "the whole input") + ", " +
                                         ("deflate_parallel_compress, num_threads = %d" % cpu_threads if parallel
                                          else "deflate_compress on one thread"),
                               "ratio": csize / sample.size}
        res["vs_cpu_baseline"] = res["e2e"]["value"] / v
        if sample.size == n:
            res["size_vs_reference"] = comp / csize
    except OSError:
        res["cpu_baseline"] = None
    return res


def measure_threads(deflate, buf, sizes, offs, level, threads, sample_bytes):
    """deflate_compress from `threads` host threads at once over a random
    sample of the batch's buffers (zlib), each thread with its own output
    buffer: what a multithreaded program gets from the drop-in entry point.
    The reference's own deflate_compress runs the same sample on the same
    number of threads."""
    L = deflate.lib()
    idx = sample_indices(sizes, sample_bytes, 31)
    base = buf.ctypes.data
    local = threading.local()

    def one(i):
        n = sizes[i]
        cap = n + (n >> 12) + (n >> 14) + (n >> 25) + 19
        o = getattr(local, "out", None)
        if o is None:
            o = local.out = np.empty((4 << 20) + (1 << 16), np.uint8)
        r = L.deflate_compress(base + int(offs[i]), n, o.ctypes.data, cap, level, 1)
        if r == 0:
            raise SystemExit("deflate_compress failed")
        return int(r)

    with cf.ThreadPoolExecutor(threads) as ex:
        # warm every engine: its arenas grow to the largest buffers once
        biggest = sorted(idx, key=lambda i: -sizes[i])[:threads * 4]
        list(ex.map(one, biggest))
        list(ex.map(one, idx[:threads * 8]))
        t0 = time.perf_counter()
        outs = list(ex.map(one, idx))
        dt = time.perf_counter() - t0
    nb = sum(sizes[i] for i in idx)
    ref, _, _, _, kind = cpu_sample_rate(buf, sizes, offs, idx, level, threads)
    return {"value": nb / dt / 1e9, "unit": UNIT, "threads": threads, "buffers": len(idx), "bytes": nb,
            "ratio": sum(outs) / nb, "api": "deflate_compress (pageable host buffers), one call per buffer",
            "reference": {"value": ref, "unit": UNIT, "threads": threads, "kind": kind},
            "vs_reference": nb / dt / 1e9 / ref}


# ---------------------------------------------------------------- GPU arm
def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from orot_b200 import deflate

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # -- workload (weak scaling: every rank compresses its own 4 GiB batch)
    sizes, offs = make_workload(args.buffers, rank)
    total = int(offs[-1])
    pinned = torch.empty(total + 64, dtype=torch.uint8, pin_memory=True)
    buf = pinned.numpy()
    fill_workload(buf, sizes, offs, rank)

    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    sh = stream.cuda_stream

    b = deflate.DeviceBatch()
    b.load(buf[:total], sizes, args.level, deflate.Format.Zlib)
    for _ in range(args.warmup):
        b.run(stream=sh, graph=True)
    torch.cuda.synchronize()

    # -- timed region (device-resident)
    barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            b.run(stream=sh, graph=True)
        ev1.record(stream)
        torch.cuda.synchronize()
    barrier()
    ms = ev0.elapsed_time(ev1) / args.steps
    ms = max_over_ranks(ms)
    value = world * total / (ms / 1e3) / 1e9
    launches_per_pass = b.launches()

    out_sizes = b.sizes()
    if any(s == 0 for s in out_sizes):
        raise SystemExit("a stream failed to compress")
    comp = sum(out_sizes)
    ratio = comp / total
    # round-trip check on a sample of the streams (zlib on the host) and of
    # every stream on the device (decoded by the GPU inflate, compared with
    # its input, framing and trailer checked)
    for i in sample_indices(sizes, 64 << 20, 9)[:200]:
        o = b.output(i, out_sizes[i])
        if zlib.decompress(o) != buf[offs[i]:offs[i + 1]].tobytes():
            raise SystemExit(f"stream {i} does not round-trip")
    t0 = time.perf_counter()
    vok = b.verify()
    first_s = time.perf_counter() - t0  # includes allocating the decode arena
    if not all(vok):
        raise SystemExit(f"{len(vok) - sum(vok)} streams fail the on-device round trip")
    t0 = time.perf_counter()
    vok = b.verify()
    verify_s = time.perf_counter() - t0
    if not all(vok):
        raise SystemExit(f"{len(vok) - sum(vok)} streams fail the on-device round trip")
    device_verify = {"streams": len(vok), "ok": int(sum(vok)), "wall_ms": verify_s * 1e3,
                     "first_call_ms": first_s * 1e3, "inflate_GBps_wall": total / verify_s / 1e9}

    # -- per-phase times (profiled passes, events between phases)
    b.profile(True)
    phases = {}
    nprof = 2
    for _ in range(nprof):
        b.run(stream=sh)
        for k, v in b.phase_ms().items():
            phases[k] = phases.get(k, 0.0) + v / nprof
    b.profile(False)
    clocks = clk.summary()
    sms = torch.cuda.get_device_properties(local).multi_processor_count
    roofline = roofline_of(phases, total, comp, clocks.get("sm_mhz"), sms)
    tb = DRAM_BYTES_PER_INPUT_BYTE.get(roofline["dominant_phase"])
    roofline["traffic"] = tb * total if tb else None
    roofline["traffic_note"] = "ncu DRAM bytes per input byte of the dominant kernel on a slice of the workload, scaled"
    b.close()

    # -- plain path: one pass per buffer (device-resident) and deflate_compress per buffer
    plain = None
    if args.plain_sample > 0 and world == 1:
        idx = sample_indices(sizes, 1 << 62, 3)[:args.plain_sample]
        single = []
        for i in idx:
            sb = deflate.DeviceBatch()
            sb.load(buf[offs[i]:offs[i + 1]], [sizes[i]], args.level, deflate.Format.Zlib)
            sb.run(stream=sh)
            single.append(sb)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for sb in single:
            sb.run(stream=sh)
        e1.record(stream)
        torch.cuda.synchronize()
        pbytes = sum(sizes[i] for i in idx)
        pms = e0.elapsed_time(e1)
        for sb in single:
            sb.close()
        t0 = time.perf_counter()
        for i in idx:
            deflate.compress(buf[offs[i]:offs[i + 1]], args.level, deflate.Format.Zlib)
        pe2e = time.perf_counter() - t0
        plain = {"value": pbytes / (pms / 1e3) / 1e9, "e2e": pbytes / pe2e / 1e9, "unit": UNIT,
                 "sample_buffers": len(idx), "sample_bytes": pbytes}

    # -- end to end through the public API (pinned host buffers; then pageable)
    e2e = None
    if not args.no_e2e:
        obound = deflate.packed_bound(sizes, deflate.Format.Zlib)
        outp = torch.empty(obound, dtype=torch.uint8, pin_memory=True).numpy()
        sizes_u64 = np.asarray(sizes, np.uint64)
        deflate.compress_pipelined(buf[:total], sizes_u64, args.level, deflate.Format.Zlib, outp)  # warm-up
        barrier()
        t0 = time.perf_counter()
        steps_e2e = max(1, min(args.steps, 3))
        packed = 0
        for _ in range(steps_e2e):
            packed, poffs, psz = deflate.compress_pipelined(buf[:total], sizes_u64, args.level, deflate.Format.Zlib,
                                                            outp)
        dt = (time.perf_counter() - t0) / steps_e2e
        barrier()
        dt = max_over_ranks(dt)
        if psz.tolist() != out_sizes:
            raise SystemExit("end-to-end sizes differ from the device-resident pass")
        e2e = {"value": world * total / dt / 1e9, "unit": UNIT, "h2d_bytes_per_step": total,
               "d2h_bytes_per_step": int(comp) + 16 * (len(sizes) + 1), "ms_per_step": dt * 1e3,
               "api": "deflate_gpu_compress_pipelined (pinned host buffers, 256 MiB groups, 6 passes in flight)"}
        if world == 1:
            # the same call from pageable (not pinned) input and output memory
            pin = np.empty(total, np.uint8)
            pin[:] = buf[:total]
            pout = np.empty(obound, np.uint8)
            deflate.compress_pipelined(pin, sizes_u64, args.level, deflate.Format.Zlib, pout)
            t0 = time.perf_counter()
            _, _, psz2 = deflate.compress_pipelined(pin, sizes_u64, args.level, deflate.Format.Zlib, pout)
            dtp = time.perf_counter() - t0
            if psz2.tolist() != out_sizes:
                raise SystemExit("pageable end-to-end sizes differ")
            e2e["pageable"] = {"value": total / dtp / 1e9, "unit": UNIT, "ms_per_step": dtp * 1e3}
            del pin, pout

    # -- deflate_compress from 16 host threads at once (drop-in entry point)
    threads16 = None
    if world == 1 and not args.no_threads:
        threads16 = measure_threads(deflate, buf, sizes, offs, args.level, 16, 1 << 30)

    # -- the other configurations: whole-buffer text, pigz-style gzip and level-9 stress
    configs = None
    if world == 1 and not args.no_configs:
        from orot_b200 import synth
        nth = os.cpu_count() or 1
        sm = clocks.get("sm_mhz")
        configs = {}
        text = synth.array(16 << 20, synth.TEXT, 42)
        configs["text_16MiB_raw_L1_whole"] = measure_config(
            deflate, "text", text, 1, 0, False, 0, stream, sh, 10, 16 << 20, 1, sm, sms)
        mixed = synth.array(256 << 20, synth.MIXED, 7)
        configs["mixed_256MiB_gzip_L6_parallel_128KiB"] = measure_config(
            deflate, "mixed", mixed, 6, 2, True, 128 << 10, stream, sh, 3, 256 << 20, nth, sm, sms)
        del mixed
        for nm, kind, seed in (("random", synth.RANDOM, 99), ("periodic_1pct_flips", synth.PERIODIC, 98),
                               ("text", synth.TEXT, 97)):
            d = synth.array(1 << 30, kind, seed)
            configs[f"stress_1GiB_{nm}_raw_L9_parallel_256KiB"] = measure_config(
                deflate, nm, d, 9, 0, True, 256 << 10, stream, sh, 2, 64 << 20, nth, sm, sms)
            del d

    # -- serving: Poisson arrivals through the continuous-batching server
    serving = None
    if args.serve_requests > 0 and world == 1:  # a one-GPU measurement; scaling runs skip it
        serving = measure_serving(deflate, buf, total, args.serve_requests, args.serve_rate,
                                  args.serve_capacity_requests, seed=rank)

    # -- CPU baseline: the reference on the host cores (rank 0, N = 1 only)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        idx = sample_indices(sizes, 1 << 30, 21)
        r, nb, dt, cratio, kind = cpu_sample_rate(buf, sizes, offs, idx, args.level, threads)
        cpu = {"value": r, "unit": UNIT, "cores": threads, "kind": kind,
               "sample": f"{len(idx)} buffers, {nb / 1e6:.0f} MB, deflate_compress per buffer on {threads} threads",
               "ratio": cratio}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u8", "data": "synthetic",
            "config": {"workload": WORKLOAD, "buffers": args.buffers, "bytes_per_gpu": total, "level": args.level,
                       "format": "zlib", "graph": True, "l2": "inputs larger than L2 (no flush)",
                       "parallelism": f"replicas x{world}", "geometry": deflate.geometry_source()},
            "ratio": ratio, "gpu_launches": launches_per_pass * args.steps, "e2e": e2e, "plain": plain,
            "roofline": roofline, "cpu_baseline": cpu, "clocks": clocks, "threads16": threads16,
            "configs": configs, "serving": serving, "device_verify": device_verify,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
