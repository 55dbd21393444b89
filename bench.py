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
             (groups of buffers in flight so copies overlap kernels);
  plain      one pass per buffer on a sample (device-resident and through
             deflate_compress), the comparison the batch is measured against;
  roofline   the dominant kernel phase against the measured HBM copy peak;
  cpu_baseline  the reference's own deflate_compress (oracle/_ref) on the
             host cores over a bounded sample;
  serving    Poisson arrivals (2,000 requests/s, 4 KiB-16 MiB, 70% level 1 /
             30% level 6, raw) through the continuous-batching server: p50/p99
             latency and sustained GB/s; then the server's capacity (the
             trace submitted at once; mixed, level 1 and level 6) beside the
             plain path.
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

METRIC = "deflate_compress_GBps_batched"
UNIT = "GB/s"
WORKLOAD = "10000 zlib buffers, log-uniform 1 KiB-4 MiB, mixed text/ints/zeros/random, level 1, one pass"
HBM_FALLBACK_GBS = 6650.0
# DRAM bytes (read + write) per input byte of the walk kernel, measured by ncu
# (dram__bytes_read.sum + dram__bytes_write.sum) on the first 600 buffers of
# this workload (301.5 MB): 602 MB + 850 MB.  Every term of that traffic is per
# byte or per tile, so it is scaled by the input size for the full launch.
WALK_DRAM_BYTES_PER_INPUT_BYTE = (602.359296e6 + 850.131200e6) / 301540590


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
    ap.add_argument("--serve-requests", type=int, default=2000)
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
def _serve(deflate, srv, buf, trace, gaps):
    """Submits the trace (arrival gaps in seconds, or None for all at once)
    and waits for every result; returns latencies (s) and the makespan from
    first submission to last completion."""
    sizes, levels, starts, outs, ooff = trace
    n = len(sizes)
    tickets = [0] * n
    t0 = time.perf_counter()
    due = t0
    for i in range(n):
        if gaps is not None:
            due += gaps[i]
            now = time.perf_counter()
            if due > now:
                time.sleep(due - now)
        tickets[i] = srv.submit(buf[starts[i]:starts[i] + sizes[i]], levels[i], deflate.Format.Raw,
                                out=outs[ooff[i]:ooff[i + 1]])
    lat = []
    for i in range(n):
        o, l = srv.wait(tickets[i], timeout=600)
        if o is None:
            raise SystemExit(f"served request {i} failed")
        lat.append(l)
    return np.array(lat), time.perf_counter() - t0


def _plain(deflate, buf, trace, k):
    """The same requests through deflate_compress, one call after another
    (service time with no queueing)."""
    sizes, levels, starts = trace[0], trace[1], trace[2]
    pl = []
    tp = time.perf_counter()
    for i in range(k):
        a = time.perf_counter()
        deflate.compress(buf[starts[i]:starts[i] + sizes[i]], levels[i], deflate.Format.Raw)
        pl.append(time.perf_counter() - a)
    tp = time.perf_counter() - tp
    return {"requests": k, "GBps": sum(sizes[:k]) / tp / 1e9,
            "p50_ms": float(np.percentile(np.array(pl) * 1e3, 50)),
            "p99_ms": float(np.percentile(np.array(pl) * 1e3, 99))}


def measure_serving(deflate, buf, total, count, rate, seed=0):
    """Serving: raw DEFLATE requests, sizes log-uniform in 4 KiB-16 MiB, cut
    from the mixed workload buffer, through the continuous-batching server
    (16 GiB device budget).
      open_loop   Poisson arrivals at `rate` requests/s, 70% level 1 / 30%
                  level 6: p50/p99 latency (submission to completion, timed by
                  the server) and sustained GB/s (bytes over first submission
                  to last completion; bounded by the offered rate).
      capacity    the same trace submitted at once, and the level-1-only and
                  level-6-only variants: the sustained GB/s the server reaches
                  when requests queue, beside the plain path (one
                  deflate_compress per request) on a prefix of the same trace.
    A sample of served results is checked byte for byte against single
    deflate_compress calls."""
    from orot_b200 import synth
    rng = np.random.default_rng(13 + seed)
    sizes = [int(x) for x in synth.loguniform_sizes(count, 4096, 16 << 20, 13 + seed)]
    mix = [1 if u < 0.7 else 6 for u in rng.random(count)]
    starts = [int(rng.integers(0, max(1, total - n))) for n in sizes]
    gaps = rng.exponential(1.0 / rate, count)
    caps = [deflate.compress_bound(n, deflate.Format.Raw) for n in sizes]
    outs = np.empty(sum(caps), np.uint8)
    ooff = np.concatenate([[0], np.cumsum(caps)])
    nbytes = sum(sizes)
    srv = deflate.Server(device_budget=16 << 30, lanes=3)
    res = {"requests": count, "rate_req_s": rate, "offered_GBps": nbytes / gaps.sum() / 1e9,
           "levels": "70% L1 / 30% L6", "format": "raw", "sizes": "log-uniform 4 KiB-16 MiB", "budget_GiB": 16}
    trace = (sizes, mix, starts, outs, ooff)
    lat, span = _serve(deflate, srv, buf, trace, gaps)
    for i in range(0, count, max(1, count // 25)):
        ref = deflate.compress(buf[starts[i]:starts[i] + sizes[i]], mix[i], deflate.Format.Raw)
        if outs[ooff[i]:ooff[i] + len(ref)].tobytes() != ref:
            raise SystemExit(f"served request {i} differs from deflate_compress")
    lat_ms = lat * 1e3
    res["open_loop"] = {"sustained_GBps": nbytes / span / 1e9, "p50_ms": float(np.percentile(lat_ms, 50)),
                        "p99_ms": float(np.percentile(lat_ms, 99))}
    k = min(count, 200)
    cap = {}
    for name, lv in (("mix", mix), ("L1", [1] * count), ("L6", [6] * count)):
        tr = (sizes, lv, starts, outs, ooff)
        lat, span = _serve(deflate, srv, buf, tr, None)
        plain = _plain(deflate, buf, tr, k)
        cap[name] = {"GBps": nbytes / span / 1e9, "p50_ms": float(np.percentile(lat * 1e3, 50)),
                     "p99_ms": float(np.percentile(lat * 1e3, 99)), "plain": plain,
                     "vs_plain": nbytes / span / 1e9 / plain["GBps"]}
    passes, inflight = srv.stats()
    srv.close()
    res["capacity"] = cap
    res["passes"] = passes
    res["max_passes_in_flight"] = inflight
    res["plain_note"] = "one deflate_compress per request, back to back, on the first 200 requests"
    return res


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
    dom = max(phases, key=phases.get)
    peak, peak_kind = measured_hbm()
    algo_bytes = total + comp  # input read once + compressed bits written once
    walk_ms = phases.get("walk", 0.0)
    achieved = algo_bytes / (walk_ms / 1e3) / 1e9 if walk_ms > 0 else None
    traffic = (WALK_DRAM_BYTES_PER_INPUT_BYTE * total) if WALK_DRAM_BYTES_PER_INPUT_BYTE else None
    roofline = {"bound": "hbm", "kernel": "k_walk (fast-level LZ77 + fixed Huffman)", "achieved": achieved,
                "peak": peak, "unit": UNIT, "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                "peak_source": peak_kind, "dominant_phase": dom,
                "phase_ms": {k: round(v, 3) for k, v in phases.items() if v > 0}}
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

    # -- end to end through the public API (pinned host buffers)
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
               "api": "deflate_gpu_compress_pipelined (pinned host buffers, 512 MiB groups, 4 passes in flight)"}

    # -- serving: Poisson arrivals through the continuous-batching server
    serving = None
    if args.serve_requests > 0 and world == 1:  # a one-GPU measurement; scaling runs skip it
        serving = measure_serving(deflate, buf, total, args.serve_requests, args.serve_rate, seed=rank)

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
                       "parallelism": f"replicas x{world}"},
            "ratio": ratio, "gpu_launches": launches_per_pass * args.steps, "e2e": e2e, "plain": plain,
            "roofline": roofline, "cpu_baseline": cpu, "clocks": clk.summary(), "serving": serving,
            "device_verify": device_verify,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
