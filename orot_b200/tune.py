"""Autotuner for the pass geometry: `python -m orot_b200.tune` on a B200.

For each level group and pass-size class it times every candidate geometry
on the device and keeps the fastest, then rewrites csrc/geometry_table.h
(the table Engine::plan reads; rebuild the library afterwards) and prints a
report of every timing.

  level 1      tile bytes at 12 hash bits (one warp walks one tile)
  levels 2-3   tile bytes at 14 hash bits (timed at level 2)
  levels 4-6, 7-9, 10-12
               tiles per CTA run (timed at levels 6, 9 and 12)

Workload per class: one buffer of the class size below 16 MiB, else
buffers log-uniform in 1 KiB-4 MiB up to the class size, all from the mixed
generator (Zipf text, sorted integers, zeros, random bytes), deflate_compress
semantics, zlib framing.  Each candidate is set through the engine's
OROT_B200_TILE / OROT_B200_LAZY_RUN overrides; the output bytes do not depend
on it (tested).  Timing: CUDA events around graph replays after a warm-up.
The hash widths of levels 1-3 are not tuned: they fix the reference's token
stream.
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
TABLE = os.path.join(HERE, "csrc", "geometry_table.h")
CLASSES = [0, 1 << 20, 4 << 20, 16 << 20, 64 << 20, 256 << 20, 1 << 30, 4 << 30]
CLASS_BYTES = [256 << 10, 1 << 20, 4 << 20, 16 << 20, 64 << 20, 256 << 20, 1 << 30, 4 << 30]
TILES12 = [4096, 8192, 16384, 32768, 65536]
TILES14 = [8192, 16384, 32768, 65536]
RUNS = [1, 2, 4, 8, 16, 32]
# largest class timed per level (larger classes take the last timed result)
MAX_CLASS = {1: 4 << 30, 2: 4 << 30, 6: 1 << 30, 9: 1 << 30, 12: 256 << 20}


def workload(nbytes: int, seed: int):
    from . import synth
    if nbytes < (16 << 20):
        sizes = [nbytes]
    else:
        sizes, acc, k = [], 0, 0
        cand = synth.loguniform_sizes(200000, 1024, 4 << 20, seed)
        while acc < nbytes:
            n = int(min(cand[k], nbytes - acc))
            sizes.append(n)
            acc += n
            k += 1
    buf = np.empty(sum(sizes) + 64, np.uint8)
    o = 0
    for i, n in enumerate(sizes):
        synth.fill(buf[o:o + n], synth.MIXED if n >= (16 << 20) else i % 4, seed * 7919 + i)
        o += n
    return buf[:o], sizes


def time_pass(deflate, torch, stream, data, sizes, level, env: dict, reps: int) -> float:
    """Milliseconds per pass with the engine overrides in `env`."""
    saved = {k: os.environ.get(k) for k in env}
    os.environ.update({k: str(v) for k, v in env.items()})
    try:
        b = deflate.DeviceBatch()  # reads the overrides when its engine is made
        b.load(data, sizes, level, deflate.Format.Zlib)
    finally:
        for k, v in saved.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    sh = stream.cuda_stream
    b.run(stream=sh, graph=True)
    b.run(stream=sh, graph=True)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        b.run(stream=sh, graph=True)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    if any(s == 0 for s in b.sizes()):
        raise SystemExit("a stream failed while tuning")
    b.close()
    return ms


def write_table(rows, source: str, path: str = TABLE) -> None:
    text = open(TABLE).read()  # the header comment and struct stay as they are
    head = text[:text.index("constexpr const char* kGeometrySource")]
    body = [f'constexpr const char* kGeometrySource = "{source}";', "constexpr GeometryRow kGeometry[] = {"]
    for r in rows:
        mb = r["min_bytes"]
        lit = "0ull" if mb == 0 else (f"{mb >> 30}ull << 30" if mb % (1 << 30) == 0 else f"{mb >> 20}ull << 20")
        body.append(f"    {{{lit}, {r['tile12']}, {r['tile14']}, {{{r['run'][0]}, {r['run'][1]}, {r['run'][2]}}}}},")
    body.append("};")
    body.append("")
    body.append("}  // namespace orotb")
    open(path, "w").write(head + "\n".join(body) + "\n")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--max-bytes", type=int, default=4 << 30, help="skip classes above this size")
    ap.add_argument("--out", default=TABLE)
    ap.add_argument("--report", default=None, help="also write the timings as JSON here")
    args = ap.parse_args()
    import torch
    from . import deflate
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    props = torch.cuda.get_device_properties(0)
    report = {"device": props.name, "sms": props.multi_processor_count, "timings": []}
    best = {}  # (level, class index) -> (value, ms)
    for ci, (lo, nbytes) in enumerate(zip(CLASSES, CLASS_BYTES)):
        if nbytes > args.max_bytes:
            continue
        data, sizes = workload(nbytes, 11 + ci)
        for level, knob, cands in ((1, "OROT_B200_TILE", TILES12), (2, "OROT_B200_TILE", TILES14),
                                   (6, "OROT_B200_LAZY_RUN", RUNS), (9, "OROT_B200_LAZY_RUN", RUNS),
                                   (12, "OROT_B200_LAZY_RUN", RUNS)):
            if nbytes > MAX_CLASS[level]:
                continue
            res = []
            for c in cands:
                ms = time_pass(deflate, torch, stream, data, sizes, level, {knob: c}, args.reps)
                res.append((ms, c))
                report["timings"].append({"class_min_bytes": lo, "pass_bytes": int(data.size), "buffers": len(sizes),
                                          "level": level, "knob": knob, "value": c, "ms": ms,
                                          "GBps": data.size / ms / 1e6})
            ms, c = min(res)
            best[(level, ci)] = (c, ms)
            print(f"class >= {lo >> 20} MiB ({data.size / 1e6:.1f} MB, {len(sizes)} buffers) level {level}: "
                  + ", ".join(f"{v}: {t:.3f} ms" for t, v in res) + f" -> {c}", flush=True)
        del data
    rows = []
    last = {}
    for ci, lo in enumerate(CLASSES):
        for level in (1, 2, 6, 9, 12):
            if (level, ci) in best:
                last[level] = best[(level, ci)][0]
        rows.append({"min_bytes": lo, "tile12": last.get(1, 65536), "tile14": last.get(2, 65536),
                     "run": [last.get(6, 16), last.get(9, 16), last.get(12, 16)]})
    stamp = datetime.date.today().isoformat()
    write_table(rows, f"orot_b200.tune on {props.name}, {props.multi_processor_count} SMs, {stamp}", args.out)
    report["table"] = rows
    if args.report:
        with open(args.report, "w") as f:
            json.dump(report, f, indent=1)
    print(json.dumps(rows))


if __name__ == "__main__":
    sys.exit(main())
