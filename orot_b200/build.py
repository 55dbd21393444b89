"""Builds the native parts of orot_b200 in-tree.

  orot_b200/liborot_b200.so   CUDA kernels + C ABI (include/orot_b200.h), sm_100a
  orot_b200/libsynth.so       seeded synthetic inputs for tests and benchmarks

`python -m orot_b200.build` or `build_all()`.  Objects go to orot_b200/_build.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_SOURCES = ["kernels_fast.cu", "kernels_lazy.cu", "kernels_common.cu", "engine.cu", "batch.cu", "server.cu",
              "shard.cu", "kernels_inflate.cu", "inflate.cu",
              "members.cu", "stream.cu"]
LIB = os.path.join(HERE, "liborot_b200.so")
SYNTH = os.path.join(HERE, "libsynth.so")


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd))
    return r.stdout + r.stderr


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_cuda(verbose_ptxas: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(HERE, "..", "include", "orot_b200.h"))
    objs = []
    log = ""
    for src in CU_SOURCES:
        path = os.path.join(CSRC, src)
        if not os.path.exists(path):
            continue
        obj = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(obj)
        if _stale(obj, [path] + headers) or verbose_ptxas:
            cmd = [NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-O3",
                   "-c", path, "-o", obj]
            if verbose_ptxas:
                cmd.insert(1, "-Xptxas=-v")
            log += _run(cmd)
    if _stale(LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcuda"])
    return log


def build_synth() -> None:
    src = os.path.join(CSRC, "synth.cpp")
    if _stale(SYNTH, [src]):
        _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-o", SYNTH, src])


def build_all(verbose_ptxas: bool = False) -> str:
    build_synth()
    return build_cuda(verbose_ptxas)


if __name__ == "__main__":
    out = build_all(verbose_ptxas="-v" in sys.argv)
    if out:
        print(out)
