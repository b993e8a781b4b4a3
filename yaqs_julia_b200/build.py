"""Builds libyaqs_b200.so in-tree with nvcc for sm_100a."""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libyaqs_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
         "-Xcompiler", "-fPIC", "-shared"]


def sources():
    return [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC)) if f.endswith((".cu", ".cuh", ".h"))] + [
        os.path.join(ROOT, "include", f) for f in sorted(os.listdir(os.path.join(ROOT, "include")))]


# translation units, compiled in parallel: engine.cu (every kernel without
# tcgen05 code), engine_tc.cu (the tensor-core trajectory kernel) and
# engine_dg.cu (the digital program in 128-thread CTAs)
UNITS = ["engine.cu", "engine_tc.cu", "engine_dg.cu"]


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and os.path.exists(OUT):
        newest = max(os.path.getmtime(s) for s in sources())
        if os.path.getmtime(OUT) >= newest:
            return OUT
    objs, procs = [], []
    for u in UNITS:
        o = os.path.join(CSRC, u.replace(".cu", ".o"))
        cmd = [NVCC] + [f for f in FLAGS if f != "-shared"] + (["-Xptxas", "-v"] if verbose else []) + [
            "-c", "-o", o, os.path.join(CSRC, u)]
        procs.append(subprocess.Popen(cmd))
        objs.append(o)
    for p in procs:
        if p.wait() != 0:
            raise subprocess.CalledProcessError(p.returncode, "nvcc")
    subprocess.run([NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", OUT] + objs, check=True)
    for o in objs:
        os.remove(o)
    return OUT


if __name__ == "__main__":
    print(build(force=True, verbose=True))
