"""Builds libloom_gpu.so in-tree for sm_100a (python -m loom_b200.build)."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = [os.path.join(HERE, "csrc", "loom_gpu.cu"), os.path.join(HERE, "csrc", "gp_noalloc.cu"),
       os.path.join(HERE, "csrc", "p2_host.cpp")]
OUT = os.path.join(HERE, "libloom_gpu.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
         "-Xcompiler", "-fPIC", "-shared"]


def sources():
    d = os.path.join(HERE, "csrc")
    return [os.path.join(d, f) for f in sorted(os.listdir(d)) if f.endswith((".cu", ".cuh", ".h", ".cpp", ".inc"))] + \
        [os.path.join(HERE, "..", "include", "loom_gpu.h")]


def up_to_date() -> bool:
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(s) <= t for s in sources())


FIELD_SRC = os.path.join(HERE, "csrc", "field.cuh")
FIELD_INC = os.path.join(HERE, "csrc", "field_src.inc")


def write_field_inc() -> None:
    """field.cuh as a C++ raw string literal: the run-time compiler of the
    constraint kernels (csrc/xjit.cuh) includes it from memory."""
    with open(FIELD_SRC) as f:
        text = f.read()
    if ')LGFIELD"' in text:
        raise RuntimeError("field.cuh contains the raw-string delimiter")
    body = 'R"LGFIELD(' + text + ')LGFIELD"\n'
    old = None
    if os.path.exists(FIELD_INC):
        with open(FIELD_INC) as f:
            old = f.read()
    if old != body:
        with open(FIELD_INC, "w") as f:
            f.write(body)


def build(force: bool = False, verbose: bool = False) -> str:
    write_field_inc()
    if not force and up_to_date():
        return OUT
    cmd = [NVCC] + FLAGS + ["-o", OUT] + SRC
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(OUT)
