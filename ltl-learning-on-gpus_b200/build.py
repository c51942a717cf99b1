"""Build libltlgpu.so and the ltli6463-compatible executable in-tree (sm_100a)."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_build")
INCLUDE = os.path.join(ROOT, "include")
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden",
                  "--expt-relaxed-constexpr", "-I", INCLUDE, "-I", CSRC]
LIB = os.path.join(OUT, "libltlgpu.so")
CLI = os.path.join(OUT, "ltli6463")

LIB_SOURCES = ["learn.cu", "engine.cu", "scarlet.cpp", "noalloc.cu", "mlp.cu", "evaluate.cu"]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(verbose_ptxas: bool = False) -> str:
    os.makedirs(OUT, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".hpp", ".h"))]
    headers.append(os.path.join(INCLUDE, "ltlgpu.h"))
    objs = []
    for src in LIB_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OUT, src + ".o")
        if _newer(o, [s] + headers):
            extra = ["-Xptxas", "-v"] if verbose_ptxas and src.endswith(".cu") else []
            lang = [] if src.endswith(".cu") else ["-x", "cu"]
            _run([NVCC] + CUFLAGS + extra + lang + ["-c", s, "-o", o])
        objs.append(o)
    if _newer(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"])
    cli_src = [os.path.join(CSRC, "cli_ltli6463.cpp"), os.path.join(CSRC, "scarlet.cpp")]
    if _newer(CLI, cli_src + headers + [LIB]):
        _run(["g++", "-O2", "-std=c++17", "-I", INCLUDE, "-I", CSRC] + cli_src +
             ["-L", OUT, "-lltlgpu", "-Wl,-rpath,$ORIGIN", "-o", CLI])
    return LIB


if __name__ == "__main__":
    build(verbose_ptxas="-v" in sys.argv)
