"""Builds the engine's native libraries in-tree (no JIT cache).

  libcgbdsm.so  the C-ABI engine (include/cgbdsm.h): CUDA kernels for sm_100a
                plus the C++ host runtime (query planner, CaLiG producer, CLI
                entry points)
  libcgbgen.so  seeded synthetic workload generator (graphs, streams, queries)
  cgbdsm        drop-in command-line program (reference main_calig.cpp)

Usage: python -m cgbdsm_b200.build [--force]
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
NVCC = os.environ.get("CGB_NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
CXX = "/usr/bin/g++"  # system compiler: dynamic libstdc++ (safe to load into Python)
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

ENGINE_CU = ["engine.cu", "noalloc.cu", "gpma.cu"]
ENGINE_CPP = ["query.cpp", "calig.cpp", "pipeline.cpp", "server.cpp"]
GEN_CPP = ["gen.cpp"]


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd: list[str]) -> None:
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(force: bool = False, verbose_ptxas: bool = False) -> dict[str, str]:
    out = {}
    os.makedirs(os.path.join(HERE, "_build"), exist_ok=True)
    hdrs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hdrs.append(os.path.join(INCLUDE, "cgbdsm.h"))

    objs = []
    for f in ENGINE_CU:
        src = os.path.join(CSRC, f)
        obj = os.path.join(HERE, "_build", f + ".o")
        if force or _newer(obj, [src] + hdrs):
            cmd = [NVCC, "-ccbin", CXX, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
                   "-I", INCLUDE, "-I", CSRC, "-c", src, "-o", obj]
            if verbose_ptxas:
                cmd.insert(1, "-Xptxas=-v")
            _run(cmd)
        objs.append(obj)
    for f in ENGINE_CPP:
        src = os.path.join(CSRC, f)
        if not os.path.exists(src):
            continue
        obj = os.path.join(HERE, "_build", f + ".o")
        if force or _newer(obj, [src] + hdrs):
            _run([CXX, "-std=c++17", "-O3", "-fPIC", "-pthread", "-I", INCLUDE, "-I", CSRC,
                  "-I", "/usr/local/cuda/include", "-c", src, "-o", obj])
        objs.append(obj)
    lib = os.path.join(HERE, "libcgbdsm.so")
    if force or _newer(lib, objs):
        _run([NVCC, "-ccbin", CXX, *ARCH, "-shared", "-o", lib, *objs, "-Xcompiler", "-pthread",
              "-lcudart"])
    out["engine"] = lib

    cli_src = os.path.join(CSRC, "cli.cpp")
    if os.path.exists(cli_src):
        exe = os.path.join(HERE, "cgbdsm")
        if force or _newer(exe, [cli_src, lib] + hdrs):
            _run([CXX, "-std=c++17", "-O2", "-I", INCLUDE, "-I", CSRC, cli_src, "-o", exe,
                  "-L", HERE, "-lcgbdsm", "-Wl,-rpath,$ORIGIN", "-pthread"])
        out["cli"] = exe

    gen = os.path.join(HERE, "libcgbgen.so")
    gsrc = [os.path.join(CSRC, f) for f in GEN_CPP]
    if force or _newer(gen, gsrc):
        _run([CXX, "-std=c++17", "-O2", "-fPIC", "-shared", "-o", gen, *gsrc])
    out["gen"] = gen
    return out


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose_ptxas="--ptxas" in sys.argv)
