"""Build recipe of the in-tree CUDA library ``libanalogsat_b200.so`` (sm_100a).

``python -m analogsat_b200.build`` compiles every source under ``csrc/`` with nvcc
into the package directory, where :mod:`analogsat_b200` loads it from.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libanalogsat_b200.so")

NVCC_FLAGS = [
    "-std=c++17", "-O3", "-lineinfo",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-shared", "-Xcompiler", "-fPIC",
]


def sources() -> list[str]:
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC)
                  if f.endswith((".cu", ".cpp")))


def headers() -> list[str]:
    inc = os.path.join(os.path.dirname(HERE), "include")
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs += [os.path.join(inc, f) for f in os.listdir(inc) if f.endswith(".h")]
    return hs


CLI_SRC = os.path.join(HERE, "frontend", "analogsat_cli.cpp")
CLI = os.path.join(HERE, "analogsat-b200")


def build_cli(force: bool = False) -> str:
    """The command-line frontend (run / speedtest / bench) linked against the library."""
    inc = os.path.join(os.path.dirname(HERE), "include")
    deps = [CLI_SRC, LIB, os.path.join(inc, "analogsat_b200.hpp"), os.path.join(inc, "analogsat_b200.h")]
    if not force and os.path.exists(CLI) and all(os.path.getmtime(f) <= os.path.getmtime(CLI) for f in deps):
        return CLI
    cxx = os.environ.get("CXX", "g++")
    subprocess.run([cxx, "-std=c++17", "-O2", "-I", inc, CLI_SRC, "-o", CLI + ".tmp", "-L", HERE,
                    "-lanalogsat_b200", "-Wl,-rpath,$ORIGIN"], check=True)
    os.replace(CLI + ".tmp", CLI)
    return CLI


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(f) <= t for f in sources() + headers())


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile the library (and the command-line frontend) if any source is newer than
    it; returns the library's path."""
    if not force and up_to_date():
        build_cli()
        return LIB
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc, *NVCC_FLAGS, "-o", LIB + ".tmp", *sources()]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    build_cli(force=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
