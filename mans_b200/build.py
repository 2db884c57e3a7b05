"""Build libmans_b200.so in-tree with nvcc for sm_100a.

Run as ``python -m mans_b200.build`` (or through ``__graft_entry__.build()``).
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libmans_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-shared",
         "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]


def sources() -> list[str]:
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))


def deps() -> list[str]:
    return sources() + glob.glob(os.path.join(HERE, "csrc", "*.cuh")) + \
        glob.glob(os.path.join(HERE, "csrc", "*.h")) + glob.glob(os.path.join(ROOT, "include", "*.h"))


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(d) <= t for d in deps())


CLI = os.path.join(HERE, "mans_cli")
CLI_SRC = os.path.join(HERE, "cli", "mans_cli.cu")


def build_cli(force: bool = False) -> str:
    """The command-line driver, linked against the library (found next to it)."""
    if not force and os.path.exists(CLI) and os.path.getmtime(CLI) >= max(
            os.path.getmtime(CLI_SRC), os.path.getmtime(LIB)):
        return CLI
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc, *ARCH, "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), "-o", CLI,
           CLI_SRC, "-L", HERE, "-lmans_b200", "-Xlinker", "-rpath,$ORIGIN"]
    subprocess.run(cmd, check=True)
    return CLI


def build(force: bool = False, verbose: bool = False) -> str:
    if force or not up_to_date():
        nvcc = os.environ.get("NVCC", "nvcc")
        cmd = [nvcc, *ARCH, *FLAGS, "-I", os.path.join(ROOT, "include"), "-o", LIB, *sources()]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    build_cli(force)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
