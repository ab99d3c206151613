"""Build the sm_100a shared library in-tree.

    python -m wholistic_registration_b200.build

Compiles ``csrc/wr_api.cu`` (the registration path), ``csrc/wr_net.cu``
(the warm-start network) and ``csrc/wr_mask.cu`` (outlier masks) with nvcc
into ``wholistic_registration_b200/_wr_b200.so``.  The library exports only
the plain C ABI declared in ``include/wr_b200.h``, ``include/wr_net.h`` and
``include/wr_mask.h``; it links the CUDA runtime statically, so it needs
nothing from torch.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(HERE, "_wr_b200.so")
SOURCES = ["wr_api.cu", "wr_net.cu", "wr_mask.cu"]


def _deps() -> list[str]:
    """Every source and header the library is built from."""
    out = [os.path.join(SRC, f) for f in sorted(os.listdir(SRC)) if f.endswith((".cu", ".cuh", ".inc", ".h"))]
    return out + [os.path.join(INCLUDE, f) for f in sorted(os.listdir(INCLUDE)) if f.endswith(".h")]


def nvcc_path() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build wholistic_registration_b200")
    return cand


def command(out: str = LIB) -> list[str]:
    return [
        nvcc_path(), "-O3", "-std=c++17",
        "-gencode", "arch=compute_100a,code=sm_100a",
        "-lineinfo",
        "-Xcompiler", "-fPIC,-ffp-contract=off,-fvisibility=hidden",
        "-I", INCLUDE,
        "-shared", "-o", out,
    ] + [os.path.join(SRC, s) for s in SOURCES]


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(d) <= t for d in _deps())


def build(force: bool = False, verbose: bool = True) -> str:
    if not force and up_to_date():
        return LIB
    cmd = command()
    if verbose:
        print(" ".join(cmd), flush=True)
    tmp = LIB + ".tmp"
    cmd[cmd.index(LIB)] = tmp
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv)
