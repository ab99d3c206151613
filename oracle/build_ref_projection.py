"""Test infrastructure: build the reference's projection kernels as a shared
library for the fixture generator (tests/golden/make_projection_golden.py).

The reference keeps the CUDA C source of its two projection kernels as
string constants in src/wholistic_registration/utils/calFlowCrossResolution.py
(_PROJECT_TO_PLANES_NANMAX_SRC :480-569, _PROJECT_TO_PLANES_WEIGHTED_AVG_SRC
:571-660) and compiles them with CuPy's RawKernel, which is absent here.  This
recipe copies those strings unchanged into oracle/_ref/ref_projection_kernels.cu
(git-ignored, never committed) and compiles them with nvcc for sm_100a
together with oracle/ref_projection_launch.cu into
oracle/_ref/libref_projection.so.  Nothing outside the tests and the fixture
generator loads it.
"""

from __future__ import annotations

import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
LIB = os.path.join(OUT, "libref_projection.so")
SRC_REL = os.path.join("src", "wholistic_registration", "utils", "calFlowCrossResolution.py")
NAMES = ("_PROJECT_TO_PLANES_NANMAX_SRC", "_PROJECT_TO_PLANES_WEIGHTED_AVG_SRC")


def extract(ref_root: str) -> str:
    text = open(os.path.join(ref_root, SRC_REL)).read()
    parts = []
    for name in NAMES:
        m = re.search(name + r" = r'''(.*?)'''", text, re.S)
        if m is None:
            raise RuntimeError(f"{name} not found in {SRC_REL}")
        parts.append(m.group(1))
    return "\n".join(parts)


def build(ref_root: str | None = None) -> str | None:
    """Compile the library; None when the reference tree is absent.

    ref_root: the reference checkout (default: $WR_REFERENCE_ROOT)."""
    ref_root = ref_root or os.environ.get("WR_REFERENCE_ROOT")
    if not ref_root or not os.path.exists(os.path.join(ref_root, SRC_REL)):
        return None
    os.makedirs(OUT, exist_ok=True)
    with open(os.path.join(OUT, "ref_projection_kernels.cu"), "w") as fh:
        fh.write(extract(ref_root))
    nvcc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    cmd = [nvcc, "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-Xcompiler", "-fPIC",
           "-I", OUT, "-o", LIB, os.path.join(HERE, "ref_projection_launch.cu")]
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(sys.argv[1] if len(sys.argv) > 1 else None))
