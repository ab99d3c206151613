"""Single-precision sensitivity of the benchmarked-configuration cases.

    python tests/golden/make_f32_oracle.py [case ...]

Runs the oracle (``oracle/lk_oracle.py``) on each case of ``bench_cases.py``
with its image arithmetic in float32 (``image_dtype=np.float32``) and stores,
on the fixture's strided subsample, how far that float32 run lands from the
reference's float64 run (``bench_<name>.npz``):
``bench_<name>_f32sens.npz`` with ``sens`` = |motion_f32 - motion_ref|
per voxel and component.  Where the method amplifies single-precision
rounding (windows whose structure tensor is nearly singular), any float32
implementation moves by about this much; the GPU parity test allows it on
top of its 1e-3 voxel bar.
"""

from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, HERE)

from bench_cases import BENCH_CASES, bench_inputs, bench_option  # noqa: E402
from oracle import lk_oracle as O  # noqa: E402


def make(name):
    d = dict(np.load(os.path.join(HERE, f"bench_{name}.npz")))
    tmpl, mov, excl, digest = bench_inputs(name)
    assert digest == str(d["sha256"]), name
    option = bench_option(name, float(d["smooth_penalty"]))
    option["mask_ref"], option["mask_mov"] = excl.copy(), excl.copy()
    motion, _, _, _ = O.get_motion(mov, tmpl, option, image_dtype=np.float32)
    s = int(d["stride"])
    sens = np.abs(motion[::s, ::s] - d["motion_sub"]).astype(np.float32)
    np.savez_compressed(os.path.join(HERE, f"bench_{name}_f32sens.npz"), sens=sens)
    print(f"{name}: float32 sensitivity max {sens.max():.3g}, voxels above 1e-3: {(sens.max(-1) > 1e-3).sum()}")


if __name__ == "__main__":
    for n in sys.argv[1:] or list(BENCH_CASES):
        make(n)
