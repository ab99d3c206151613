"""Parity of the CUDA path with the reference at the benchmarked configuration.

The reference's own ``getMotion`` / ``correctMotion`` were run on four cases
with 33 x 33 patches (r = 16) and 10 iterations per level
(``tests/golden/bench_cases.py``): slabs of the config-0 and config-1
generators with the 70 % ellipsoid exclusion mask at 3 and 4 levels, the full
64 x 256 x 256 config-0 volume (3 levels, no exclusion) and an
8 x 1024 x 1024 config-1 slab (4 levels, masked).  The inputs are regenerated
from the seeded generator and must hash to the fixture's SHA-256.

Bars: the per-level iteration counts equal the reference's (the device's own
stopping decisions, no replay); on the fixture's strided subsample the motion
within 1e-3 voxel of the reference plus, per voxel, the method's own
single-precision sensitivity there (``bench_<name>_f32sens.npz``: how far the
oracle lands from the reference when its image arithmetic runs in float32,
``make_f32_oracle.py``; zero almost everywhere, up to 0.05 voxel in a few
nearly singular windows of the 8 x 1024 x 1024 slab), and everywhere within
0.1 voxel; the warped volume within 1e-4 relative L2 and the per-level error
log within 1e-4 relative.
"""

from __future__ import annotations

import os
import sys

import numpy as np
import pytest

from conftest import GOLDEN

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

sys.path.insert(0, GOLDEN)
from bench_cases import BENCH_CASES, bench_inputs, bench_option  # noqa: E402

FLOW_TOL = 1e-3     # voxel, max-abs
WARP_TOL = 1e-4     # relative L2
CASES = [n for n in BENCH_CASES if os.path.exists(os.path.join(GOLDEN, f"bench_{n}.npz"))]


@pytest.mark.parametrize("name", CASES)
def test_benchmarked_configuration_matches_reference(name):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from wholistic_registration_b200 import calFlow3d_Wei_v1 as cf3

    d = dict(np.load(os.path.join(GOLDEN, f"bench_{name}.npz")))
    tmpl, mov, excl, digest = bench_inputs(name)
    assert digest == str(d["sha256"]), f"{name}: regenerated inputs differ from the fixture's"
    layer = BENCH_CASES[name][4]
    option = bench_option(name, float(d["smooth_penalty"]))
    option["mask_ref"], option["mask_mov"] = excl.copy(), excl.copy()
    motion, err, _, log = cf3.getMotion(mov, tmpl, option)
    ref_counts = [len(d[f"layer_{l}/currentError"]) for l in range(layer + 1)]
    counts = [len(log[f"layer_{l}"]["currentError"]) for l in range(layer + 1)]
    assert counts == ref_counts, f"{name}: evaluations per level {counts}, reference {ref_counts}"
    s = int(d["stride"])
    diff = np.abs(motion[::s, ::s] - d["motion_sub"])
    sens = np.load(os.path.join(GOLDEN, f"bench_{name}_f32sens.npz"))["sens"]
    over = diff > FLOW_TOL + sens
    print(f"{name}: counts {counts}, max |dmotion| {diff.max():.3g} voxel, float32 sensitivity max {sens.max():.3g}, "
          f"{int((diff > FLOW_TOL).sum())} components above 1e-3")
    assert not over.any(), f"{name}: {int(over.sum())} components beyond 1e-3 + float32 sensitivity"
    assert diff.max() <= 0.1
    for l in range(layer + 1):
        np.testing.assert_allclose(log[f"layer_{l}"]["currentError"], d[f"layer_{l}/currentError"], rtol=1e-4,
                                   err_msg=f"{name} layer {l}")
    np.testing.assert_allclose(err, float(d["current_error"]), rtol=1e-4)
    warped = cf3.correctMotion(mov.astype(np.float32), motion)[::s, ::s].astype(np.float64)
    want = d["warped_sub"].astype(np.float64)
    rel = float(np.linalg.norm(warped - want) / np.linalg.norm(want))
    assert rel <= WARP_TOL, f"{name}: warp rel L2 {rel:.3g}"
