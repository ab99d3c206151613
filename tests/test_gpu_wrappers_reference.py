"""wbi_registration_3d / wbi_registration_2d against runs of the reference's
own wrappers (utils/registration.py:192-352 and :41-189).

``tests/golden/wrappers.npz`` holds, per case, the uint16 frames (and calcium
channel), the given template or initial motion when the case uses them, the
config the reference read (as TOML), and the reference's outputs: corrected
membrane and calcium frames, the template in (x, y, z), per-frame initial and
eventual errors and the motions.  Cases: automatic template picking, dual
channel with the sqrt and log2 transforms, a given template with an initial
motion, 3-D and 2-D.

Bars: motions within 1e-3 voxel max-abs, corrected frames within 1e-4
relative L2, the template and the initial errors within 1e-6 relative, the
eventual errors within 1e-4.
"""

from __future__ import annotations

import json
import os

import numpy as np
import pytest

from conftest import GOLDEN

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

CASES = ["w3d_auto", "w3d_dual_sqrt", "w3d_given_init", "w2d_auto", "w2d_dual_log2"]


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.parametrize("name", CASES)
def test_wrapper_matches_reference_run(name):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from wholistic_registration_b200.registration import wbi_registration_2d, wbi_registration_3d

    d = dict(np.load(os.path.join(GOLDEN, "wrappers.npz")))
    g = lambda k: d[f"{name}/{k}"]
    cfg = json.loads(str(g("config")))
    dual = cfg["channels"]["dual_channel"]
    given = not cfg["reference"]["pick_reference_auto"]
    fn = wbi_registration_3d if name.startswith("w3d") else wbi_registration_2d
    use_init = name.endswith("_init")
    mem_out, ca_out, dat_ref, errors, motion_out = fn(
        g("mem"), cfg, reference_image=g("ref") if given else None, motion_init=g("init") if use_init else None,
        verbose=False, moving_Ca_image=g("ca") if dual else None)
    np.testing.assert_allclose(np.asarray(dat_ref, np.float64), g("dat_ref").astype(np.float64), rtol=1e-6,
                               atol=1e-6)
    assert motion_out.shape == g("motion_out").shape
    dmax = float(np.abs(motion_out - g("motion_out")).max())
    assert dmax <= 1e-3, f"{name}: max |dmotion| {dmax:.3g}"
    assert rel_l2(mem_out, g("mem_out")) <= 1e-4
    if dual:
        assert rel_l2(ca_out, g("ca_out")) <= 1e-4
    np.testing.assert_allclose([e["initial_error"] for e in errors], g("initial_error"), rtol=1e-6)
    # the eventual error follows the motion (1e-3 voxel), so its bar is the warp's
    np.testing.assert_allclose([e["eventual_error"] for e in errors], g("eventual_error"), rtol=1e-4)
