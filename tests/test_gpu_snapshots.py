"""getMotion's error_log snapshots against a run of the reference with
save_ite = 2 (``tests/golden/snapshots.npz``): per level the dense motion
("motion_current") and the warped moving level ("data_mov_corrected") at
iterations 0, 2, 4 (before each iteration's update), and the level images
("data_ref", "data_mov").  Opt-in through option["keep_snapshots"].

Bars: the same update counts; motions within 1e-3 voxel; warped levels and
level images within 1e-4 relative L2 (the library's levels are float32, the
reference's float64).
"""

from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import GOLDEN

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_error_log_snapshots_match_reference():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from wholistic_registration_b200 import calFlow3d_Wei_v1 as cf3

    d = dict(np.load(os.path.join(GOLDEN, "snapshots.npz")))
    option = {"mask_ref": d["excl"].copy(), "mask_mov": d["excl"].copy(), "layer": 1, "iter": 6, "r": 3,
              "zRatio": 1.0, "movRange": 5.0, "motion": None, "smoothPenalty": float(d["smooth_penalty"]),
              "tol": 1e-3, "save_ite": 2, "keep_snapshots": True}
    motion, _, _, log = cf3.getMotion(d["mov"], d["ref"], option)
    assert float(np.abs(motion - d["motion"]).max()) <= 1e-3
    for l in (1, 0):
        key = f"layer_{l}"
        entry = log[key]
        assert len(entry["currentError"]) == len(d[f"{key}/currentError"])
        ref_m, ref_w = d[f"{key}/motion_current"], d[f"{key}/data_mov_corrected"]
        assert len(entry["motion_current"]) == len(ref_m) == len(entry["data_mov_corrected"])
        for k in range(len(ref_m)):
            assert entry["motion_current"][k].shape == ref_m[k].shape
            assert float(np.abs(entry["motion_current"][k] - ref_m[k]).max()) <= 1e-3, (key, k)
            assert _rel(entry["data_mov_corrected"][k], ref_w[k]) <= 1e-4, (key, k)
        assert _rel(entry["data_ref"], d[f"{key}/data_ref"]) <= 1e-4
        assert _rel(entry["data_mov"], d[f"{key}/data_mov"]) <= 1e-4
    # without the option the snapshot lists stay empty
    option["keep_snapshots"] = False
    _, _, _, log2 = cf3.getMotion(d["mov"], d["ref"], option)
    assert log2["layer_0"]["motion_current"] == []
