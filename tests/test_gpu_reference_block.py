"""The reference builder on the device against the reference's own run."""

from __future__ import annotations

import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def test_compute_reference_from_block_matches_reference():
    """compute_reference_from_block (utils/reference.py:102-124) against the
    reference's own function run on the same block (fixture from
    tests/golden/make_golden.py): the same frames picked, in order, and the
    same reference volume (the frame correlation from the library's float64
    Gram kernel, float64 means; float32 means for float32 frames) for a
    single channel, dual channel with sqrt and log2 transforms, and k = 0."""
    import os

    import numpy as np

    from wholistic_registration_b200.registration import compute_reference_from_block

    d = dict(np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_block.npz")))
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    mem, ca = torch.from_numpy(d["mem"]).cuda(), torch.from_numpy(d["ca"]).cuda()
    for name in ("single", "dual_sqrt", "dual_log2", "dual_k0"):
        dual, k = d[f"{name}_params"]
        config = {"channels": {"k": float(k), "function": str(d[f"{name}_function"]), "dual_channel": bool(dual)}}
        ref, idx = compute_reference_from_block(mem, config, ca if dual else None)
        np.testing.assert_array_equal(idx, d[f"{name}_idx"], err_msg=name)
        np.testing.assert_allclose(ref, d[f"{name}_ref"], rtol=1e-12, atol=1e-9, err_msg=name)
    # float32 frames: the reference's mean (and its transform) stays float32
    mem32, ca32 = torch.from_numpy(d["mem_f32"]).cuda(), torch.from_numpy(d["ca_f32"]).cuda()
    for name in ("single", "dual_sqrt", "dual_log2", "dual_k0"):
        dual, k = d[f"{name}_params"]
        config = {"channels": {"k": float(k), "function": str(d[f"{name}_function"]), "dual_channel": bool(dual)}}
        ref, idx = compute_reference_from_block(mem32, config, ca32 if dual else None)
        want = d[f"f32_{name}_ref"]
        assert ref.dtype == want.dtype == np.float32, (name, ref.dtype)
        np.testing.assert_array_equal(idx, d[f"f32_{name}_idx"], err_msg=name)
        # float32 sums in the same order; log2 / sqrt within a few float32 ulps
        np.testing.assert_allclose(ref, want, rtol=1e-6, atol=0, err_msg=name)
