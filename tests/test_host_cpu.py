"""Host-side logic that needs no GPU: the autotuner's candidate set and
cache, and the batch registrar's argument checks before any launch."""

from __future__ import annotations

import json

import pytest

torch = pytest.importorskip("torch")


def test_autotune_candidates_and_cache_roundtrip(tmp_path, monkeypatch):
    from wholistic_registration_b200 import _lib, autotune

    c = autotune.candidates()
    assert len(c) == len(set(c)) == len(autotune.ORDERS) * len(autotune.CTAS_PER_SM)
    assert 0 in c and _lib.WR_LK_TILE_ORDER_X in c
    for f in c:
        assert (f >> _lib.WR_LK_CTAS_PER_SM_SHIFT) & 15 in autotune.CTAS_PER_SM
    monkeypatch.setenv("WR_B200_CACHE", str(tmp_path / "sub"))
    assert autotune.cache_path() == str(tmp_path / "sub" / "autotune.json")
    autotune._store({"k": {"flags": 256, "ms": {"0": 1.0}}})
    assert autotune._load() == {"k": {"flags": 256, "ms": {"0": 1.0}}}
    (tmp_path / "sub" / "autotune.json").write_text("not json")
    assert autotune._load() == {}


def test_flag_bits_match_header():
    import os
    import re

    from wholistic_registration_b200 import _lib

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    h = open(os.path.join(root, "include", "wr_b200.h")).read()
    assert re.search(r"WR_LK_TILE_ORDER_X = 1 << 8", h)
    assert re.search(r"WR_LK_CTAS_PER_SM_SHIFT = 12", h)
    assert re.search(r"#define WR_MAX_BATCH 64", h)
    assert _lib.WR_LK_TILE_ORDER_X == 1 << 8 and _lib.WR_LK_CTAS_PER_SM(3) == 3 << 12 and _lib.MAX_BATCH == 64


def test_wrapper_host_helpers(tmp_path):
    import numpy as np

    from wholistic_registration_b200.registration import _load_config, _mse, transform

    p = tmp_path / "c.toml"
    p.write_text('[mask]\nthresFactor = 5\nmaskRange = [5, 4000]\n')
    assert _load_config(p)["mask"]["maskRange"] == [5, 4000]
    assert _load_config({"a": 1}) == {"a": 1}
    a = torch.tensor([1, 5, 65535], dtype=torch.int32).to(torch.uint16)
    b = torch.tensor([3, 2, 0], dtype=torch.int32).to(torch.uint16)
    an, bn = a.to(torch.int32).numpy().astype(np.uint16), b.to(torch.int32).numpy().astype(np.uint16)
    assert _mse(a, b) == float(np.mean((an - bn) ** 2))
    x = torch.tensor([0.0, 9.0, 99.0], dtype=torch.float64)
    assert torch.allclose(transform(x, 2, "log10"), 2 * torch.log10(1 + x))
    with pytest.raises(ValueError):
        transform(x, 1, "cube")


def test_division_multiplier_bound():
    """The tile-index division of the iteration kernel: m = ceil(2^32 / d)
    and q = (n * m) >> 32 equal n // d whenever n * d <= 2^32 (the bound the
    host checks before handing the kernel a multiplier)."""
    import numpy as np

    rng = np.random.default_rng(7)
    for d in list(range(2, 300)) + [int(v) for v in rng.integers(300, 1 << 16, size=200)]:
        m = ((1 << 32) + d - 1) // d
        nmax = (1 << 32) // d
        ns = np.concatenate([np.arange(0, min(nmax, 5000)), rng.integers(0, nmax + 1, size=2000),
                             [nmax, nmax - 1, (nmax // d) * d, (nmax // d) * d - 1]])
        ns = ns[(ns >= 0) & (ns <= nmax)].astype(object)
        assert all((int(n) * m) >> 32 == int(n) // d for n in ns), d


def test_xres_wrong_region_options_validated():
    """wr_xres_workspace_size sizes the wrong-region correction's buffers
    (with global scratch for the per-slice detection once a slice has more
    control points than shared memory holds) and rejects an unknown exclusion
    mode or a quantile outside [0, 1].  Host-only: no GPU."""
    import ctypes

    from wholistic_registration_b200 import _lib
    from wholistic_registration_b200.registrar import LKParams

    lib = _lib.load()
    assert ctypes.sizeof(_lib.WrXresWrongRegion) == 36
    p = LKParams(layer=1, iter=6, r=3, zRatio=3.0, movRange=5.0, smoothPenalty=0.05, tol=1e-3).to_c()

    def size(wr, shape=(6, 48, 40), ref=(9, 48, 40)):
        n = ctypes.c_size_t(0)
        rc = lib.wr_xres_workspace_size(*shape, *ref, ctypes.byref(p), 2.0, 0, 0,
                                        None if wr is None else ctypes.byref(wr), ctypes.byref(n))
        return rc, n.value

    def wr(mode=0, q=0.8):
        return _lib.WrXresWrongRegion(1, 0, 3.0, 2, 2.0, 1.0, 2.0, mode, q)

    rc0, off = size(None)
    rc1, direct = size(wr())
    rc2, high = size(wr(1))
    assert rc0 == rc1 == rc2 == 0 and off < direct < high
    assert size(_lib.WrXresWrongRegion(0, 0, 3.0, 2, 2.0, 1.0, 2.0, 0, 0.8))[1] == off   # enable = 0: off
    assert size(wr(2))[0] == 3                       # WR_E_PARAM
    assert size(wr(1, 1.5))[0] == 3
    # 146 x 146 control points per slice: 0.5 MB of detection scratch per slice
    rc_big, big_off = size(None, (2, 1024, 1024), (2, 1024, 1024))
    rc_big2, big_on = size(wr(), (2, 1024, 1024), (2, 1024, 1024))
    assert rc_big == rc_big2 == 0 and big_on - big_off > 2 * (146 * 146 * 24)


def test_pick_initial_reference_needs_a_cuda_tensor():
    """The template picking's frame correlation runs in the library's kernel
    (wr_frame_gram); CPU tensors are refused, not computed on the host."""
    import numpy as np
    import pytest
    import torch

    from wholistic_registration_b200.registration import pick_initial_reference

    frames = torch.from_numpy(np.random.default_rng(0).uniform(0, 100, (4, 3, 16, 16)).astype(np.float32))
    with pytest.raises(ValueError, match="CUDA"):
        pick_initial_reference(frames, max_corr_frames=2)


def test_get_motion_v2_wrong_region_options(monkeypatch):
    """getMotion_v2 reads the wrong-region option keys as the reference does,
    before it touches a device: an unknown metric raises ValueError
    (utils/calFlowCrossResolution.py accepts "mse" / "mae"), and the exclusion
    mode is "highresidual" only for that exact string; every other value
    (None, "Direct", "lowresidual") takes the direct exclusion, as the
    reference's equality test at utils/calFlowCrossResolution.py:2340 does."""
    import numpy as np
    import pytest

    from wholistic_registration_b200 import _lib
    from wholistic_registration_b200 import calFlowCrossResolution as C

    mov = np.zeros((8, 8, 2), np.float32)
    ref = np.zeros((8, 8, 3), np.float32)
    base = {"mask_ref": 0, "mask_mov": 0, "layer": 0, "iter": 2, "r": 1, "zRatio": 2.0, "zRatio_HR": 1.0,
            "smoothPenalty": 0.05}
    with pytest.raises(ValueError, match="metric"):
        C.getMotion_v2(mov, ref, dict(base, wrong_region_metric="l2"))

    class Captured(Exception):
        pass

    seen = []

    def fake(*args):
        seen.append(args[7])   # exclusion mode: 0 direct, 1 high residual
        raise Captured

    monkeypatch.setattr(_lib, "WrXresWrongRegion", fake)
    for mode, want in (("highresidual", 1), ("direct", 0), ("Direct", 0), (None, 0), ("lowresidual", 0)):
        with pytest.raises(Captured):
            C.getMotion_v2(mov, ref, dict(base, wrong_region_exclude_mode=mode))
        assert seen[-1] == want, (mode, seen[-1])
