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
    assert re.search(r"#define WR_MAX_BATCH 32", h)
    assert _lib.WR_LK_TILE_ORDER_X == 1 << 8 and _lib.WR_LK_CTAS_PER_SM(3) == 3 << 12 and _lib.MAX_BATCH == 32
