"""C-ABI checks that need no GPU: the library loads, exports every symbol of
include/wr_b200.h, computes the resize tables bit-exactly, plans workspaces
and rejects bad arguments before touching the device."""

from __future__ import annotations

import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT
from oracle import lk_oracle as O
from wholistic_registration_b200 import _lib


@pytest.fixture(scope="module")
def lib():
    return _lib.load()


def test_exports_match_header(lib):
    import glob

    header = ""
    for h in sorted(glob.glob(os.path.join(ROOT, "include", "*.h"))):
        with open(h) as fh:
            header += fh.read()
    declared = set(re.findall(r"WR_API\s+[\w\s\*]*?\b(wr_\w+)\s*\(", header))
    assert declared == set(_lib.EXPORTS)
    for name in declared:
        assert hasattr(lib, name)
    assert lib.wr_abi_version() == 1


def test_struct_layout_matches_header(tmp_path):
    """sizeof / offsetof of the C structs (compiled from the header) equal ctypes'."""
    import shutil
    import subprocess

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    fields = {
        "WrVolume": ["data", "dtype", "nz", "ny", "nx"],
        "WrLKParams": ["layer", "iter", "r", "zRatio", "movRange", "smoothPenalty", "tol", "precision",
                       "forced_updates"],
        "WrLKStats": ["levels", "evals", "updates", "nan_solves", "current_error", "diff_error", "penalty_error",
                      "max_diff_motion"],
        "WrLKItem": ["mov", "ref", "excl_mask_mov", "excl_mask_ref", "motion_init", "motion_out", "warped_out",
                     "stats"],
        "WrProfile": ["acc_begin", "acc_end", "capacity", "recorded", "launches"],
        "WrConvGeom": ["n", "oz", "iz", "stride", "c1", "c2", "up1", "cout", "act"],
    }
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "wr_b200.h"', '#include "wr_net.h"',
             'int main(void){']
    for st, fs in fields.items():
        lines.append(f'printf("{st} %zu\\n", sizeof({st}));')
        for f in fs:
            lines.append(f'printf("{st}.{f} %zu\\n", offsetof({st}, {f}));')
    lines.append("return 0;}")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = dict(l.split() for l in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines())
    for st, fs in fields.items():
        cls = getattr(_lib, st)
        assert int(out[st]) == ctypes.sizeof(cls), st
        for f in fs:
            assert int(out[f"{st}.{f}"]) == getattr(cls, f).offset, f"{st}.{f}"


def _c_table(lib, n_in, n_out, method):
    taps = ctypes.c_int32(0)
    _lib.check("wr_resize_table", lib.wr_resize_table(n_in, n_out, method, None, None, ctypes.byref(taps)))
    w = np.zeros((n_out, taps.value), np.float64)
    i = np.zeros((n_out, taps.value), np.int32)
    _lib.check("wr_resize_table", lib.wr_resize_table(n_in, n_out, method, w.ctypes.data, i.ctypes.data,
                                                      ctypes.byref(taps)))
    return w, i


@pytest.mark.parametrize("n_in,n_out", [(256, 128), (256, 64), (1024, 128), (1000, 125), (66, 33), (70, 17),
                                        (33, 16), (37, 18), (5, 5), (12, 25), (128, 256), (125, 250)])
@pytest.mark.parametrize("method", [0, 1])
def test_resize_table_bit_exact(lib, n_in, n_out, method):
    kernel = O.cubic if method == 0 else O.triangle
    w, i = _c_table(lib, n_in, n_out, method)
    scale = n_out / n_in
    # oracle before zero-column removal
    import math

    if scale < 1:
        h = lambda t: scale * kernel(scale * t)
        width = 4.0 / scale
    else:
        h = kernel
        width = 4.0
    k = np.arange(1, n_out + 1, dtype=np.float64)
    u = k / scale + 0.5 * (1 - 1 / scale)
    left = np.floor(u - width / 2)
    P = int(math.ceil(width)) + 2
    ind = (left[:, None] + np.arange(P) - 1).astype(np.int32)
    ww = h(u[:, None] - ind - 1)
    ww = ww / np.sum(ww, axis=1)[:, None]
    aux = np.concatenate((np.arange(n_in), np.arange(n_in - 1, -1, -1))).astype(np.int32)
    ind = aux[np.mod(ind, aux.size)]
    assert w.shape == ww.shape
    np.testing.assert_array_equal(w, ww)
    np.testing.assert_array_equal(i, ind)
    # and the compacted form equals the oracle's contributions()
    w2, i2 = O.contributions(n_in, n_out, scale, kernel)
    keep = np.any(ww != 0, axis=0)
    np.testing.assert_array_equal(w[:, keep], w2)
    np.testing.assert_array_equal(i[:, keep], i2)


def _params(**kw):
    p = _lib.WrLKParams()
    p.layer, p.iter, p.r = kw.get("layer", 2), kw.get("iter", 10), kw.get("r", 16)
    p.zRatio, p.movRange = kw.get("zRatio", 1.0), kw.get("movRange", 5.0)
    p.smoothPenalty, p.tol = kw.get("smoothPenalty", 1.0), kw.get("tol", 1e-3)
    p.precision = kw.get("precision", 0)
    for i in range(_lib.MAX_LEVELS):
        p.forced_updates[i] = -1
    return p


def test_workspace_size_scales_with_volume(lib):
    sz = ctypes.c_size_t(0)
    _lib.check("ws", lib.wr_lk_workspace_size(64, 256, 256, ctypes.byref(_params()), ctypes.byref(sz)))
    small = sz.value
    _lib.check("ws", lib.wr_lk_workspace_size(128, 1024, 1024, ctypes.byref(_params(layer=3)), ctypes.byref(sz)))
    big = sz.value
    n0 = 64 * 256 * 256
    assert 20 * n0 < small < 80 * n0
    assert big > 30 * small


@pytest.mark.parametrize("kw,code", [
    (dict(layer=8), 3), (dict(layer=-1), 3), (dict(iter=0), 3), (dict(iter=65), 3), (dict(r=0), 3),
    (dict(r=49), 3), (dict(zRatio=0.0), 3), (dict(movRange=-1.0), 3), (dict(precision=7), 3),
])
def test_workspace_size_rejects_bad_params(lib, kw, code):
    sz = ctypes.c_size_t(0)
    rc = lib.wr_lk_workspace_size(16, 64, 64, ctypes.byref(_params(**kw)), ctypes.byref(sz))
    assert rc == code
    assert lib.wr_last_error()


def test_no_control_point_level_is_rejected(lib):
    # 24 voxels, r=5, 3 levels: level 2 is 6 wide and holds no control point
    sz = ctypes.c_size_t(0)
    rc = lib.wr_lk_workspace_size(4, 24, 24, ctypes.byref(_params(layer=2, r=5)), ctypes.byref(sz))
    assert rc == 6


def test_register_argument_errors_without_gpu(lib):
    p = _params(layer=1, r=2)
    vol = _lib.volume(0, _lib.WR_U16, (4, 32, 32))
    ok = _lib.volume(16, _lib.WR_U16, (4, 32, 32))
    bad_shape = _lib.volume(16, _lib.WR_U16, (4, 32, 31))
    bad_dtype = _lib.volume(16, 9, (4, 32, 32))
    out = 256
    assert lib.wr_lk_register(ctypes.byref(vol), ctypes.byref(ok), None, None, ctypes.byref(p), None, out, None,
                              256, 1 << 30, None) == 1
    assert lib.wr_lk_register(ctypes.byref(ok), ctypes.byref(bad_shape), None, None, ctypes.byref(p), None, out,
                              None, 256, 1 << 30, None) == 2
    assert lib.wr_lk_register(ctypes.byref(ok), ctypes.byref(bad_dtype), None, None, ctypes.byref(p), None, out,
                              None, 256, 1 << 30, None) == 4
    assert lib.wr_lk_register(ctypes.byref(ok), ctypes.byref(ok), None, None, ctypes.byref(p), None, out, None,
                              256, 16, None) == 5
    assert lib.wr_lk_register(ctypes.byref(ok), ctypes.byref(ok), None, None, ctypes.byref(p), None, out, None,
                              260, 1 << 30, None) == 5
    with pytest.raises(ValueError):
        _lib.check("wr_lk_register", 2)
