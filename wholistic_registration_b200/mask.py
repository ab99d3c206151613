"""Outlier masks of the per-batch registration (utils/mask.py) on the device.

``getMask`` and ``bwareafilt3_wei`` keep the reference's names and argument
meaning; volumes are (z, y, x) CUDA tensors here (the reference's (x, y, z)
arrays are the same memory, so its (3, 3, 1) footprint is a 3x3 square in
each z slice and 26-connectivity is unchanged).  Both run in the sm_100a
library (``wr_get_mask``, ``wr_bwareafilt3`` in ``include/wr_mask.h``).
"""

from __future__ import annotations

import ctypes

import torch

from . import _lib
from .registrar import _require_cuda, _stream_ptr, _vol

_ws_cache: dict = {}


def _workspace(shape, device):
    key = (str(device), tuple(int(s) for s in shape))
    ws = _ws_cache.get(key)
    if ws is None:
        lib = _lib.load()
        nbytes = ctypes.c_size_t(0)
        _lib.check("wr_mask_workspace_size", lib.wr_mask_workspace_size(*key[1], ctypes.byref(nbytes)))
        buf = torch.empty(int(nbytes.value) + 256, dtype=torch.uint8, device=device)
        ws = (buf, (buf.data_ptr() + 255) // 256 * 256, int(nbytes.value))
        _ws_cache.clear()          # one workspace: the wrapper calls these per frame with one shape
        _ws_cache[key] = ws
    return ws


def getMask(dat: torch.Tensor, thres_factor: float, percentile: float = 95.0, stats: torch.Tensor | None = None):
    """Boolean (z, y, x) mask: |(dat - mu) / sigma| > thres_factor with mu,
    sigma the mean / std of the values at or below the 95th percentile, then
    a (3, 3, 1) binary opening and dilation (utils/mask.py:59-111).
    ``stats`` (float64 CUDA tensor of 3) receives mu, sigma and the
    percentile value."""
    lib = _lib.load()
    v = _vol(dat, "dat")
    out = torch.empty(dat.shape, dtype=torch.uint8, device=dat.device)
    _, ws, nbytes = _workspace(dat.shape, dat.device)
    sp = None
    if stats is not None:
        _require_cuda(stats, "stats")
        if stats.dtype != torch.float64 or stats.numel() < 3:
            raise ValueError("stats must be a float64 CUDA tensor of at least 3 values")
        sp = stats.data_ptr()
    _lib.check("wr_get_mask", lib.wr_get_mask(ctypes.byref(v), float(thres_factor), float(percentile), out.data_ptr(),
                                              sp, ws, nbytes, _stream_ptr()))
    return out.view(torch.bool)


def bwareafilt3_wei(vol: torch.Tensor, size_range, n_components: torch.Tensor | None = None):
    """Boolean (z, y, x) mask keeping the 26-connected components of ``vol``
    (nonzero = set) whose voxel count lies in ``size_range`` (inclusive)
    (utils/mask.py:8-56).  ``n_components`` (int32 CUDA tensor) receives the
    number of components kept."""
    lib = _lib.load()
    _require_cuda(vol, "vol")
    if vol.dim() != 3:
        raise ValueError("vol must be a 3-D (z, y, x) volume")
    if vol.dtype == torch.bool:
        m = vol.view(torch.uint8)
    elif vol.dtype == torch.uint8:
        m = vol
    else:
        m = (vol != 0).to(torch.uint8)
    out = torch.empty(vol.shape, dtype=torch.uint8, device=vol.device)
    _, ws, nbytes = _workspace(vol.shape, vol.device)
    err = torch.zeros(1, dtype=torch.int32, device=vol.device)
    ncp = None
    if n_components is not None:
        _require_cuda(n_components, "n_components")
        if n_components.dtype != torch.int32:
            raise ValueError("n_components must be an int32 CUDA tensor")
        ncp = n_components.data_ptr()
    nz, ny, nx = (int(s) for s in vol.shape)
    _lib.check("wr_bwareafilt3", lib.wr_bwareafilt3(m.data_ptr(), nz, ny, nx, int(size_range[0]), int(size_range[1]),
                                                    out.data_ptr(), ncp, err.data_ptr(), ws, nbytes, _stream_ptr()))
    return out.view(torch.bool)
