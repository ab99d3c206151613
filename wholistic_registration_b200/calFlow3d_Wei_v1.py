"""Drop-in replacement for the reference's ``utils/calFlow3d_Wei_v1.py`` entry points.

``getMotion(dat_mov, dat_ref, option, verbose=False)`` and
``correctMotion(data_raw, motion_field)`` keep the reference's signatures,
argument meaning, array layout and return values
(utils/calFlow3d_Wei_v1.py:295-706):

* volumes are indexed (x, y, z) like the reference (the callers'
  (z, y, x) arrays transposed by (2, 1, 0)); motion fields are (x, y, z, 3)
  float32 with component c displacing axis c;
* NumPy inputs give NumPy outputs; CUDA torch tensors (same layout) give CUDA
  tensors and stay on the device;
* ``option`` carries mask_ref, mask_mov (exclusion masks, True = excluded, or
  the default scalar 0 = none), layer, iter, r, zRatio, movRange, motion,
  smoothPenalty and tol.  Two optional keys extend it: ``forced_updates``
  (layer -> number of motion updates, replaying another run's iteration
  counts) and ``precision``.

Every computation runs on the GPU through the sm_100a library; the call
raises if the library or a CUDA device is missing.

Differences from the reference, all without effect on the motion field:
``option["mask_ref"]``/``["mask_mov"]`` are not rewritten into float32
arrays; ``error_log`` holds the per-level error and max-update lists but not
the per-iteration volume snapshots; ``coords_new`` is computed only when it is
converted to an array.
"""

from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .registrar import LKParams, LKRegistrar, stats_to_log, warp

__all__ = ["getMotion", "correctMotion"]

_cache: dict = {}


def _registrar(shape_zyx, params: LKParams, device) -> LKRegistrar:
    key = (shape_zyx, params.layer, params.iter, params.r, params.zRatio, params.movRange, params.smoothPenalty,
           params.tol, params.precision, tuple(sorted(params.forced_updates.items())), str(device))
    reg = _cache.get(key)
    if reg is None:
        if len(_cache) > 4:
            _cache.clear()
        reg = LKRegistrar(shape_zyx, params, device)
        _cache[key] = reg
    return reg


def _device_volume(a, device) -> torch.Tensor:
    """(x, y, z) array -> contiguous (z, y, x) CUDA tensor of a supported dtype."""
    if isinstance(a, torch.Tensor):
        t = a.to(device)
    else:
        a = np.asarray(a)
        if a.dtype not in (np.uint16, np.uint8, np.float32):
            a = a.astype(np.float32)
        t = torch.from_numpy(np.ascontiguousarray(a.transpose(2, 1, 0))).to(device, non_blocking=False)
        return t
    if t.dtype not in (torch.uint16, torch.uint8, torch.float32):
        t = t.to(torch.float32)
    return t.permute(2, 1, 0).contiguous()


def _device_mask(m, shape_xyz, device):
    if m is None or np.isscalar(m) or (hasattr(m, "ndim") and m.ndim == 0):
        if m is not None and bool(np.asarray(m)):
            raise ValueError("a scalar exclusion mask must be 0/False")
        return None
    if isinstance(m, torch.Tensor):
        t = (m.to(device) != 0).permute(2, 1, 0).contiguous()
    else:
        a = np.asarray(m)
        if tuple(a.shape) != tuple(shape_xyz):
            raise ValueError(f"mask shape {a.shape} does not match the volume {tuple(shape_xyz)}")
        t = torch.from_numpy(np.ascontiguousarray((a != 0).transpose(2, 1, 0))).to(device)
    if not bool(t.any()):
        return None
    return t.view(torch.uint8)


def _device_motion(m, shape_xyz, device):
    if m is None:
        return None
    if isinstance(m, torch.Tensor):
        t = m.to(device=device, dtype=torch.float32)
    else:
        t = torch.from_numpy(np.asarray(m, dtype=np.float32)).to(device)
    if tuple(t.shape) != tuple(shape_xyz) + (3,):
        raise ValueError("option['motion'] must be (x, y, z, 3)")
    return t.permute(2, 1, 0, 3).contiguous()


class _LazyCoords:
    """``coords_new`` of getMotion (motion + index grid), built on demand."""

    def __init__(self, motion_xyz3):
        self._m = motion_xyz3
        self._arr = None

    def _build(self):
        if self._arr is None:
            m = self._m
            if isinstance(m, torch.Tensor):
                grid = torch.meshgrid(*[torch.arange(n, dtype=torch.float32, device=m.device) for n in m.shape[:3]],
                                      indexing="ij")
                self._arr = m + torch.stack(grid, dim=-1)
            else:
                grid = np.meshgrid(*[np.arange(n, dtype=np.float32) for n in m.shape[:3]], indexing="ij")
                self._arr = m + np.stack(grid, axis=-1)
        return self._arr

    def __array__(self, dtype=None, copy=None):
        a = self._build()
        a = a.cpu().numpy() if isinstance(a, torch.Tensor) else a
        return a if dtype is None else a.astype(dtype)

    def __getattr__(self, name):
        return getattr(self._build(), name)

    def __getitem__(self, idx):
        return self._build()[idx]


def _snapshot_buffers(shape_zyx, params, save_ite, device):
    """Device buffers for getMotion's error_log snapshots: per level, one slot
    per iteration index that is a multiple of save_ite."""
    if save_ite < 1:
        raise ValueError("option['save_ite'] must be >= 1")
    z, y, x = shape_zyx
    cap = -(-params.iter // save_ite)
    snap = _lib.WrSnapshots()
    snap.save_ite, snap.capacity = save_ite, cap
    bufs = {}
    for l in range(params.layer + 1):
        yl, xl = int(y / 2 ** l), int(x / 2 ** l)
        b = {"motion": torch.empty((cap, z, yl, xl, 3), dtype=torch.float32, device=device),
             "warped": torch.empty((cap, z, yl, xl), dtype=torch.float32, device=device),
             "ref": torch.empty((z, yl, xl), dtype=torch.float32, device=device),
             "mov": torch.empty((z, yl, xl), dtype=torch.float32, device=device)}
        snap.motion[l], snap.warped[l] = b["motion"].data_ptr(), b["warped"].data_ptr()
        snap.level_ref[l], snap.level_mov[l] = b["ref"].data_ptr(), b["mov"].data_ptr()
        bufs[l] = b
    return snap, bufs


def _fill_snapshots(log, st, snaps, save_ite, on_device):
    """The reference's error_log snapshot entries (utils/calFlow3d_Wei_v1.py:
    329-353, 451-470) in its (x, y, z[, 3]) layout."""
    _, bufs = snaps
    xyz = (lambda t: t.permute(2, 1, 0)) if on_device else (lambda t: t.cpu().numpy().transpose(2, 1, 0))
    xyz3 = (lambda t: t.permute(2, 1, 0, 3)) if on_device else (lambda t: t.cpu().numpy().transpose(2, 1, 0, 3))
    for l, b in bufs.items():
        n = min(-(-int(st.evals[l]) // save_ite), b["motion"].shape[0])
        entry = log[f"layer_{l}"]
        entry["motion_current"] = [xyz3(b["motion"][k]) for k in range(n)]
        entry["data_mov_corrected"] = [xyz(b["warped"][k]) for k in range(n)]
        entry["data_ref"] = xyz(b["ref"])
        entry["data_mov"] = xyz(b["mov"])


def getMotion(dat_mov, dat_ref, option, verbose=False):
    """Pyramid patch-wise Lucas-Kanade registration of ``dat_mov`` onto ``dat_ref``.

    Same contract as utils/calFlow3d_Wei_v1.py:295-673; returns
    ``(motion (x,y,z,3) float32, currentError, coords_new, error_log)``.
    ``error_log`` holds the per-level error and motion-change lists; with
    ``option["keep_snapshots"] = True`` it also holds the reference's
    snapshots — "motion_current" and "data_mov_corrected" at every iteration
    that is a multiple of ``option["save_ite"]`` (taken before that
    iteration's update) and the level images "data_ref" / "data_mov", all
    float32 — which cost a device-to-host copy of about three times the
    volume's float32 motion per level, so they are opt-in.
    """
    on_device = isinstance(dat_mov, torch.Tensor) and dat_mov.is_cuda
    device = dat_mov.device if on_device else torch.device("cuda", torch.cuda.current_device())
    shape_xyz = tuple(int(s) for s in dat_mov.shape)
    if len(shape_xyz) != 3 or tuple(dat_ref.shape) != shape_xyz:
        raise ValueError("dat_mov and dat_ref must be 3-D arrays of the same shape")
    params = LKParams.from_option(option)
    mov = _device_volume(dat_mov, device)
    ref = _device_volume(dat_ref, device)
    if mov.dtype != ref.dtype:
        mov, ref = mov.to(torch.float32), ref.to(torch.float32)
    mask_mov = _device_mask(option.get("mask_mov"), shape_xyz, device)
    mask_ref = _device_mask(option.get("mask_ref"), shape_xyz, device)
    init = _device_motion(option.get("motion"), shape_xyz, device)
    reg = _registrar(tuple(mov.shape), params, device)
    snaps = _snapshot_buffers(tuple(mov.shape), params, int(option.get("save_ite", 100)), device) \
        if option.get("keep_snapshots") else None
    motion = reg.register(mov, ref, mask_mov, mask_ref, init, snapshots=snaps[0] if snaps else None)
    log, current_error = stats_to_log(reg.stats(), params.layer + 1)
    if snaps:
        _fill_snapshots(log, reg.stats(), snaps, int(option.get("save_ite", 100)), on_device)
    if verbose:
        for k, v in log.items():
            for i, e in enumerate(v["currentError"]):
                print(f"Downsample {k}\tIter: {i}\tError: {e:.3f}")
    motion_xyz = motion.permute(2, 1, 0, 3)
    if not on_device:
        motion_xyz = motion.cpu().numpy().transpose(2, 1, 0, 3)
    return motion_xyz, current_error, _LazyCoords(motion_xyz), log


def correctMotion(data_raw, motion_field):
    """Pull-warp ``data_raw`` (x,y,z) through ``motion_field`` (x,y,z,3):
    float32 result (utils/calFlow3d_Wei_v1.py:676-706)."""
    on_device = isinstance(data_raw, torch.Tensor) and data_raw.is_cuda
    device = data_raw.device if on_device else torch.device("cuda", torch.cuda.current_device())
    shape_xyz = tuple(int(s) for s in data_raw.shape)
    src = _device_volume(data_raw, device)
    mot = _device_motion(motion_field, shape_xyz, device)
    out = warp(src, mot)
    if on_device:
        return out.permute(2, 1, 0)
    return out.cpu().numpy().transpose(2, 1, 0)
