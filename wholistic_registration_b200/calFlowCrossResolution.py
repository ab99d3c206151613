"""Drop-in replacement for the reference's cross-resolution entry point.

``getMotion_v2(data_mov, data_ref, option, verbose=False)`` keeps the
signature, option keys, array layout and return values of
``utils/calFlowCrossResolution.py:2470-2663``: the moving stack (x, y, z) and a
reference stack (x_hr, y_hr, z_hr) sampled with another z spacing
(``zRatio`` / ``zRatio_HR``: physical units per z index), registered by the
pyramid patch-wise Lucas-Kanade scheme with the reference read through its
cubic B-spline at the phase (x, y, z zRatio / zRatio_HR) + motion.  It
returns ``(phase_new, motion_current, data_ref_sampled)``: two (x, y, z, 3)
float32 fields and the reference sampled at the phase (float64, as the
reference returns it).

Every computation runs on the GPU through the sm_100a library
(``wr_xres_register``); the call raises if the library or a CUDA device is
missing.  NumPy inputs give NumPy outputs; CUDA torch tensors in the same
(x, y, z) layout give CUDA tensors.

The module also carries the continuous reference ``H``
(``generate_continuous_H_gpu`` / ``apply_H_to_matrix_gpu``, :463-478,
1144-1154) and the two fixed-plane projections of mapped samples
(``project_coords_to_fixed_planes_gpu``, max splat, :480-569 + 878-1141;
``project_coords_to_fixed_planes_weighted_gpu``, weighted bilinear splat,
:571-660 + 700-876) with the reference's signatures; they return CUDA torch
tensors where the reference returns CuPy arrays.

The wrong-region correction the reference runs by default
(``wrong_region_enable=True``: bad-region detection on the CP errors, a trap
mask in reference space and two re-runs, :2240-2467) runs on the device too,
in both exclusion modes ("direct" and "highresidual").  One optional key extends the options:
``forced_updates`` (layer -> number of motion updates, replaying another
run's iteration counts).
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .registrar import LKParams, _stream_ptr, stats_to_log

__all__ = ["getMotion_v2", "XresRegistrar", "generate_continuous_H_gpu", "apply_H_to_matrix_gpu",
           "project_coords_to_fixed_planes_gpu", "project_coords_to_fixed_planes_weighted_gpu"]


class XresRegistrar:
    """Cross-resolution registration of a (z, y, x) moving stack onto a
    (zh, yh, xh) reference stack on one GPU (``wr_xres_register``)."""

    def __init__(self, shape_zyx, ref_shape_zyx, params: LKParams, zRatio_HR: float, has_mask_ref: bool = True,
                 device=None, has_phase_init: bool = False, wrong_region=None):
        self.lib = _lib.load()
        self.shape = tuple(int(s) for s in shape_zyx)
        self.ref_shape = tuple(int(s) for s in ref_shape_zyx)
        self.params = params
        self.zRatio_HR = float(zRatio_HR)
        self.has_mask_ref = bool(has_mask_ref)
        self.has_phase_init = bool(has_phase_init)
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self._cp = params.to_c()
        # the wrong-region correction's options (None: off), a WrXresWrongRegion
        self._wr = wrong_region
        nbytes = ctypes.c_size_t(0)
        _lib.check("wr_xres_workspace_size",
                   self.lib.wr_xres_workspace_size(*self.shape, *self.ref_shape, ctypes.byref(self._cp),
                                                   self.zRatio_HR, int(self.has_mask_ref), int(self.has_phase_init),
                                                   self._wr_ptr(), ctypes.byref(nbytes)))
        self.workspace_bytes = int(nbytes.value)
        self.workspace = torch.empty(self.workspace_bytes + 256, dtype=torch.uint8, device=self.device)
        self._ws_ptr = (self.workspace.data_ptr() + 255) // 256 * 256
        self.stats_dev = torch.zeros(ctypes.sizeof(_lib.WrLKStats), dtype=torch.uint8, device=self.device)

    def _wr_ptr(self):
        return ctypes.byref(self._wr) if self._wr is not None else None

    @staticmethod
    def _check(t, name, shape, dtypes):
        if t is None:
            return None
        if not isinstance(t, torch.Tensor) or not t.is_cuda or not t.is_contiguous():
            raise ValueError(f"{name} must be a contiguous CUDA tensor")
        if tuple(t.shape) != tuple(shape) or t.dtype not in dtypes:
            raise ValueError(f"{name} must be {tuple(shape)} of {dtypes}")
        return t.data_ptr()

    def register(self, mov, ref, mask_mov=None, mask_ref=None, motion_init=None, phase_out=None, motion_out=None,
                 sampled_out=None, stream=None, phase_init=None):
        """(phase, motion, sampled) as (z, y, x, 3), (z, y, x, 3), (z, y, x) float32 tensors."""
        if mask_ref is not None and not self.has_mask_ref:
            raise ValueError("this registrar was built without room for a reference mask")
        if phase_init is not None and not self.has_phase_init:
            raise ValueError("this registrar was built without room for an initial phase")
        pm = self._check(mov, "mov", self.shape, (torch.float32,))
        pr = self._check(ref, "ref", self.ref_shape, (torch.float32,))
        if mask_mov is not None and mask_mov.dtype == torch.bool:
            mask_mov = mask_mov.view(torch.uint8)
        if mask_ref is not None and mask_ref.dtype == torch.bool:
            mask_ref = mask_ref.view(torch.uint8)
        pmm = self._check(mask_mov, "mask_mov", self.shape, (torch.uint8,))
        pmr = self._check(mask_ref, "mask_ref", self.ref_shape, (torch.uint8,))
        pin = self._check(motion_init, "motion_init", self.shape + (3,), (torch.float32,))
        pph = self._check(phase_init, "phase_init", self.shape + (3,), (torch.float32,))
        new = lambda shp: torch.empty(shp, dtype=torch.float32, device=self.device)  # noqa: E731
        phase_out = new(self.shape + (3,)) if phase_out is None else phase_out
        motion_out = new(self.shape + (3,)) if motion_out is None else motion_out
        sampled_out = new(self.shape) if sampled_out is None else sampled_out
        for t, name, shp in ((phase_out, "phase_out", self.shape + (3,)), (motion_out, "motion_out", self.shape + (3,)),
                             (sampled_out, "sampled_out", self.shape)):
            self._check(t, name, shp, (torch.float32,))
        _lib.check("wr_xres_register",
                   self.lib.wr_xres_register(pm, *self.shape, pr, *self.ref_shape, pmm, pmr, pin, pph,
                                             ctypes.byref(self._cp), self.zRatio_HR, self._wr_ptr(),
                                             phase_out.data_ptr(),
                                             motion_out.data_ptr(), sampled_out.data_ptr(), self.stats_dev.data_ptr(),
                                             self._ws_ptr, self.workspace_bytes, _stream_ptr(stream)))
        return phase_out, motion_out, sampled_out

    def stats(self) -> _lib.WrLKStats:
        return _lib.WrLKStats.from_buffer_copy(self.stats_dev.cpu().numpy().tobytes())

    def error_log(self):
        return stats_to_log(self.stats(), self.params.layer + 1)


def _to_device(a, device, dtype):
    """(x, y, z[, 3]) array -> contiguous (z, y, x[, 3]) CUDA tensor."""
    if isinstance(a, torch.Tensor):
        t = a.to(device=device, dtype=dtype)
    else:
        t = torch.from_numpy(np.ascontiguousarray(np.asarray(a).astype(np.float32 if dtype == torch.float32 else
                                                                       np.float64, copy=False))).to(device)
        t = t.to(dtype)
    perm = (2, 1, 0, 3) if t.dim() == 4 else (2, 1, 0)
    return t.permute(*perm).contiguous()


def _mask_to_device(m, shape_xyz, device):
    """Exclusion mask (x, y, z) -> (z, y, x) uint8 CUDA tensor, or None for
    an all-zero / scalar-zero mask.  Values are kept (the reference resizes
    the float32 cast of the mask and thresholds it at 0.5)."""
    if m is None or np.isscalar(m) or (hasattr(m, "ndim") and m.ndim == 0):
        if m is not None and float(np.asarray(m)) > 0.5:
            raise ValueError("a scalar exclusion mask must be 0")
        return None
    if isinstance(m, torch.Tensor):
        t = m.to(device)
        if tuple(t.shape) != tuple(shape_xyz):
            raise ValueError(f"mask shape {tuple(t.shape)} does not match the volume {tuple(shape_xyz)}")
        vals = t
    else:
        a = np.asarray(m)
        if tuple(a.shape) != tuple(shape_xyz):
            raise ValueError(f"mask shape {a.shape} does not match the volume {tuple(shape_xyz)}")
        vals = torch.from_numpy(np.ascontiguousarray(a)).to(device)
    if vals.dtype == torch.bool:
        vals = vals.to(torch.uint8)
    if vals.dtype != torch.uint8:
        f = vals.to(torch.float32)
        if bool(((f != 0) & (f != 1)).any()):
            raise ValueError("exclusion masks must hold 0/1 (or bool) values")
        vals = f.to(torch.uint8)
    return vals.permute(2, 1, 0).contiguous()


_cache: dict = {}
last_registrar = None   # the XresRegistrar of the latest getMotion_v2 call (its error_log / stats)


def getMotion_v2(data_mov, data_ref, option, verbose=False):
    """Cross-resolution registration (utils/calFlowCrossResolution.py:2470-2663).

    Returns (phase_new, motion_current, data_ref_sampled) in the reference's
    (x, y, z[, 3]) layout.
    """
    wr = None
    if bool(option.get("wrong_region_enable", True)):
        metric = str(option.get("wrong_region_metric", "mse")).lower()
        if metric not in ("mse", "mae"):
            raise ValueError("metric must be 'mse' or 'mae'")
        # utils/calFlowCrossResolution.py:2340 tests only for "highresidual";
        # every other value (None, "Direct", ...) takes the direct exclusion
        exclude_high = option.get("wrong_region_exclude_mode", "direct") == "highresidual"
        wr = _lib.WrXresWrongRegion(1, 0 if metric == "mse" else 1,
                                    float(option.get("wrong_region_mad_threshold", 3.0)),
                                    int(option.get("wrong_region_min_component_size", 2)),
                                    float(option.get("expand_radius_xy", 2.0)), float(option.get("sigma_grad", 1.0)),
                                    float(option.get("intensity_k", 2.0)), 1 if exclude_high else 0,
                                    float(option.get("quantile_threshold_q", 0.8)))
    as_torch = isinstance(data_mov, torch.Tensor)
    device = data_mov.device if as_torch and data_mov.is_cuda else torch.device("cuda", torch.cuda.current_device())
    mov = _to_device(data_mov, device, torch.float32)
    ref = _to_device(data_ref, device, torch.float32)
    shape_xyz = tuple(mov.shape[::-1])
    ref_xyz = tuple(ref.shape[::-1])
    mask_mov = _mask_to_device(option["mask_mov"], shape_xyz, device)
    mask_ref = _mask_to_device(option["mask_ref"], ref_xyz, device)
    init = option.get("motion")
    init_t = None if init is None else _to_device(init, device, torch.float32)
    phase0 = option.get("phase")
    phase_t = None if phase0 is None else _to_device(phase0, device, torch.float32)
    params = LKParams(
        layer=int(option["layer"]), iter=int(option["iter"]), r=int(option["r"]),
        zRatio=float(option.get("zRatio", 1.0)), movRange=float(option.get("movRange", 5.0)),
        smoothPenalty=float(option["smoothPenalty"]), tol=float(option.get("tol", 1e-3)),
        forced_updates=dict(option.get("forced_updates") or {}))
    zr_hr = float(option["zRatio_HR"])
    key = (tuple(mov.shape), tuple(ref.shape), params.layer, params.iter, params.r, params.zRatio, params.movRange,
           params.smoothPenalty, params.tol, tuple(sorted(params.forced_updates.items())), zr_hr,
           mask_ref is not None, phase_t is not None,
           None if wr is None else tuple(getattr(wr, f) for f, _ in wr._fields_), str(device))
    reg = _cache.get(key)
    if reg is None:
        if len(_cache) > 4:
            _cache.clear()
        reg = XresRegistrar(tuple(mov.shape), tuple(ref.shape), params, zr_hr, mask_ref is not None, device,
                            has_phase_init=phase_t is not None, wrong_region=wr)
        _cache[key] = reg
    global last_registrar
    last_registrar = reg
    phase, motion, sampled = reg.register(mov, ref, mask_mov, mask_ref, init_t, phase_init=phase_t)
    if verbose:
        log, err = reg.error_log()
        for name, lv in log.items():
            for i, (d, p) in enumerate(zip(lv["diffError"], lv["penaltyError"])):
                print(f"[{name}] iter={i:02d} error={d + p:.4f} diff={d:.4f} penalty={p:.4f}")
    phase = phase.permute(2, 1, 0, 3)
    motion = motion.permute(2, 1, 0, 3)
    sampled = sampled.permute(2, 1, 0).to(torch.float64)
    if as_torch:
        return phase.contiguous(), motion.contiguous(), sampled.contiguous()
    return (np.ascontiguousarray(phase.cpu().numpy()), np.ascontiguousarray(motion.cpu().numpy()),
            np.ascontiguousarray(sampled.cpu().numpy()))


# ---------------------------------------------------------------------------
# continuous reference H and fixed-plane projections
# ---------------------------------------------------------------------------

def _cuda_f32(a, device=None):
    device = device or torch.device("cuda", torch.cuda.current_device())
    if isinstance(a, torch.Tensor):
        return a.to(device=device, dtype=torch.float32)
    return torch.from_numpy(np.ascontiguousarray(np.asarray(a, dtype=np.float32))).to(device)


def _workspace(nbytes, device):
    return torch.empty(int(nbytes) + 256, dtype=torch.uint8, device=device)


def _aligned(buf):
    return (buf.data_ptr() + 255) // 256 * 256


def spline_sample(vol_zyx: torch.Tensor, coords_xyz: torch.Tensor, stream=None) -> torch.Tensor:
    """Cubic B-spline (order 3, mode "nearest") of a (z, y, x) float32 CUDA
    volume at (n, 3) points (x, y, z); (n,) float32 (``wr_spline_sample``)."""
    lib = _lib.load()
    vol = vol_zyx.to(torch.float32).contiguous()
    pts = coords_xyz.to(device=vol.device, dtype=torch.float32).reshape(-1, 3).contiguous()
    nz, ny, nx = (int(v) for v in vol.shape)
    need = ctypes.c_size_t(0)
    _lib.check("wr_spline_workspace_size", lib.wr_spline_workspace_size(nz, ny, nx, ctypes.byref(need)))
    ws = _workspace(need.value, vol.device)
    out = torch.empty(pts.shape[0], dtype=torch.float32, device=vol.device)
    _lib.check("wr_spline_sample", lib.wr_spline_sample(vol.data_ptr(), nz, ny, nx, pts.data_ptr(), pts.shape[0],
                                                        out.data_ptr(), _aligned(ws), int(need.value),
                                                        _stream_ptr(stream)))
    return out


def generate_continuous_H_gpu(stack, zRatio):
    """``H`` of calFlowCrossResolution.py:463-478: a callable mapping
    (..., 3) physical coordinates (z divided by ``zRatio``) to the cubic
    spline of ``stack`` (x, y, z), float32."""
    vol = _cuda_f32(stack).permute(2, 1, 0).contiguous()
    zr = float(zRatio)

    def H(coords_phys):
        c = _cuda_f32(coords_phys, vol.device).clone()
        c[..., 2] = c[..., 2] / zr
        return spline_sample(vol, c.reshape(-1, 3)).reshape(c.shape[:-1])

    return H


def apply_H_to_matrix_gpu(A, H):
    """calFlowCrossResolution.py:1144-1154: H at every (x, y, z) of A (..., 3)."""
    return H(A)


def _ref_xyz_shape(ref_volume, order):
    if order == "xyz":
        X, Y, Z = ref_volume.shape
    elif order == "zyx":
        Z, Y, X = ref_volume.shape
    else:
        raise ValueError("ref_volume_order should be 'xyz' or 'zyx'.")
    return int(X), int(Y), int(Z)


def _projection_inputs(coords_ref_xyk_xyz, ref_volume, target_z_planes, values_xyk, ref_volume_order,
                       downsample_xy):
    coords = _cuda_f32(coords_ref_xyk_xyz)
    if coords.dim() != 4 or coords.shape[-1] != 3:
        raise ValueError(f"coords_ref_xyk_xyz should have shape (X,Y,K,3), got {tuple(coords.shape)}")
    ref = _cuda_f32(ref_volume, coords.device)
    if ref.dim() != 3:
        raise ValueError(f"ref_volume should be 3D, got {tuple(ref.shape)}")
    X, Y, _ = _ref_xyz_shape(ref, ref_volume_order)
    ds = int(downsample_xy)
    if ds < 1:
        raise ValueError("downsample_xy should be >= 1.")
    target = _cuda_f32(np.atleast_1d(np.asarray(target_z_planes, dtype=np.float32)), coords.device).reshape(-1)
    pts = coords.reshape(-1, 3).contiguous()
    if values_xyk is None:
        vol_zyx = ref.permute(2, 1, 0).contiguous() if ref_volume_order == "xyz" else ref.contiguous()
        values = spline_sample(vol_zyx, pts)
    else:
        values = _cuda_f32(values_xyk, coords.device)
        if tuple(values.shape) != tuple(coords.shape[:-1]):
            raise ValueError(f"values_xyk shape {tuple(values.shape)} does not match coords shape "
                             f"{tuple(coords.shape[:-1])}")
        values = values.reshape(-1).contiguous()
    return pts, values, target, X, Y, ds


def project_coords_to_fixed_planes_gpu(coords_ref_xyk_xyz, ref_volume=None, target_z_planes=None, values_xyk=None,
                                       ref_volume_order="xyz", z_window=1.5, downsample_xy=1, fill_value=0.0,
                                       return_numpy=False, output_order="zyx", xy_splat_mode="subpixel_footprint",
                                       xy_extra_radius=0):
    """Max splat of mapped samples onto fixed reference z planes
    (calFlowCrossResolution.py:878-1141, kernel :480-569)."""
    if target_z_planes is None:
        raise ValueError("target_z_planes must be provided.")
    if ref_volume is None:
        raise ValueError("ref_volume must be provided to infer reference shape.")
    if xy_splat_mode == "nearest":
        nearest, extra = 1, 0
    elif xy_splat_mode == "subpixel_footprint":
        nearest, extra = 0, int(xy_extra_radius)
        if extra < 0:
            raise ValueError("xy_extra_radius should be >= 0.")
    else:
        raise ValueError("xy_splat_mode should be 'nearest' or 'subpixel_footprint'.")
    if output_order not in ("zyx", "zxy"):
        raise ValueError("output_order should be 'zyx' or 'zxy'.")
    pts, values, target, X, Y, ds = _projection_inputs(coords_ref_xyk_xyz, ref_volume, target_z_planes, values_xyk,
                                                       ref_volume_order, downsample_xy)
    lib = _lib.load()
    npl = int(target.numel())
    xo, yo = (X + ds - 1) // ds, (Y + ds - 1) // ds
    need = ctypes.c_size_t(0)
    _lib.check("wr_project_workspace_size", lib.wr_project_workspace_size(npl, X, Y, ds, ctypes.byref(need)))
    ws = _workspace(need.value, pts.device)
    out = torch.empty((npl, xo, yo), dtype=torch.float32, device=pts.device)
    _lib.check("wr_project_planes_max",
               lib.wr_project_planes_max(values.data_ptr(), pts.data_ptr(), values.numel(), target.data_ptr(), npl, X,
                                         Y, ds, float(z_window), nearest, extra,
                                         0.0 if fill_value is None else float(fill_value),
                                         0 if fill_value is None else 1, out.data_ptr(), _aligned(ws), int(need.value),
                                         _stream_ptr(None)))
    if output_order == "zyx":
        out = out.transpose(1, 2)
    return out.cpu().numpy() if return_numpy else out


def project_coords_to_fixed_planes_weighted_gpu(coords_ref_xyk_xyz, ref_volume, target_z_planes, values_xyk=None,
                                                ref_volume_order="xyz", z_window=1.5, z_sigma=None,
                                                z_weight_mode="gaussian", downsample_xy=1, fill_value=0.0,
                                                return_numpy=False, output_order="zyx", eps=1e-6):
    """Weighted bilinear splat onto fixed reference z planes
    (calFlowCrossResolution.py:700-876, kernel :571-660); returns
    (planes, summed weights)."""
    modes = {"hard": 0, "triangular": 1, "gaussian": 2}
    if z_weight_mode not in modes:
        raise ValueError("z_weight_mode should be 'hard', 'triangular', or 'gaussian'.")
    if output_order not in ("zyx", "zxy"):
        raise ValueError("output_order should be 'zyx' or 'zxy'.")
    pts, values, target, X, Y, ds = _projection_inputs(coords_ref_xyk_xyz, ref_volume, target_z_planes, values_xyk,
                                                       ref_volume_order, downsample_xy)
    if z_sigma is None:
        z_sigma = float(z_window) * 0.5
    lib = _lib.load()
    npl = int(target.numel())
    xo, yo = (X + ds - 1) // ds, (Y + ds - 1) // ds
    need = ctypes.c_size_t(0)
    _lib.check("wr_project_workspace_size", lib.wr_project_workspace_size(npl, X, Y, ds, ctypes.byref(need)))
    ws = _workspace(need.value, pts.device)
    out = torch.empty((npl, xo, yo), dtype=torch.float32, device=pts.device)
    wout = torch.empty((npl, xo, yo), dtype=torch.float32, device=pts.device)
    _lib.check("wr_project_planes_weighted",
               lib.wr_project_planes_weighted(values.data_ptr(), pts.data_ptr(), values.numel(), target.data_ptr(),
                                              npl, X, Y, ds, float(z_window), float(z_sigma),
                                              modes[z_weight_mode], float(fill_value), float(eps), out.data_ptr(),
                                              wout.data_ptr(), _aligned(ws), int(need.value), _stream_ptr(None)))
    if output_order == "zyx":
        out, wout = out.transpose(1, 2), wout.transpose(1, 2)
    if return_numpy:
        return out.cpu().numpy(), wout.cpu().numpy()
    return out, wout
