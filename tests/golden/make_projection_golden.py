"""Fixtures of the reference's own projection kernels (needs a GPU).

Runs project_to_planes_nanmax_kernel and project_to_planes_weighted_avg_kernel
(src/wholistic_registration/utils/calFlowCrossResolution.py:480-660), built
from the reference's source by oracle/build_ref_projection.py, on seeded
inputs, with the steps their wrappers take around the launch done here in
NumPy as the wrappers do them in CuPy:

* max splat (project_coords_to_fixed_planes_gpu, :878-1141): values shifted
  by max(1 - min(finite values), 0) in float32, output initialised to -inf,
  shift taken off the finite outputs, fill value elsewhere;
* weighted splat (project_coords_to_fixed_planes_weighted_gpu, :700-876):
  sums initialised to 0, z_sigma = z_window / 2 when not given, output
  sum_val / max(sum_w, eps) where sum_w > eps, fill value elsewhere.

Writes projection_ref.npz (inputs, raw kernel outputs, final outputs, in the
wrappers' internal (planes, Xout, Yout) order) to the directory given (default
this one).  Usage: python tests/golden/make_projection_golden.py [out_dir]
"""

from __future__ import annotations

import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
LIB = os.path.join(ROOT, "oracle", "_ref", "libref_projection.so")

# (seed, planes, z_window, splat mode, extra radius, downsample, fill)
MAX_CASES = {
    "max_sub_e0_d1": (5, [0.0, 2.5, 5.0], 1.2, "subpixel_footprint", 0, 1, -7.0),
    "max_sub_e1_d2": (5, [0.0, 2.5, 5.0], 1.2, "subpixel_footprint", 1, 2, -7.0),
    "max_near_d3": (5, [0.0, 2.5, 5.0], 1.2, "nearest", 0, 3, -7.0),
    "max_sub_e2_d1_negative": (7, [1.0, 4.0], 2.0, "subpixel_footprint", 2, 1, 0.0),
}
# (seed, planes, z_window, z_sigma or None, weight mode, downsample, fill, eps)
WEIGHTED_CASES = {
    "w_hard_d2": (6, [1.0, 3.0], 1.5, None, "hard", 2, 0.0, 1e-6),
    "w_tri_d2": (6, [1.0, 3.0], 1.5, None, "triangular", 2, 0.0, 1e-6),
    "w_gauss_d2": (6, [1.0, 3.0], 1.5, None, "gaussian", 2, 0.0, 1e-6),
    "w_gauss_sigma_d1": (8, [0.5, 2.0, 4.5], 1.0, 0.7, "gaussian", 1, -1.0, 1e-6),
}
WMODES = {"hard": 0, "triangular": 1, "gaussian": 2}


def projection_inputs(seed):
    """Samples at mapped coordinates (X, Y, K, 3) around a (21, 19, 6)
    reference, with a NaN value and an infinite coordinate."""
    rng = np.random.default_rng(seed)
    X, Y, K = 20, 18, 4
    coords = np.stack([rng.uniform(-2, 22, (X, Y, K)), rng.uniform(-2, 20, (X, Y, K)),
                       rng.uniform(-1, 7, (X, Y, K))], -1).astype(np.float32)
    values = rng.normal(50, 80, (X, Y, K)).astype(np.float32)
    values[0, 0, 0] = np.nan
    coords[1, 1, 1, 0] = np.inf
    return coords, values, (21, 19)


def _dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def main(out_dir):
    import torch

    lib = ctypes.CDLL(LIB)
    P, i64, i32, f32 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32, ctypes.c_float
    lib.ref_project_nanmax_launch.argtypes = [P, P, P, P, i64, i32, i32, i32, i32, i32, f32, i32, i32, i32]
    lib.ref_project_weighted_launch.argtypes = [P, P, P, P, P, i64, i32, i32, i32, i32, i32, f32, f32, i32, i32]
    rec = {}
    for name, (seed, planes, zw, mode, extra, ds, fill) in MAX_CASES.items():
        coords, values, (xr, yr) = projection_inputs(seed)
        if name.endswith("negative"):
            values = values - np.float32(400.0)
        xo, yo = (xr + ds - 1) // ds, (yr + ds - 1) // ds
        fin = values[np.isfinite(values)]
        shift = np.maximum(-fin.min() + np.float32(1.0), np.float32(0.0)).astype(np.float32)
        vk = (values + shift).astype(np.float32)
        tz = np.asarray(planes, np.float32)
        out = torch.full((len(planes), xo, yo), -np.inf, dtype=torch.float32, device="cuda")
        dv, dc, dz = _dev(vk.reshape(-1)), _dev(coords.reshape(-1, 3)), _dev(tz)
        rc = lib.ref_project_nanmax_launch(dv.data_ptr(), dc.data_ptr(), dz.data_ptr(), out.data_ptr(), vk.size,
                                           len(planes), xr, yr, xo, yo, zw, ds, int(mode == "nearest"),
                                           extra if mode != "nearest" else 0)
        assert rc == 0, rc
        raw = out.cpu().numpy()
        fo = np.where(np.isfinite(raw), raw - shift, raw)
        fo = np.where(np.isfinite(fo), fo, np.float32(fill)).astype(np.float32)
        rec[f"{name}_coords"], rec[f"{name}_values"], rec[f"{name}_planes"] = coords, values, tz
        rec[f"{name}_params"] = np.array([xr, yr, zw, int(mode == "nearest"), extra, ds, fill], np.float64)
        rec[f"{name}_raw"], rec[f"{name}_out"] = raw, fo
    for name, (seed, planes, zw, zs, wmode, ds, fill, eps) in WEIGHTED_CASES.items():
        coords, values, (xr, yr) = projection_inputs(seed)
        xo, yo = (xr + ds - 1) // ds, (yr + ds - 1) // ds
        tz = np.asarray(planes, np.float32)
        sv = torch.zeros((len(planes), xo, yo), dtype=torch.float32, device="cuda")
        sw = torch.zeros_like(sv)
        dv, dc, dz = _dev(values.reshape(-1)), _dev(coords.reshape(-1, 3)), _dev(tz)
        sigma = float(zw) * 0.5 if zs is None else zs
        rc = lib.ref_project_weighted_launch(dv.data_ptr(), dc.data_ptr(), dz.data_ptr(), sv.data_ptr(),
                                             sw.data_ptr(), values.size, len(planes), xr, yr, xo, yo, zw, sigma, ds,
                                             WMODES[wmode])
        assert rc == 0, rc
        s_val, s_w = sv.cpu().numpy(), sw.cpu().numpy()
        e32 = np.float32(eps)
        fo = np.where(s_w > e32, s_val / np.maximum(s_w, e32), np.float32(fill)).astype(np.float32)
        rec[f"{name}_coords"], rec[f"{name}_values"], rec[f"{name}_planes"] = coords, values, tz
        rec[f"{name}_params"] = np.array([xr, yr, zw, -1.0 if zs is None else zs, WMODES[wmode], ds, fill, eps],
                                         np.float64)
        rec[f"{name}_sum_val"], rec[f"{name}_sum_w"], rec[f"{name}_out"] = s_val, s_w, fo
    path = os.path.join(out_dir, "projection_ref.npz")
    np.savez_compressed(path, **rec)
    print(path, len(MAX_CASES), "max cases,", len(WEIGHTED_CASES), "weighted cases")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else HERE)
