"""ctypes binding of the C ABI in ``include/wr_b200.h`` (and ``wr_net.h``, ``wr_mask.h``, ``wr_xres.h``).

The shared library ``_wr_b200.so`` is built in-tree by
``wholistic_registration_b200.build``.  Loading fails loudly when it is
missing: there is no CPU fallback for the registration path.
"""

from __future__ import annotations

import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_wr_b200.so")

MAX_LEVELS = 8
MAX_ITERS = 64
MAX_BATCH = 64

WR_U8, WR_U16, WR_F32 = 1, 2, 3
WR_PREC_F32, WR_PREC_F16, WR_PREC_BF16 = 0, 1, 2
WR_LK_REUSE_REFERENCE = 1
WR_LK_TILE_ORDER_X = 1 << 8
WR_LK_CTAS_PER_SM_SHIFT = 12


def WR_LK_CTAS_PER_SM(n: int) -> int:
    return (int(n) & 15) << WR_LK_CTAS_PER_SM_SHIFT

ERRORS = {
    1: "WR_E_NULL",
    2: "WR_E_SHAPE",
    3: "WR_E_PARAM",
    4: "WR_E_DTYPE",
    5: "WR_E_WORKSPACE",
    6: "WR_E_NOCP",
}

EXPORTS = (
    "wr_abi_version",
    "wr_last_error",
    "wr_lk_workspace_size",
    "wr_lk_register",
    "wr_lk_register_profiled",
    "wr_lk_register_warp",
    "wr_lk_register_snapshots",
    "wr_lk_batch_workspace_size",
    "wr_lk_register_batch",
    "wr_lk_batch_each_workspace_size",
    "wr_lk_register_batch_each",
    "wr_warp_trilinear",
    "wr_penalty_factor",
    "wr_penalty_factor_noalloc",
    "wr_penalty_factor_scratch",
    "wr_resize_table",
    "wr_net_last_error",
    "wr_net_tc_error",
    "wr_net_conv3d_fwd",
    "wr_net_conv3d_dgrad",
    "wr_net_conv3d_wgrad",
    "wr_net_act_backward",
    "wr_net_split_grad",
    "wr_net_adam",
    "wr_net_weights_to_bf16",
    "wr_net_flow_loss",
    "wr_net_prepare_input",
    "wr_net_masked_sse",
    "wr_net_pool_flow",
    "wr_net_upsample_flow",
    "wr_mask_last_error",
    "wr_frame_gram",
    "wr_mask_workspace_size",
    "wr_get_mask",
    "wr_bwareafilt3",
    "wr_xres_workspace_size",
    "wr_xres_register",
    "wr_spline_workspace_size",
    "wr_spline_sample",
    "wr_project_workspace_size",
    "wr_project_planes_max",
    "wr_project_planes_weighted",
)


class WrXresWrongRegion(ctypes.Structure):
    """include/wr_xres.h: getMotion_v2's wrong-region correction options."""
    _fields_ = [
        ("enable", ctypes.c_int32),
        ("metric", ctypes.c_int32),
        ("mad_threshold", ctypes.c_float),
        ("min_component_size", ctypes.c_int32),
        ("expand_radius_xy", ctypes.c_float),
        ("sigma_grad", ctypes.c_float),
        ("intensity_k", ctypes.c_float),
        ("exclude_mode", ctypes.c_int32),
        ("quantile_q", ctypes.c_float),
    ]


class WrVolume(ctypes.Structure):
    _fields_ = [
        ("data", ctypes.c_void_p),
        ("dtype", ctypes.c_int32),
        ("nz", ctypes.c_int32),
        ("ny", ctypes.c_int32),
        ("nx", ctypes.c_int32),
    ]


class WrLKParams(ctypes.Structure):
    _fields_ = [
        ("layer", ctypes.c_int32),
        ("iter", ctypes.c_int32),
        ("r", ctypes.c_int32),
        ("zRatio", ctypes.c_float),
        ("movRange", ctypes.c_float),
        ("smoothPenalty", ctypes.c_double),
        ("tol", ctypes.c_double),
        ("precision", ctypes.c_int32),
        ("flags", ctypes.c_int32),
        ("forced_updates", ctypes.c_int32 * MAX_LEVELS),
    ]


class WrLKStats(ctypes.Structure):
    _fields_ = [
        ("levels", ctypes.c_int32),
        ("evals", ctypes.c_int32 * MAX_LEVELS),
        ("updates", ctypes.c_int32 * MAX_LEVELS),
        ("nan_solves", ctypes.c_int32),
        ("fp64_solves", ctypes.c_int32),
        ("current_error", ctypes.c_double),
        ("diff_error", (ctypes.c_double * MAX_ITERS) * MAX_LEVELS),
        ("penalty_error", (ctypes.c_double * MAX_ITERS) * MAX_LEVELS),
        ("max_diff_motion", (ctypes.c_double * MAX_ITERS) * MAX_LEVELS),
    ]


class WrProfile(ctypes.Structure):
    _fields_ = [
        ("acc_begin", ctypes.POINTER(ctypes.c_void_p)),
        ("acc_end", ctypes.POINTER(ctypes.c_void_p)),
        ("capacity", ctypes.c_int32),
        ("recorded", ctypes.c_int32),
        ("launches", ctypes.c_int32),
        ("pad", ctypes.c_int32),
    ]


class WrSnapshots(ctypes.Structure):
    """getMotion's error_log snapshots (include/wr_b200.h): device float32 arrays per level."""
    _fields_ = [
        ("save_ite", ctypes.c_int32),
        ("capacity", ctypes.c_int32),
        ("motion", ctypes.c_void_p * MAX_LEVELS),
        ("warped", ctypes.c_void_p * MAX_LEVELS),
        ("level_ref", ctypes.c_void_p * MAX_LEVELS),
        ("level_mov", ctypes.c_void_p * MAX_LEVELS),
    ]


class WrLKItem(ctypes.Structure):
    _fields_ = [
        ("mov", WrVolume),
        ("ref", WrVolume),
        ("excl_mask_mov", ctypes.c_void_p),
        ("excl_mask_ref", ctypes.c_void_p),
        ("motion_init", ctypes.c_void_p),
        ("motion_out", ctypes.c_void_p),
        ("warped_out", ctypes.c_void_p),
        ("stats", ctypes.c_void_p),
    ]


class WrConvGeom(ctypes.Structure):
    _fields_ = [(k, ctypes.c_int32) for k in
                ("n", "oz", "oy", "ox", "iz", "iy", "ix", "stride", "c1", "c2", "up1", "cout", "act")]


class WrError(RuntimeError):
    """A C-ABI call returned a nonzero status."""

    def __init__(self, fn, code, msg):
        kind = ERRORS.get(code, f"CUDA error {-code}" if code < 0 else f"code {code}")
        super().__init__(f"{fn}: {kind}: {msg}")
        self.code = code


class ArgumentError(WrError, ValueError):
    """Invalid argument reported by the library (maps to the reference's ValueError)."""


_lock = threading.Lock()
_lib = None


def load():
    """Load the library (once) and declare argument types."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m wholistic_registration_b200.build` "
                "(the registration path has no CPU fallback)")
        lib = ctypes.CDLL(LIB_PATH)
        vp, i32, sz = ctypes.c_void_p, ctypes.c_int32, ctypes.c_size_t
        lib.wr_abi_version.restype = ctypes.c_int
        lib.wr_last_error.restype = ctypes.c_char_p
        lib.wr_lk_workspace_size.argtypes = [i32, i32, i32, ctypes.POINTER(WrLKParams), ctypes.POINTER(sz)]
        lib.wr_lk_register.argtypes = [ctypes.POINTER(WrVolume), ctypes.POINTER(WrVolume), vp, vp,
                                       ctypes.POINTER(WrLKParams), vp, vp, vp, vp, sz, vp]
        lib.wr_lk_register_profiled.argtypes = lib.wr_lk_register.argtypes + [ctypes.POINTER(WrProfile)]
        lib.wr_lk_register_snapshots.argtypes = lib.wr_lk_register.argtypes + [ctypes.POINTER(WrSnapshots)]
        lib.wr_frame_gram.argtypes = [vp, i32, ctypes.c_int64, vp, vp, vp]
        lib.wr_lk_batch_workspace_size.argtypes = [ctypes.POINTER(WrLKItem), i32, ctypes.POINTER(WrLKParams),
                                                   ctypes.POINTER(sz)]
        lib.wr_lk_register_batch.argtypes = [ctypes.POINTER(WrLKItem), i32, ctypes.POINTER(WrLKParams), vp, sz, vp]
        lib.wr_lk_batch_each_workspace_size.argtypes = [ctypes.POINTER(WrLKItem), ctypes.POINTER(WrLKParams), i32,
                                                        ctypes.POINTER(sz)]
        lib.wr_lk_register_batch_each.argtypes = [ctypes.POINTER(WrLKItem), ctypes.POINTER(WrLKParams), i32, vp, sz,
                                                  vp]
        lib.wr_lk_register_warp.argtypes = (lib.wr_lk_register.argtypes[:7] + [vp] + lib.wr_lk_register.argtypes[7:]
                                            + [ctypes.POINTER(WrProfile)])
        lib.wr_warp_trilinear.argtypes = [ctypes.POINTER(WrVolume), vp, vp, vp]
        lib.wr_penalty_factor.argtypes = [ctypes.POINTER(WrVolume), vp, vp, vp, sz, vp]
        lib.wr_penalty_factor_noalloc.argtypes = [ctypes.POINTER(WrVolume), vp, vp, vp]
        lib.wr_penalty_factor_scratch.argtypes = [i32, i32, i32, ctypes.POINTER(sz)]
        lib.wr_resize_table.argtypes = [i32, i32, i32, vp, vp, ctypes.POINTER(i32)]
        G = ctypes.POINTER(WrConvGeom)
        f32, i64, fl = ctypes.c_float, ctypes.c_longlong, ctypes.c_float
        lib.wr_net_conv3d_fwd.argtypes = [G, vp, vp, vp, vp, vp, vp, vp]
        lib.wr_net_conv3d_dgrad.argtypes = [G, vp, vp, vp, vp]
        lib.wr_net_conv3d_wgrad.argtypes = [G, vp, vp, vp, vp, vp, vp]
        lib.wr_net_act_backward.argtypes = [vp, vp, ctypes.c_int, vp, i64, ctypes.c_int, vp]
        lib.wr_net_split_grad.argtypes = [G, vp, vp, vp, vp]
        lib.wr_net_adam.argtypes = [vp, vp, vp, vp, i64, f32, f32, f32, f32, ctypes.c_int, f32, vp]
        lib.wr_net_weights_to_bf16.argtypes = [vp, vp, vp, ctypes.c_int, ctypes.c_int, vp]
        lib.wr_net_flow_loss.argtypes = [vp, vp, vp, vp, vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_int, fl, fl, fl, vp]
        ci = ctypes.c_int
        lib.wr_net_prepare_input.argtypes = [ctypes.POINTER(WrVolume), ctypes.POINTER(WrVolume), ci, vp, vp, vp, vp, vp]
        lib.wr_net_masked_sse.argtypes = [vp, ctypes.POINTER(WrVolume), vp, vp, vp]
        lib.wr_net_pool_flow.argtypes = [vp, ci, ci, ci, ci, vp, vp]
        lib.wr_net_upsample_flow.argtypes = [vp, ci, ci, ci, ci, vp, vp]
        lib.wr_mask_workspace_size.argtypes = [i32, i32, i32, ctypes.POINTER(sz)]
        lib.wr_get_mask.argtypes = [ctypes.POINTER(WrVolume), ctypes.c_double, ctypes.c_double, vp, vp, vp, sz, vp]
        lib.wr_bwareafilt3.argtypes = [vp, i32, i32, i32, ctypes.c_int64, ctypes.c_int64, vp, vp, vp, vp, sz, vp]
        P = ctypes.POINTER(WrLKParams)
        WR = ctypes.POINTER(WrXresWrongRegion)
        lib.wr_xres_workspace_size.argtypes = [i32, i32, i32, i32, i32, i32, P, ctypes.c_float, i32, i32, WR,
                                               ctypes.POINTER(sz)]
        lib.wr_xres_register.argtypes = [vp, i32, i32, i32, vp, i32, i32, i32, vp, vp, vp, vp, P, ctypes.c_float,
                                         WR, vp, vp, vp, vp, vp, sz, vp]
        i64_, f32_ = ctypes.c_int64, ctypes.c_float
        lib.wr_spline_workspace_size.argtypes = [i32, i32, i32, ctypes.POINTER(sz)]
        lib.wr_spline_sample.argtypes = [vp, i32, i32, i32, vp, i64_, vp, vp, sz, vp]
        lib.wr_project_workspace_size.argtypes = [i32, i32, i32, i32, ctypes.POINTER(sz)]
        lib.wr_project_planes_max.argtypes = [vp, vp, i64_, vp, i32, i32, i32, i32, f32_, i32, i32, f32_, i32, vp,
                                              vp, sz, vp]
        lib.wr_project_planes_weighted.argtypes = [vp, vp, i64_, vp, i32, i32, i32, i32, f32_, f32_, i32, f32_, f32_,
                                                   vp, vp, vp, sz, vp]
        for name in EXPORTS:
            getattr(lib, name).restype = (ctypes.c_char_p if name.endswith("last_error") else ctypes.c_int)
        if lib.wr_abi_version() != 1:
            raise ImportError("wr_b200 ABI version mismatch")
        _lib = lib
        return lib


def check(fn, code):
    if code != 0:
        lib = load()
        if fn.startswith("wr_net"):
            raw = lib.wr_net_last_error()
        elif fn in ("wr_get_mask", "wr_bwareafilt3", "wr_frame_gram") or fn.startswith("wr_mask"):
            raw = lib.wr_mask_last_error()
        else:
            raw = lib.wr_last_error()
        msg = raw.decode(errors="replace")
        if code > 0:
            raise ArgumentError(fn, code, msg)
        raise WrError(fn, code, msg)


def volume(ptr, dtype_code, shape_zyx):
    nz, ny, nx = (int(s) for s in shape_zyx)
    return WrVolume(ctypes.c_void_p(ptr), dtype_code, nz, ny, nx)
