"""Generate golden fixtures by running the reference package itself.

Run in a container where the reference checkout is available:

    python tests/golden/make_golden.py --ref <reference checkout>
    (or set WR_REFERENCE_ROOT)

It imports the reference's NumPy path (``wholistic_registration.utils``) through
a stub top-level package, because the package ``__init__`` pulls in I/O
libraries that the hot path does not need.  Outputs are written next to this
script as compressed ``.npz`` files and committed; the tests read only those
files, never the reference tree.

Every array is in the reference's internal (x, y, z) layout.
"""

from __future__ import annotations

import argparse
import importlib
import json
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from wholistic_registration_b200 import synthetic  # noqa: E402

sys.path.insert(0, HERE)
from bench_cases import BENCH_CASES, BENCH_ITER, BENCH_R, BENCH_RAW_PENALTY, bench_inputs  # noqa: E402


def load_reference(root):
    src = os.path.join(root, "src", "wholistic_registration")
    if "wholistic_registration" not in sys.modules:
        pkg = types.ModuleType("wholistic_registration")
        pkg.__path__ = [src]
        sys.modules["wholistic_registration"] = pkg
    mods = {}
    for name in ("calFlow3d_Wei_v1", "imresize", "preprocess", "calculate"):
        mods[name] = importlib.import_module(f"wholistic_registration.utils.{name}")
    return mods


def _pair_xyz(zyx, seed, n_blobs, max_disp, drift=0.0):
    tmpl, mov, field = synthetic.make_pair(zyx, seed, n_blobs=n_blobs, max_disp=max_disp, drift=drift)
    t = tmpl.to(dtype=__import__("torch").int32).numpy().astype(np.uint16).transpose(2, 1, 0)
    m = mov.to(dtype=__import__("torch").int32).numpy().astype(np.uint16).transpose(2, 1, 0)
    f = field.numpy().transpose(2, 1, 0, 3)
    return np.ascontiguousarray(t), np.ascontiguousarray(m), np.ascontiguousarray(f)


# name: (z, y, x), seed, blobs, max_disp, r, layer, iter, zRatio, tol, raw penalty, mask kind, init
MOTION_CASES = {
    "tiny_r1_l0": ((4, 24, 24), 1, 40, (1.5, 1.5, 0.5), 1, 0, 5, 1.0, 1e-3, 0.08, "none", False),
    "small_r2_l1": ((6, 48, 48), 2, 120, (2.0, 2.0, 0.8), 2, 1, 10, 1.0, 1e-3, 0.08, "none", False),
    "mask_r3_l1_z2": ((8, 64, 64), 3, 200, (2.5, 2.5, 1.0), 3, 1, 10, 2.0, 1e-3, 0.08, "ellipse", False),
    "init_r4_l2": ((5, 64, 48), 4, 150, (3.0, 3.0, 1.0), 4, 2, 10, 1.0, 1e-4, 0.05, "none", True),
    "ragged_r3_l2": ((6, 70, 66), 5, 200, (3.0, 2.0, 1.0), 3, 2, 10, 1.0, 1e-3, 0.08, "ellipse", False),
    "twomask_r2_l1_z5": ((6, 40, 56), 6, 120, (2.0, 2.0, 0.5), 2, 1, 8, 5.0, 1e-3, 0.08, "two", False),
    "iter1_r2_l1": ((4, 32, 32), 7, 60, (1.0, 1.0, 0.5), 2, 1, 1, 1.0, 1e-3, 0.08, "none", False),
    "r5_l2_big": ((8, 96, 96), 8, 400, (4.0, 4.0, 1.5), 5, 2, 10, 1.0, 1e-3, 0.08, "none", False),
}


def make_motion_cases(ref, out_dir):
    cf3 = ref["calFlow3d_Wei_v1"]
    prep = ref["preprocess"]
    index = {}
    for name, (zyx, seed, nb, md, r, layer, it, zr, tol, spr, mk, use_init) in MOTION_CASES.items():
        tmpl, mov, field = _pair_xyz(zyx, seed, nb, md)
        shape = tmpl.shape
        rng = np.random.default_rng(seed + 1000)
        if mk == "none":
            mref = np.zeros(shape, bool)
            mmov = np.zeros(shape, bool)
        elif mk == "ellipse":
            inc = synthetic.ellipsoid_inclusion(zyx, 0.7).numpy().transpose(2, 1, 0)
            mref = ~inc
            mmov = ~inc
        else:
            mref = np.zeros(shape, bool)
            mref[: shape[0] // 4, :, :] = True
            mmov = rng.uniform(size=shape) > 0.97
        opt_mask = {"mask_ref": mref}
        factor = prep.getSmPnltNormFctr(tmpl.astype(np.float64), opt_mask)
        init = None
        if use_init:
            init = (0.5 * field + rng.normal(scale=0.1, size=field.shape)).astype(np.float32)
        option = {
            "mask_ref": mref.copy(), "mask_mov": mmov.copy(), "layer": layer, "iter": it, "r": r,
            "zRatio": zr, "movRange": 5.0, "motion": init, "smoothPenalty": float(factor * spr),
            "tol": tol, "save_ite": 100,
        }
        motion, err, coords, log = cf3.getMotion(mov.copy(), tmpl.copy(), option)
        warped = cf3.correctMotion(mov.astype(np.float32), motion)
        rec = {
            "mov": mov, "ref": tmpl, "mask_ref": mref, "mask_mov": mmov,
            "motion": motion.astype(np.float32), "warped": warped.astype(np.float32),
            "current_error": np.float64(err), "penalty_factor": np.float64(factor),
        }
        if init is not None:
            rec["motion_init"] = init
        meta = {"layer": layer, "iter": it, "r": r, "zRatio": zr, "movRange": 5.0, "tol": tol,
                "smoothPenalty": float(factor * spr), "smoothPenalty_raw": spr}
        for lk, lv in log.items():
            for key in ("diffError", "penaltyError", "currentError", "max_diff_motion"):
                rec[f"{lk}/{key}"] = np.asarray(lv[key], dtype=np.float64)
        np.savez_compressed(os.path.join(out_dir, f"motion_{name}.npz"), **rec)
        index[name] = meta
        counts = [len(v["currentError"]) for v in log.values()]
        print(f"{name}: shape {shape} error {err:.6f} evals/level {counts}")
    with open(os.path.join(out_dir, "motion_cases.json"), "w") as fh:
        json.dump(index, fh, indent=1, sort_keys=True)


def make_bench_case(ref, out_dir, name):
    import time

    cf3 = ref["calFlow3d_Wei_v1"]
    prep = ref["preprocess"]
    zyx, seed, nb, md, layer, cov, stride = BENCH_CASES[name]
    tmpl, mov, excl, digest = bench_inputs(name)
    factor = prep.getSmPnltNormFctr(tmpl.astype(np.float64), {"mask_ref": excl})
    option = {
        "mask_ref": excl.copy(), "mask_mov": excl.copy(), "layer": layer, "iter": BENCH_ITER, "r": BENCH_R,
        "zRatio": 1.0, "movRange": 5.0, "motion": None, "smoothPenalty": float(factor * BENCH_RAW_PENALTY),
        "tol": 1e-3, "save_ite": 100,
    }
    t0 = time.time()
    motion, err, _, log = cf3.getMotion(mov.copy(), tmpl.copy(), option)
    t1 = time.time()
    warped = cf3.correctMotion(mov.astype(np.float32), motion)
    rec = {
        "sha256": np.asarray(digest), "stride": np.int64(stride),
        "motion_sub": np.ascontiguousarray(motion[::stride, ::stride].astype(np.float32)),
        "warped_sub": np.ascontiguousarray(warped[::stride, ::stride].astype(np.float32)),
        "warped_norm": np.float64(np.linalg.norm(warped.astype(np.float64))),
        "current_error": np.float64(err), "penalty_factor": np.float64(factor),
        "smooth_penalty": np.float64(factor * BENCH_RAW_PENALTY), "reference_seconds": np.float64(t1 - t0),
    }
    for lk, lv in log.items():
        for key in ("diffError", "penaltyError", "currentError", "max_diff_motion"):
            rec[f"{lk}/{key}"] = np.asarray(lv[key], dtype=np.float64)
    np.savez_compressed(os.path.join(out_dir, f"bench_{name}.npz"), **rec)
    counts = [len(v["currentError"]) for v in log.values()]
    print(f"{name}: {t1 - t0:.0f} s, error {err:.6f}, evals/level {counts}", flush=True)


def make_snapshot_case(ref, out_dir):
    """getMotion with save_ite = 2: the error_log snapshots (motion_current,
    data_mov_corrected) of every second iteration and the level images."""
    cf3 = ref["calFlow3d_Wei_v1"]
    prep = ref["preprocess"]
    zyx = (6, 48, 56)
    tmpl, mov, _ = _pair_xyz(zyx, 41, 150, (2.5, 2.5, 0.8))
    excl = np.ascontiguousarray(~synthetic.ellipsoid_inclusion(zyx, 0.8).numpy().transpose(2, 1, 0))
    factor = prep.getSmPnltNormFctr(tmpl.astype(np.float64), {"mask_ref": excl})
    option = {"mask_ref": excl.copy(), "mask_mov": excl.copy(), "layer": 1, "iter": 6, "r": 3, "zRatio": 1.0,
              "movRange": 5.0, "motion": None, "smoothPenalty": float(factor * 0.08), "tol": 1e-3, "save_ite": 2}
    motion, err, _, log = cf3.getMotion(mov.copy(), tmpl.copy(), option)
    rec = {"mov": mov, "ref": tmpl, "excl": excl, "motion": motion.astype(np.float32),
           "smooth_penalty": np.float64(factor * 0.08)}
    for lk, lv in log.items():
        rec[f"{lk}/currentError"] = np.asarray(lv["currentError"], np.float64)
        rec[f"{lk}/motion_current"] = np.stack([np.asarray(a, np.float32) for a in lv["motion_current"]])
        rec[f"{lk}/data_mov_corrected"] = np.stack([np.asarray(a, np.float32) for a in lv["data_mov_corrected"]])
        rec[f"{lk}/data_ref"] = np.asarray(lv["data_ref"], np.float32)
        rec[f"{lk}/data_mov"] = np.asarray(lv["data_mov"], np.float32)
        print(f"snapshots {lk}: evals {len(lv['currentError'])}, snapshots {len(lv['motion_current'])}")
    np.savez_compressed(os.path.join(out_dir, "snapshots.npz"), **rec)


def make_primitive_cases(ref, out_dir):
    imr = ref["imresize"]
    cf3 = ref["calFlow3d_Wei_v1"]
    calc = ref["calculate"]
    rng = np.random.default_rng(123)
    rec = {}
    vol = rng.uniform(0, 4000, (37, 50, 5))
    rec["resize_in"] = vol
    for i, shp in enumerate([(18, 25, 5), (9, 12, 5), (4, 6, 5), (37, 50, 5)]):
        rec[f"resize_bicubic_{i}"] = imr.imresize(vol, output_shape=shp)
    u16 = rng.integers(0, 65535, (33, 20, 4)).astype(np.uint16)
    rec["resize_u16_in"] = u16
    rec["resize_u16_out"] = imr.imresize(u16, output_shape=(16, 10, 4))
    u8 = rng.integers(0, 255, (21, 18, 3)).astype(np.uint8)
    rec["resize_u8_in"] = u8
    rec["resize_u8_out"] = imr.imresize(u8, output_shape=(10, 9, 3))
    fld = rng.normal(size=(18, 25, 5)).astype(np.float32)
    rec["resize_bilinear_in"] = fld
    rec["resize_bilinear_out"] = imr.imresize(fld, output_shape=(37, 50, 5), method="bilinear")
    mask = np.zeros((40, 36, 4), np.float32)
    mask[10:25, 5:20, :] = 1
    rec["resize_mask_in"] = mask
    rec["resize_mask_out"] = imr.imresize(mask, output_shape=(10, 9, 4))

    data = rng.uniform(0, 1000, (40, 32, 6)).astype(np.float32)
    motion = (rng.normal(size=(40, 32, 6, 3)) * 2.5).astype(np.float32)
    motion[0, 0, 0] = (-50, 3, 2)
    motion[-1, -1, -1] = (40, -60, 9)
    rec["warp_in"] = data
    rec["warp_motion"] = motion
    rec["warp_out"] = cf3.correctMotion(data, motion)

    comps = [rng.normal(size=(5, 4, 3)) for _ in range(9)]
    spd = np.abs(rng.normal(size=(5, 4, 3))) * 3
    comps[0] = comps[0] ** 2 + spd
    comps[3] = comps[3] ** 2 + spd
    comps[5] = comps[5] ** 2 + spd
    nei = rng.normal(size=(5, 4, 3, 3)).astype(np.float32)
    for i, c in enumerate(comps):
        rec[f"solve_in_{i}"] = c.copy()
    rec["solve_nei"] = nei
    rec["solve_out"] = cf3.getFlow3_withPenalty6(*[c.copy() for c in comps], 0.7, nei)
    cpm = rng.normal(size=(6, 5, 4, 3)).astype(np.float32)
    rec["neidiff_in"] = cpm
    rec["neidiff_out"] = cf3.getNeiDiff(cpm, 1)
    a = rng.normal(size=(9, 7, 3))
    rec["box_in"] = a
    rec["box_out_5x3"] = calc.imfilter(a, np.ones((5, 3, 1)), "replicate", "same", "corr")
    np.savez_compressed(os.path.join(out_dir, "primitives.npz"), **rec)
    print("primitives written")


class _RegionProps:
    def __init__(self, coords):
        self.coords = coords
        self.area = len(coords)


def _skimage_standin():
    """scikit-image (>= 0.21, the reference's pyproject.toml:21) is not
    installed here.  The reference's mask module is run with these stand-ins,
    which restate the four functions it calls from their documented
    semantics: binary_erosion = ndimage.binary_erosion(border_value=1),
    binary_dilation = ndimage.binary_dilation(border_value=0), binary_opening
    = dilation of the erosion, label(connectivity=ndim) = ndimage.label with a
    full 3x3x3 structure, regionprops = area and coordinates per label."""
    from scipy import ndimage

    morph = types.ModuleType("skimage.morphology")
    measure = types.ModuleType("skimage.measure")

    def binary_erosion(image, footprint):
        return ndimage.binary_erosion(image, structure=footprint, border_value=1)

    def binary_dilation(image, footprint):
        return ndimage.binary_dilation(image, structure=footprint, border_value=0)

    def binary_opening(image, footprint):
        return binary_dilation(binary_erosion(image, footprint), footprint)

    def label(vol, connectivity):
        st = ndimage.generate_binary_structure(vol.ndim, connectivity)
        return ndimage.label(vol, structure=st)[0]

    def regionprops(lab):
        return [_RegionProps(np.argwhere(lab == k)) for k in range(1, int(lab.max()) + 1)]

    morph.binary_dilation, morph.binary_opening = binary_dilation, binary_opening
    measure.label, measure.regionprops = label, regionprops
    pkg = types.ModuleType("skimage")
    pkg.morphology, pkg.measure = morph, measure
    return {"skimage": pkg, "skimage.morphology": morph, "skimage.measure": measure}


# name: (x, y, z) shape, seed, background, outlier blobs, thresFactor, maskRange
MASK_CASES = {
    "mask_a": ((66, 70, 6), 11, 100.0, 12, 3.0, (5, 5000)),
    "mask_b": ((40, 56, 6), 12, 300.0, 6, 2.5, (20, 400)),
    "mask_c": ((96, 96, 8), 13, 50.0, 30, 4.0, (1, 10 ** 9)),
}


def make_mask_cases(root, out_dir):
    try:
        import skimage  # noqa: F401
    except ImportError:
        sys.modules.update(_skimage_standin())
    src = os.path.join(root, "src", "wholistic_registration")
    if "wholistic_registration" not in sys.modules:
        pkg = types.ModuleType("wholistic_registration")
        pkg.__path__ = [src]
        sys.modules["wholistic_registration"] = pkg
    mask = importlib.import_module("wholistic_registration.utils.mask")
    prep = importlib.import_module("wholistic_registration.utils.preprocess")
    rec = {}
    for name, (shape, seed, bg, nblob, thres, rng_) in MASK_CASES.items():
        rng = np.random.default_rng(seed)
        vol = rng.poisson(bg, size=shape).astype(np.float64)
        for _ in range(nblob):
            c = [rng.integers(0, s) for s in shape]
            rad = rng.integers(1, 4)
            amp = rng.uniform(3, 20) * np.sqrt(bg) * rng.choice([-1, 1])
            sl = tuple(slice(max(0, ci - rad), min(s, ci + rad + 1)) for ci, s in zip(c, shape))
            vol[sl] += amp
        vol = np.clip(vol, 0, 65535).astype(np.uint16)
        m = mask.getMask(vol, thres)
        f = mask.bwareafilt3_wei(m, list(rng_))
        mu, sg = prep.robust_mean_std(vol.astype(np.float32))
        rec[f"{name}_vol"] = vol
        rec[f"{name}_mask"] = m
        rec[f"{name}_filtered"] = f
        rec[f"{name}_params"] = np.array([thres, rng_[0], rng_[1]], np.float64)
        rec[f"{name}_musig"] = np.array([mu, sg], np.float32)
    np.savez_compressed(os.path.join(out_dir, "masks.npz"), **rec)
    print("masks written")


# name: mov (x, y, z), ref (x, y, z), zRatio, zRatio_HR, r, layer, iter, tol, smoothPenalty, masks, init
XRES_CASES = {
    "xr_small_r3_l1": ((40, 48, 6), (40, 48, 9), 3.0, 2.0, 3, 1, 6, 1e-3, 0.05, False, False),
    "xr_mask_r2_l1": ((48, 40, 5), (48, 40, 10), 2.0, 1.0, 2, 1, 8, 1e-3, 0.05, True, False),
    "xr_init_r4_l2": ((64, 56, 4), (64, 56, 8), 4.0, 2.0, 4, 2, 8, 1e-4, 0.02, False, True),
    "xr_ragged_r3_l2": ((70, 66, 6), (70, 66, 12), 2.5, 1.25, 3, 2, 10, 1e-3, 0.05, True, False),
    "xr_iter1_r2_l1": ((32, 32, 4), (32, 32, 4), 1.0, 1.0, 2, 1, 1, 1e-3, 0.05, False, False),
    "xr_refwide_r2_l1": ((40, 40, 5), (48, 44, 10), 2.0, 1.0, 2, 1, 8, 1e-3, 0.05, True, False),
    "xr_z1_r3_l1": ((44, 40, 1), (44, 40, 3), 3.0, 1.0, 3, 1, 8, 1e-3, 0.05, False, False),
    "xr_refz1_r2_l0": ((36, 36, 4), (36, 36, 1), 1.0, 4.0, 2, 0, 6, 1e-3, 0.05, True, False),
    "xr_phase_r3_l1": ((48, 44, 5), (48, 44, 10), 2.0, 1.0, 3, 1, 8, 1e-3, 0.05, False, "phase"),
}


# cases re-run with wrong_region_enable=True (accepted and rejected corrections,
# a low valid ratio, an empty trap mask)
XRES_WR_CASES = ("xr_mask_r2_l1", "xr_small_r3_l1", "xr_init_r4_l2", "xr_ragged_r3_l2", "xr_refz1_r2_l0",
                 "xr_z1_r3_l1", "xr_phase_r3_l1")


# cases re-run with wrong_region_exclude_mode="highresidual" (the trap seeded
# only by the bad voxels whose error dropped most); q 0.8 is the default
XRES_HR_CASES = {"xr_mask_r2_l1": 0.8, "xr_small_r3_l1": 0.8, "xr_ragged_r3_l2": 0.5, "xr_phase_r3_l1": 0.8}


# cases re-run with non-default wrong-region options (metric, thresholds,
# radii, no Gaussian smoothing)
XRES_OPT_CASES = {
    "xr_mask_r2_l1": {"wrong_region_metric": "mae", "wrong_region_mad_threshold": 2.5,
                      "wrong_region_min_component_size": 3, "expand_radius_xy": 3.0, "intensity_k": 1.5},
    "xr_small_r3_l1": {"sigma_grad": 0.0, "expand_radius_xy": 1.0, "wrong_region_mad_threshold": 2.0},
    "xr_ragged_r3_l2": {"wrong_region_metric": "mae", "sigma_grad": 1.6, "wrong_region_min_component_size": 1},
}


def xres_pair(mov_shape, ref_shape, zr, zr_hr, seed):
    """Moving and reference stacks of one blob field sampled at z spacings zr
    and zr_hr (physical units per z index), the moving one displaced by a
    smooth field and Poisson-noised.  (x, y, z) layout, float32."""
    rng = np.random.default_rng(seed)
    n_blobs = max(20, mov_shape[0] * mov_shape[1] // 12)
    zphys = max(mov_shape[2] * zr, ref_shape[2] * zr_hr)
    cx = rng.uniform(0, max(mov_shape[0], ref_shape[0]), n_blobs)
    cy = rng.uniform(0, max(mov_shape[1], ref_shape[1]), n_blobs)
    cz = rng.uniform(0, zphys, n_blobs)
    amp = rng.uniform(50, 400, n_blobs)
    sig = rng.uniform(1.5, 3.0, n_blobs)

    def render(shape, zs, dx=0.0, dy=0.0, dz=0.0):
        X, Y, Z = np.meshgrid(np.arange(shape[0], dtype=np.float64), np.arange(shape[1], dtype=np.float64),
                              np.arange(shape[2], dtype=np.float64) * zs, indexing="ij")
        X, Y, Z = X + dx, Y + dy, Z + dz
        out = np.full(shape, 100.0)
        for i in range(n_blobs):
            out += amp[i] * np.exp(-((X - cx[i]) ** 2 + (Y - cy[i]) ** 2 + ((Z - cz[i]) / 1.5) ** 2) / (2 * sig[i] ** 2))
        return out

    X, Y, Z = np.meshgrid(*[np.arange(n, dtype=np.float64) for n in mov_shape], indexing="ij")
    dx = 1.2 * np.sin(2 * np.pi * Y / 37.0 + 0.3) + 0.5
    dy = 1.0 * np.cos(2 * np.pi * X / 41.0) - 0.4
    dz = 0.6 * np.sin(2 * np.pi * (X + Y) / 53.0)
    ref = render(ref_shape, zr_hr)
    mov = render(mov_shape, zr, dx, dy, dz)
    mov = rng.poisson(np.clip(mov, 0, None)).astype(np.float32)
    ref = rng.poisson(np.clip(ref, 0, None)).astype(np.float32)
    return mov, ref


def make_xres_cases(root, out_dir):
    src = os.path.join(root, "src", "wholistic_registration")
    if "wholistic_registration" not in sys.modules:
        pkg = types.ModuleType("wholistic_registration")
        pkg.__path__ = [src]
        sys.modules["wholistic_registration"] = pkg
    cf = importlib.import_module("wholistic_registration.utils.calFlowCrossResolution")
    index = {}
    for i, (name, (ms, rs, zr, zrh, r, layer, it, tol, sp, masks, use_init)) in enumerate(XRES_CASES.items()):
        mov, ref = xres_pair(ms, rs, zr, zrh, 100 + i)
        rng = np.random.default_rng(200 + i)
        mmov = np.zeros(ms, np.uint8)
        mref = np.zeros(rs, np.uint8)
        if masks:
            mmov[: ms[0] // 6, : ms[1] // 5, :] = 1
            X, Y, Z = np.meshgrid(*[np.arange(n) for n in rs], indexing="ij")
            mref[((X - 0.7 * rs[0]) / (0.2 * rs[0])) ** 2 + ((Y - 0.6 * rs[1]) / (0.25 * rs[1])) ** 2 < 1] = 1
        init = None
        phase0 = None
        if use_init == "phase":
            # an initial phase: the default map shifted by a smooth field in x and z
            X, Y, Z = np.meshgrid(*[np.arange(n, dtype=np.float64) for n in ms], indexing="ij")
            phase0 = np.stack([X + 0.6 * np.sin(Y / 8.0), Y - 0.3, Z * zr / zrh + 0.2 * np.cos(X / 11.0)],
                              -1).astype(np.float32)
        elif use_init:
            X, Y, Z = np.meshgrid(*[np.arange(n, dtype=np.float64) for n in ms], indexing="ij")
            init = np.stack([0.4 * np.sin(X / 9.0), 0.3 * np.cos(Y / 7.0), 0.1 + 0 * Z], -1).astype(np.float32)
            init += rng.normal(scale=0.05, size=init.shape).astype(np.float32)
        option = {"mask_ref": mref.copy(), "mask_mov": mmov.copy(), "layer": layer, "iter": it, "r": r,
                  "zRatio": zr, "zRatio_HR": zrh, "smoothPenalty": sp, "movRange": 5.0, "tol": tol,
                  "motion": init, "wrong_region_enable": False}
        if phase0 is not None:
            option["phase"] = phase0
        phase, motion, sampled = cf.getMotion_v2(mov.copy(), ref.copy(), option)
        rec = {"mov": mov, "ref": ref, "mask_mov": mmov, "mask_ref": mref, "phase": np.asarray(phase, np.float32),
               "motion": np.asarray(motion, np.float32), "ref_sampled": np.asarray(sampled, np.float64)}
        if init is not None:
            rec["motion_init"] = init
        if phase0 is not None:
            rec["phase_init"] = phase0
        np.savez_compressed(os.path.join(out_dir, f"xres_{name}.npz"), **rec)
        index[name] = {"layer": layer, "iter": it, "r": r, "zRatio": zr, "zRatio_HR": zrh, "tol": tol,
                       "smoothPenalty": sp, "movRange": 5.0}
        print(f"{name}: mov {ms} ref {rs} max |motion| {float(np.abs(motion).max()):.3f}")
    with open(os.path.join(out_dir, "xres_cases.json"), "w") as fh:
        json.dump(index, fh, indent=1, sort_keys=True)
    # the same inputs with the wrong-region correction on (the reference's default)
    for name in XRES_WR_CASES:
        d = dict(np.load(os.path.join(out_dir, f"xres_{name}.npz")))
        meta = index[name]
        option = dict(meta)
        option.update({"mask_ref": d["mask_ref"].copy(), "mask_mov": d["mask_mov"].copy(),
                       "motion": d.get("motion_init"), "wrong_region_enable": True})
        if "phase_init" in d:
            option["phase"] = d["phase_init"]
        phase, motion, sampled = cf.getMotion_v2(d["mov"].copy(), d["ref"].copy(), option)
        np.savez_compressed(os.path.join(out_dir, f"xreswr_{name}.npz"), phase=np.asarray(phase, np.float32),
                            motion=np.asarray(motion, np.float32), ref_sampled=np.asarray(sampled, np.float64))
        print(f"{name} (wrong-region correction on): max |motion| {float(np.abs(motion).max()):.3f}")
    make_xres_hr_cases(cf, out_dir)
    make_xres_opt_cases(cf, out_dir)


# compute_reference_from_block (utils/reference.py:102-124): (dual_channel, k, function)
REFBLOCK_CASES = {"single": (False, 0.0, "raw"), "dual_sqrt": (True, 0.5, "sqrt"), "dual_log2": (True, 2.0, "log2"),
                  "dual_k0": (True, 0.0, "raw")}


def make_reference_block_cases(root, out_dir):
    """A block of 12 uint16 [T, Z, Y, X] frames (a blob volume, per-frame
    Poisson noise and drift, four frames strongly displaced) and its calcium
    channel, through the reference's compute_reference_from_block."""
    src = os.path.join(root, "src", "wholistic_registration")
    if "wholistic_registration" not in sys.modules:
        pkg = types.ModuleType("wholistic_registration")
        pkg.__path__ = [src]
        sys.modules["wholistic_registration"] = pkg
    rf = importlib.import_module("wholistic_registration.utils.reference")
    rng = np.random.default_rng(321)
    T, Z, Y, X = 12, 5, 40, 36
    Zg, Yg, Xg = np.meshgrid(np.arange(Z), np.arange(Y), np.arange(X), indexing="ij")
    cy, cx, amp = rng.uniform(0, Y, 25), rng.uniform(0, X, 25), rng.uniform(200, 900, 25)

    def vol(dy, dx):
        out = np.full((Z, Y, X), 120.0)
        for i in range(25):
            out += amp[i] * np.exp(-((Yg - cy[i] - dy) ** 2 + (Xg - cx[i] - dx) ** 2) / 18.0) * (1 + 0.1 * Zg)
        return out

    mem = np.stack([rng.poisson(vol(0.3 * t if t < 8 else 6.0, 0.2 * t if t < 8 else -5.0)) for t in range(T)])
    mem = mem.astype(np.uint16)
    ca = rng.poisson(np.broadcast_to(vol(0.0, 0.0) * 0.3, (T, Z, Y, X))).astype(np.uint16)
    rec = {"mem": mem, "ca": ca}
    for name, (dual, k, fn) in REFBLOCK_CASES.items():
        config = {"channels": {"k": k, "function": fn, "dual_channel": dual}}
        ref, idx = rf.compute_reference_from_block(mem.copy(), config, ca.copy() if dual else None)
        rec[f"{name}_ref"], rec[f"{name}_idx"] = np.asarray(ref, np.float64), np.asarray(idx, np.int64)
        rec[f"{name}_params"] = np.array([float(dual), k], np.float64)
        rec[f"{name}_function"] = np.array(fn)
        print(f"reference block {name}: indices {list(np.asarray(idx))}")
    # float32 frames (non-integer values): the reference's mean keeps float32
    mem32 = (mem.astype(np.float32) * np.float32(0.37)).astype(np.float32)
    ca32 = (ca.astype(np.float32) * np.float32(1.13)).astype(np.float32)
    rec["mem_f32"], rec["ca_f32"] = mem32, ca32
    for name, (dual, k, fn) in REFBLOCK_CASES.items():
        config = {"channels": {"k": k, "function": fn, "dual_channel": dual}}
        ref, idx = rf.compute_reference_from_block(mem32.copy(), config, ca32.copy() if dual else None)
        rec[f"f32_{name}_ref"], rec[f"f32_{name}_idx"] = np.asarray(ref), np.asarray(idx, np.int64)
        print(f"reference block f32 {name}: dtype {np.asarray(ref).dtype}, indices {list(np.asarray(idx))}")
    np.savez_compressed(os.path.join(out_dir, "reference_block.npz"), **rec)


# Per-batch wrappers (utils/registration.py:41-189 and :192-352) run through
# the reference itself.  name: (wrapper, config overrides, given reference,
# dual channel, motion_init)
WRAPPER_CASES = {
    "w3d_auto": ("3d", {}, False, False, False),
    "w3d_dual_sqrt": ("3d", {"channels": {"dual_channel": True, "k": 0.5, "function": "sqrt"}}, False, True, False),
    "w3d_given_init": ("3d", {"reference": {"pick_reference_auto": False}}, True, False, True),
    "w2d_auto": ("2d", {}, False, False, False),
    "w2d_dual_log2": ("2d", {"channels": {"dual_channel": True, "k": 2.0, "function": "log2"}}, False, True, False),
}


def wrapper_config(overrides):
    """The config dict of a wrapper case (the reference reads it as TOML)."""
    cfg = {
        "reference": {"pick_reference_auto": True, "chunk_size": 2},
        "channels": {"dual_channel": False, "k": 0.0, "function": "raw"},
        "mask": {"maskRange": [5, 5000], "thresFactor": 3.0},
        "pyramid": {"r": 3, "layer": 1, "iter": 6, "smoothPenalty": 0.08, "tolerance": 1e-3},
        "MetaData": {"zRatio": 2.0},
    }
    for sec, kv in overrides.items():
        cfg[sec] = dict(cfg[sec], **kv)
    return cfg


def wrapper_inputs(kind, seed):
    """(membrane, calcium, reference, motion_init): uint16 [T, Z, Y, X] (3d)
    or [T, Y, X] (2d) frames of a blob volume under small smooth shifts, with
    a few bright outlier spots for the masks, and the calcium channel."""
    rng = np.random.default_rng(seed)
    zyx = (6, 56, 64) if kind == "3d" else (1, 60, 68)
    T = 3
    tmpl, _, _ = synthetic.make_pair(zyx, seed, n_blobs=160, max_disp=(1.0, 1.0, 0.3), noise=False)
    base = tmpl.numpy().astype(np.float64)
    mem, ca = [], []
    for t in range(T):
        _, mov, _ = synthetic.make_pair(zyx, seed + 10 + t, max_disp=(2.0, 2.0, 0.5 if kind == "3d" else 0.0),
                                        template=torch_from(base), noise=False)
        v = mov.numpy().astype(np.float64)
        spots = rng.integers(0, np.array(zyx), size=(3, 3))
        for z, y, x in spots:
            v[z, max(0, y - 1):y + 2, max(0, x - 1):x + 2] += 20000.0
        mem.append(rng.poisson(v))
        ca.append(rng.poisson(0.3 * v + 50.0))
    mem = np.clip(np.asarray(mem), 0, 65535).astype(np.uint16)
    ca = np.clip(np.asarray(ca), 0, 65535).astype(np.uint16)
    ref = mem.astype(np.float64).mean(axis=0)
    init = rng.normal(scale=0.3, size=zyx + (3,)).astype(np.float32)
    if kind == "2d":
        mem, ca, ref, init = mem[:, 0], ca[:, 0], ref[0], init[0, :, :, :]
    return mem, ca, ref, init


def torch_from(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a, np.float32))


def make_wrapper_cases(root, out_dir):
    import tempfile

    import toml

    try:
        import skimage  # noqa: F401
    except ImportError:
        sys.modules.update(_skimage_standin())
    load_reference(root)
    reg = importlib.import_module("wholistic_registration.utils.registration")
    rec = {}
    for i, (name, (kind, over, given, dual, use_init)) in enumerate(WRAPPER_CASES.items()):
        cfg = wrapper_config(over)
        mem, ca, ref, init = wrapper_inputs(kind, 500 + i)
        with tempfile.NamedTemporaryFile("w", suffix=".toml", delete=False) as fh:
            toml.dump(cfg, fh)
            path = fh.name
        fn = reg.wbi_registration_3d if kind == "3d" else reg.wbi_registration_2d
        out = fn(mem.copy(), path, reference_image=ref.copy() if given else None,
                 motion_init=(init.copy() if use_init else None), verbose=False,
                 moving_Ca_image=ca.copy() if dual else None)
        os.unlink(path)
        mem_out, ca_out, dat_ref, errors, motion_out = out
        rec[f"{name}/mem"], rec[f"{name}/ca"], rec[f"{name}/ref"], rec[f"{name}/init"] = mem, ca, ref, init
        rec[f"{name}/mem_out"] = np.asarray(mem_out, np.float32)
        rec[f"{name}/ca_out"] = np.asarray(ca_out, np.float32)
        rec[f"{name}/dat_ref"] = np.asarray(dat_ref)
        rec[f"{name}/motion_out"] = np.asarray(motion_out, np.float32)
        rec[f"{name}/initial_error"] = np.array([e["initial_error"] for e in errors], np.float64)
        rec[f"{name}/eventual_error"] = np.array([e["eventual_error"] for e in errors], np.float64)
        rec[f"{name}/config"] = np.array(json.dumps(cfg))
        print(f"{name}: motion {np.asarray(motion_out).shape}, max |m| {np.abs(motion_out).max():.3f}, "
              f"errors {[round(float(e['eventual_error']), 3) for e in errors]}", flush=True)
    np.savez_compressed(os.path.join(out_dir, "wrappers.npz"), **rec)


def make_xres_opt_cases(cf, out_dir):
    """xres cases re-run with the wrong-region correction at non-default options."""
    with open(os.path.join(out_dir, "xres_cases.json")) as fh:
        index = json.load(fh)
    for name, extra in XRES_OPT_CASES.items():
        d = dict(np.load(os.path.join(out_dir, f"xres_{name}.npz")))
        option = dict(index[name])
        option.update({"mask_ref": d["mask_ref"].copy(), "mask_mov": d["mask_mov"].copy(),
                       "motion": d.get("motion_init"), "wrong_region_enable": True})
        option.update(extra)
        if "phase_init" in d:
            option["phase"] = d["phase_init"]
        phase, motion, sampled = cf.getMotion_v2(d["mov"].copy(), d["ref"].copy(), option)
        np.savez_compressed(os.path.join(out_dir, f"xresopt_{name}.npz"), phase=np.asarray(phase, np.float32),
                            motion=np.asarray(motion, np.float32), ref_sampled=np.asarray(sampled, np.float64),
                            options=np.array(json.dumps(extra, sort_keys=True)))
        print(f"{name} (wrong-region options {extra}): max |motion| {float(np.abs(motion).max()):.3f}")


def make_xres_hr_cases(cf, out_dir):
    """xres cases re-run with the "highresidual" exclusion mode."""
    with open(os.path.join(out_dir, "xres_cases.json")) as fh:
        index = json.load(fh)
    for name, q in XRES_HR_CASES.items():
        d = dict(np.load(os.path.join(out_dir, f"xres_{name}.npz")))
        option = dict(index[name])
        option.update({"mask_ref": d["mask_ref"].copy(), "mask_mov": d["mask_mov"].copy(),
                       "motion": d.get("motion_init"), "wrong_region_enable": True,
                       "wrong_region_exclude_mode": "highresidual", "quantile_threshold_q": q})
        if "phase_init" in d:
            option["phase"] = d["phase_init"]
        phase, motion, sampled = cf.getMotion_v2(d["mov"].copy(), d["ref"].copy(), option)
        np.savez_compressed(os.path.join(out_dir, f"xreshr_{name}.npz"), phase=np.asarray(phase, np.float32),
                            motion=np.asarray(motion, np.float32), ref_sampled=np.asarray(sampled, np.float64),
                            quantile_q=np.float64(q))
        print(f"{name} (highresidual exclusion, q {q}): max |motion| {float(np.abs(motion).max()):.3f}")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("WR_REFERENCE_ROOT"),
                    help="root of the reference checkout (default: $WR_REFERENCE_ROOT)")
    ap.add_argument("--only", choices=["primitives", "motion", "masks", "xres", "xreshr", "xresopt", "refblock",
                                       "bench", "wrappers", "snapshots"], default=None)
    ap.add_argument("--case", default=None, help="with --only bench: one case of BENCH_CASES")
    args = ap.parse_args()
    if not args.ref:
        ap.error("the reference root is required (--ref or WR_REFERENCE_ROOT)")
    if args.only == "snapshots":
        make_snapshot_case(load_reference(args.ref), HERE)
        return
    if args.only == "wrappers":
        make_wrapper_cases(args.ref, HERE)
        return
    if args.only == "bench":
        ref = load_reference(args.ref)
        for name in ([args.case] if args.case else BENCH_CASES):
            make_bench_case(ref, HERE, name)
        return
    if args.only in (None, "masks"):
        make_mask_cases(args.ref, HERE)
    if args.only in (None, "xres"):
        make_xres_cases(args.ref, HERE)
    if args.only in (None, "refblock"):
        make_reference_block_cases(args.ref, HERE)
    if args.only == "refblock":
        return
    if args.only in ("xreshr", "xresopt"):
        src = os.path.join(args.ref, "src", "wholistic_registration")
        if "wholistic_registration" not in sys.modules:
            pkg = types.ModuleType("wholistic_registration")
            pkg.__path__ = [src]
            sys.modules["wholistic_registration"] = pkg
        cf = importlib.import_module("wholistic_registration.utils.calFlowCrossResolution")
        (make_xres_hr_cases if args.only == "xreshr" else make_xres_opt_cases)(cf, HERE)
    if args.only in ("masks", "xres", "xreshr", "xresopt"):
        return
    ref = load_reference(args.ref)
    if args.only in (None, "primitives"):
        make_primitive_cases(ref, HERE)
    if args.only in (None, "motion"):
        make_motion_cases(ref, HERE)


if __name__ == "__main__":
    main()
