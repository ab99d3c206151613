"""CPU oracle for the cross-resolution registration ``getMotion_v2``.

TEST INFRASTRUCTURE ONLY.  This module checks the product: only ``tests/`` may
import it.  The product path (``wholistic_registration_b200``) never calls
into it and fails loudly when its CUDA library is missing.

It restates, in NumPy, the reference's cross-resolution path, with and
without its wrong-region correction; paths are relative to
``src/wholistic_registration``:

* ``utils/calFlowCrossResolution.py:2470-2663``  ``getMotion_v2``: pyramid of
  the moving stack on its grid and of the reference stack on its own
  (cross-resolution) grid
* ``utils/calFlowCrossResolution.py:2031-2237``  ``optimize_layer_cross_resolution``
* ``utils/calFlowCrossResolution.py:1904-2028``  phase composition, mask
  resampling (threshold 0.5), motion / phase initialisation (``option["phase"]``
  included), CP grid, valid mask
* ``utils/calFlowCrossResolution.py:463-478, 1144-1154``  the continuous
  reference ``H``: ``map_coordinates(order=3, mode="nearest")``
* ``utils/calFlowCrossResolution.py:1190-1900, 2240-2467``  the wrong-region
  correction: CP errors, outlier regions, the trap mask in reference space,
  the two re-runs and the keep / discard choice, in both exclusion modes
  ("direct" and "highresidual") and at non-default options; pinned to
  fourteen runs of the reference
* ``utils/calFlowCrossResolution.py:480-660, 700-1141``  the two projection
  splats, pinned to fixtures of the reference's own kernels
* ``utils/calFlowCrossResolution.py:41-272``  neighbour difference, error,
  gradients, 3x3 solve and CP grid interpolation, the same functions as
  ``calFlow3d_Wei_v1.py`` (restated in ``oracle.lk_oracle``)

The cubic-spline sampler is the library call the reference makes:
``scipy.ndimage.map_coordinates`` (SciPy 1.18.1 here; CuPy's
``cupyx.scipy.ndimage.map_coordinates`` implements the same algorithm).
``bspline_coefficients`` / ``cubic_sample`` restate that algorithm (edge
padding by 12, recursive cubic B-spline prefilter, 64-tap evaluation) the way
the CUDA path computes it; ``tests/test_oracle_golden.py`` checks them against
SciPy.

Arrays use the reference's internal (x, y, z) layout.  Parity is pinned
against fixtures made by running the reference itself
(``tests/golden/make_golden.py --only xres``).

``project_max`` / ``project_weighted`` restate the reference's two
fixed-plane projection kernels (``_PROJECT_TO_PLANES_NANMAX_SRC`` and
``_PROJECT_TO_PLANES_WEIGHTED_AVG_SRC``, :480-660) and their wrappers
(:700-1141).  Those exist only as CuPy RawKernels, which cannot run here:
parity unpinned for the projections (the restatement follows the kernel
source line by line; no reference output exists to pin it).
"""

from __future__ import annotations

import numpy as np
from scipy import ndimage

from .lk_oracle import (
    _grid,
    _window_sums_segmented,
    cal_error,
    get_nei_diff,
    imresize,
    solve_flow_with_penalty,
    spatial_gradient,
    trilinear,
)

__all__ = ["cubic_sample_scipy", "bspline_coefficients", "cubic_sample", "get_motion_v2", "SPLINE_PAD",
           "project_max", "project_weighted", "make_ball", "local_cp_error", "bad_region_mask", "trap_mask"]

SPLINE_PAD = 12                       # SciPy's edge padding before the prefilter (mode "nearest")
_Z1 = float(np.sqrt(3.0) - 2.0)       # pole of the cubic B-spline prefilter


def cubic_sample_scipy(vol, px, py, pz):
    """``H(coords)`` of calFlowCrossResolution.py:463-478 (zRatio = 1): cubic
    spline of ``vol`` at (px, py, pz), mode "nearest"; output dtype = vol's."""
    coords = np.stack([np.asarray(px, np.float64).ravel(), np.asarray(py, np.float64).ravel(),
                       np.asarray(pz, np.float64).ravel()])
    out = ndimage.map_coordinates(np.asarray(vol), coords, order=3, mode="nearest")
    return out.reshape(np.shape(px))


def _prefilter_line(s):
    """Cubic B-spline coefficients of one line (gain 6, causal then
    anti-causal recursion with pole sqrt(3) - 2), initialised for a constant
    continuation of the line beyond both ends."""
    c = np.asarray(s, dtype=np.float64) * 6.0
    n = c.shape[0]
    z = _Z1
    c[0] = c[0] / (1.0 - z)
    for k in range(1, n):
        c[k] = c[k] + z * c[k - 1]
    se = 6.0 * float(s[n - 1])
    c[n - 1] = -z * (se / (1.0 - z) ** 2 + (c[n - 1] - se / (1.0 - z)) / (1.0 - z * z))
    for k in range(n - 2, -1, -1):
        c[k] = z * (c[k + 1] - c[k])
    return c


def bspline_coefficients(vol):
    """Coefficients of the edge-padded volume (SPLINE_PAD on every side)."""
    p = np.pad(np.asarray(vol, np.float64), SPLINE_PAD, mode="edge")
    for ax in range(3):
        p = np.apply_along_axis(_prefilter_line, ax, p)
    return p


def _bspline_weights(t):
    return ((1 - t) ** 3 / 6, (3 * t ** 3 - 6 * t ** 2 + 4) / 6, (-3 * t ** 3 + 3 * t ** 2 + 3 * t + 1) / 6, t ** 3 / 6)


def cubic_sample(coef, px, py, pz):
    """64-tap cubic B-spline evaluation of padded coefficients at (px, py, pz)
    given in the unpadded index space; coordinates are clamped to the padded
    extent and taps to the padded array."""
    n = coef.shape
    taps, wts = [], []
    for d, c in enumerate((px, py, pz)):
        c = np.clip(np.asarray(c, np.float64) + SPLINE_PAD, 0.0, n[d] - 1)
        f = np.floor(c)
        t = c - f
        i0 = f.astype(np.int64) - 1
        taps.append([np.clip(i0 + k, 0, n[d] - 1) for k in range(4)])
        wts.append(_bspline_weights(t))
    out = np.zeros(np.shape(px), np.float64)
    for a in range(4):
        for b in range(4):
            for e in range(4):
                out += wts[0][a] * wts[1][b] * wts[2][e] * coef[taps[0][a], taps[1][b], taps[2][e]]
    return out


def _optimize_layer(mov_l, ref_l, mask_mov_l, mask_ref_f, phase_cur, motion, r, n_iter, sps, mov_range, tol,
                    zratio_hr, lg, forced=None, noise=None):
    """optimize_layer_cross_resolution (calFlowCrossResolution.py:2031-2237).

    ``mask_ref_f``: the reference-grid exclusion mask (float32 0/1) read
    through its spline; ``motion``: the initial field (copied).  Returns the
    final motion, phase, sampled reference, smoothed masked residual, valid
    mask and the final recompute's error (its neighbour difference is not
    z-scaled, as in the reference).  ``noise = (window (rng, rel), sample (rng,
    rel))`` perturbs window sums / spline samples (see get_motion_v2)."""
    motion = motion.copy()
    x, y, z = mov_l.shape
    xg = np.arange(r, x - 1, 2 * r + 1)
    yg = np.arange(r, y - 1, 2 * r + 1)
    ncx, ncy = len(xg), len(yg)
    grid = _grid(mov_l.shape)
    box3 = np.ones((3, 3, 1), dtype=np.float32) / 9
    old_error = np.inf * np.ones(3, dtype=np.float32)
    wnoise, snoise = noise if noise is not None else (None, None)
    n_updates = 0

    def evaluate(motion):
        phase = phase_cur + motion
        sampled = cubic_sample_scipy(ref_l, phase[..., 0], phase[..., 1], phase[..., 2])
        if snoise is not None:
            sampled = sampled * (1.0 + snoise[1] * snoise[0].standard_normal(sampled.shape))
        ref_ex = cubic_sample_scipy(mask_ref_f, phase[..., 0], phase[..., 1], phase[..., 2]) > 0.5
        valid = ~mask_mov_l & ~ref_ex
        res = ndimage.correlate(mov_l - sampled, box3, mode="nearest")
        res[~valid] = 0
        return phase, sampled, valid, res

    error_init = None
    for it_idx in range(n_iter):
        old_motion = motion.copy()
        phase_new, ref_sampled, valid, res = evaluate(motion)
        if it_idx == 0:
            error_init = res ** 2
        cpm = motion[xg][:, yg]
        nei = get_nei_diff(cpm)
        nei[..., 2] *= zratio_hr
        nei_sum = sps * nei
        diff_e, pen_e = cal_error(res, nei, sps)
        current_error = diff_e + pen_e
        lg["diffError"].append(diff_e)
        lg["penaltyError"].append(pen_e)
        lg["currentError"].append(current_error)
        if forced is not None:
            if n_updates >= forced:
                break
        else:
            if it_idx == n_iter - 1:
                break
            if np.sum(old_error <= current_error) > 1:
                break
            if np.abs(old_error[-1] - current_error) < tol:
                break
        old_error[:-1] = old_error[1:]
        old_error[-1] = current_error

        gx, gy, gz = spatial_gradient(ref_l, phase_new)
        gx[~valid] = 0
        gy[~valid] = 0
        gz[~valid] = 0
        gz = gz / zratio_hr
        prods = {
            "xx": gx * gx, "xy": gx * gy, "xz": gx * gz, "yy": gy * gy, "yz": gy * gz,
            "zz": gz * gz, "xt": gx * res, "yt": gy * res, "zt": gz * res,
        }
        sums = {k: _window_sums_segmented(v, r, ncx, ncy) for k, v in prods.items()}
        if wnoise is not None:
            for k in sums:
                sums[k] = sums[k] * (1.0 + wnoise[1] * wnoise[0].standard_normal(sums[k].shape))
        v = solve_flow_with_penalty(sums, sps, nei_sum)
        dist = np.maximum(np.sqrt(np.sum(v ** 2, axis=3)) / mov_range, 1.0)
        v = v / dist[..., None]
        v[..., 2] = v[..., 2] / zratio_hr
        cp_new = cpm + v
        gx_n = np.clip((grid[0] - np.float32(r)) / np.float32(2 * r + 1), 0.0, ncx).astype(np.float32)
        gy_n = np.clip((grid[1] - np.float32(r)) / np.float32(2 * r + 1), 0.0, ncy).astype(np.float32)
        for d in range(3):
            motion[..., d] = trilinear(cp_new[..., d], gx_n, gy_n, grid[2], out_dtype=np.float64)
        n_updates += 1
        max_diff = float(np.max(np.abs(motion - old_motion)))
        lg["max_diff_motion"].append(max_diff)
        if forced is None and max_diff < tol:
            break

    phase_new, ref_sampled, valid, res = evaluate(motion)
    nei = get_nei_diff(motion[xg][:, yg])
    diff_e, pen_e = cal_error(res, nei, sps)
    error_last = res ** 2
    return {"motion": motion, "phase_new": phase_new, "data_ref_sampled": ref_sampled, "residual": res,
            "valid_mask": valid, "current_error": diff_e + pen_e,
            "error_init": error_init if error_init is not None else error_last.copy(), "error_last": error_last}


# ----------------------------------------------------------------------------
# wrong-region correction (calFlowCrossResolution.py:1190-1900, 2240-2467)
# ----------------------------------------------------------------------------

MAX_BALL_RADIUS_Z = 64   # the reference's cap on a structuring element's z radius


def make_ball(radius_xy, z_ratio):
    """Anisotropic ball: offsets within radius_xy physical units, z spaced
    z_ratio (calFlowCrossResolution.py:1363-1396); float32 distances."""
    radius_xy = int(max(1, radius_xy))
    z_ratio = float(z_ratio)
    radius_z = int(max(1, min(np.ceil(radius_xy / z_ratio), MAX_BALL_RADIUS_Z)))
    xs = np.arange(-radius_xy, radius_xy + 1, dtype=np.float32)
    zs = np.arange(-radius_z, radius_z + 1, dtype=np.float32)
    XX, YY, ZZ = np.meshgrid(xs, xs, zs, indexing="ij")
    dist2 = XX ** 2 + YY ** 2 + (ZZ * z_ratio) ** 2
    return dist2 <= radius_xy ** 2 + 1e-6


def local_cp_error(residual, xg, yg, kernelsize, metric="mse"):
    """get_local_error_on_control_points (:1190-1222): window mean of the
    squared (or absolute) residual at the control points."""
    err = residual ** 2 if metric.lower() == "mse" else np.abs(residual)
    kernel = np.ones((kernelsize, kernelsize, 1), dtype=np.float32) / (kernelsize ** 2)
    avg = ndimage.correlate(err, kernel, mode="nearest")
    return avg[xg][:, yg]


def bad_region_mask(err_cp, r, xg, yg, x_size, y_size, mad_threshold=3.0, min_component_size=2,
                    large_cp_threshold=144, eps=1e-12):
    """build_bad_region_mask_from_cp_error (:1570-1787): per z slice, control
    points whose robust z-score exceeds the threshold (inner points only on a
    grid of more than 144), 4-connected in the slice, components of at least
    min_component_size points, each widened by ceil(1.5 r) voxels to a box."""
    nx, ny, z_size = err_cp.shape
    sig = np.zeros(err_cp.shape, bool)
    inner = nx * ny > large_cp_threshold and nx > 2 and ny > 2
    sub = err_cp[1:-1, 1:-1, :] if inner else err_cp
    flat = sub.reshape(-1, z_size)
    med = np.median(flat, axis=0)
    mad = np.median(np.abs(flat - med[None, :]), axis=0)
    rz = np.abs(flat - med[None, :]) / (1.4826 * mad[None, :] + eps)
    s_flat = rz > mad_threshold
    s_flat[:, mad < eps] = False
    if inner:
        sig[1:-1, 1:-1, :] = s_flat.reshape(nx - 2, ny - 2, z_size)
    else:
        sig = s_flat.reshape(nx, ny, z_size)
    bad = np.zeros((x_size, y_size, z_size), bool)
    if not sig.any():
        return bad, 0
    structure = np.zeros((3, 3, 3), bool)
    structure[:, :, 1] = [[0, 1, 0], [1, 1, 1], [0, 1, 0]]
    labels, nlab = ndimage.label(sig, structure=structure)
    dx = int(np.ceil(1.5 * r))
    kept = 0
    for lab in range(1, nlab + 1):
        where = np.argwhere(labels == lab)
        if len(where) < min_component_size:
            continue
        kept += 1
        x0 = max(0, int(xg[where[:, 0].min()]) - dx)
        x1 = min(x_size - 1, int(xg[where[:, 0].max()]) + dx)
        y0 = max(0, int(yg[where[:, 1].min()]) - dx)
        y1 = min(y_size - 1, int(yg[where[:, 1].max()]) + dx)
        z0, z1 = int(where[:, 2].min()), int(where[:, 2].max())
        bad[x0:x1 + 1, y0:y1 + 1, z0:z1 + 1] = True
    return bad, kept


def quantile_threshold(arr, q):
    """get_quantile_threshold (:1790-1799): the element of rank
    floor((n - 1) q) of the flattened values (0 for none)."""
    flat = np.asarray(arr).ravel()
    if flat.size == 0:
        return 0.0
    k = int(np.clip(np.floor((flat.size - 1) * q), 0, flat.size - 1))
    return np.partition(flat, k)[k]


def high_residual_refine(bad, error_init, error_last, q):
    """The "highresidual" exclusion mode (:2340-2355): inside the bad boxes,
    keep only the voxels whose 3x3-smoothed error drop (first iteration minus
    final) reaches the q quantile of the drops in the boxes."""
    box3 = np.ones((3, 3, 1), dtype=np.float32) / 9
    dense = ndimage.correlate(error_init - error_last, box3, mode="nearest")
    dense[~bad] = 0
    th = quantile_threshold(dense[bad], q) if bad.any() else 0
    return bad & (dense >= th)


def trap_mask(bad_mask, phase_new, ref_l, z_ratio_ref, expand_radius_xy=2.0, sigma_grad=1.0, intensity_k=2.5):
    """build_reference_trap_mask_from_bad_moving_fast_roi (:1413-1567): the
    bad moving voxels' rounded phases as seeds in reference space, closed by
    a unit ball, grown inside a distance ball through reference voxels whose
    Gaussian-smoothed intensity is within intensity_k robust deviations of the
    seeds'."""
    shp = ref_l.shape
    trap = np.zeros(shp, bool)
    if not bad_mask.any():
        return trap
    sc = phase_new[bad_mask]
    sx, sy, sz = (np.rint(sc[:, k]).astype(np.int32) for k in range(3))
    keep = (sx >= 0) & (sx < shp[0]) & (sy >= 0) & (sy < shp[1]) & (sz >= 0) & (sz < shp[2])
    sx, sy, sz = sx[keep], sy[keep], sz[keep]
    if sx.size == 0:
        return trap
    margin_xy = int(max(1, expand_radius_xy + 2))
    margin_z = int(max(1, np.ceil((expand_radius_xy + 2) / max(float(z_ratio_ref), 1e-6))))
    x0, x1 = max(0, int(sx.min()) - margin_xy), min(shp[0], int(sx.max()) + margin_xy + 1)
    y0, y1 = max(0, int(sy.min()) - margin_xy), min(shp[1], int(sy.max()) + margin_xy + 1)
    z0, z1 = max(0, int(sz.min()) - margin_z), min(shp[2], int(sz.max()) + margin_z + 1)
    seed = np.zeros((x1 - x0, y1 - y0, z1 - z0), bool)
    seed[sx - x0, sy - y0, sz - z0] = True
    small = make_ball(1, z_ratio_ref)
    seed = ndimage.binary_closing(seed, structure=small)
    if not seed.any():
        return trap
    crop = ref_l[x0:x1, y0:y1, z0:z1].astype(np.float32)
    sm = ndimage.gaussian_filter(crop, sigma=(sigma_grad,) * 3) if sigma_grad > 0 else crop
    vals = sm[seed]
    i_med = float(np.median(vals))
    i_mad = float(np.median(np.abs(vals - i_med)))
    tol = max(intensity_k * 1.4826 * i_mad, 1e-3)
    near = ndimage.binary_dilation(seed, structure=make_ball(max(1, int(round(expand_radius_xy))), z_ratio_ref),
                                   iterations=1)
    allowed = (near & (np.abs(sm - i_med) <= tol)) | seed
    region = seed.copy()
    for _ in range(int(expand_radius_xy)):
        grown = ndimage.binary_dilation(region, structure=small) & allowed
        if np.all(grown == region):
            break
        region = grown
    trap[x0:x1, y0:y1, z0:z1] = region | seed
    return trap


def get_motion_v2(dat_mov, dat_ref, option, replay_updates=None, window_noise=None, sample_noise=None):
    """``getMotion_v2`` (calFlowCrossResolution.py:2470-2663).

    Returns (phase_new float32 (x,y,z,3), motion float32 (x,y,z,3),
    data_ref_sampled float64 (x,y,z), log) where log["layer_l"] holds the
    diffError / penaltyError / currentError lists and the max |motion change|
    of every update (all passes of a layer, in order), and, with the
    wrong-region correction, log["layer_l"]["wrong_region"] its decisions.
    ``replay_updates`` maps layer -> number of updates to perform, overriding
    the stopping rules (wrong-region correction off only).  ``window_noise =
    (seed, rel)`` multiplies every window sum by (1 + rel N(0, 1)): a model
    of single-precision accumulation, used by the tests to measure how far
    the reference's own result moves under rounding-level changes (it is
    chaotic where a window is nearly empty or the phase leaves the reference
    volume).  ``sample_noise = (seed, rel)`` does the same to every value of
    the reference's spline at the phase (single-precision spline evaluation).
    """
    mask_ref_full = np.asarray(option["mask_ref"], dtype=np.float32)
    mask_mov_full = np.asarray(option["mask_mov"], dtype=np.float32)
    n_layer = int(option["layer"])
    n_iter = int(option["iter"])
    r = int(option["r"])
    zratio_raw = float(option.get("zRatio", 1.0))
    zratio_hr_raw = float(option["zRatio_HR"])
    sp = float(option["smoothPenalty"])
    mov_range = float(option.get("movRange", 5.0))
    tol = float(option.get("tol", 1e-3))
    wr_enable = bool(option.get("wrong_region_enable", True))
    wr_metric = option.get("wrong_region_metric", "mse")
    wr_mad = float(option.get("wrong_region_mad_threshold", 3.0))
    wr_min = int(option.get("wrong_region_min_component_size", 2))
    wr_mode = option.get("wrong_region_exclude_mode", "direct")
    expand = float(option.get("expand_radius_xy", 2.0))
    sigma_grad = float(option.get("sigma_grad", 1.0))
    intensity_k = float(option.get("intensity_k", 2.0))
    quantile_q = float(option.get("quantile_threshold_q", 0.8))
    if wr_enable and replay_updates is not None:
        raise NotImplementedError("oracle: the wrong-region correction runs without replay")
    if wr_enable and wr_mode not in ("direct", "highresidual"):
        raise ValueError(f"unknown wrong_region_exclude_mode {wr_mode!r}")
    dat_mov = np.asarray(dat_mov, dtype=np.float32)
    dat_ref = np.asarray(dat_ref, dtype=np.float32)
    sz, sz_hr = dat_mov.shape, dat_ref.shape
    motion = None
    log = {}
    noise = None
    if window_noise is not None or sample_noise is not None:
        noise = ((np.random.default_rng(window_noise[0]), window_noise[1]) if window_noise is not None else None,
                 (np.random.default_rng(sample_noise[0]), sample_noise[1]) if sample_noise is not None else None)
    res = None

    for layer in range(n_layer, -1, -1):
        lg = {"diffError": [], "penaltyError": [], "currentError": [], "max_diff_motion": []}
        log[f"layer_{layer}"] = lg
        x, y, z = int(sz[0] / 2 ** layer), int(sz[1] / 2 ** layer), sz[2]
        shape = (x, y, z)
        shape_hr = (int(sz_hr[0] / 2 ** layer), int(sz_hr[1] / 2 ** layer), sz_hr[2])
        mov_l = imresize(dat_mov, shape)
        ref_l = imresize(dat_ref, shape_hr)
        mask_mov_l = imresize(mask_mov_full, shape) > 0.5
        mask_ref_l = imresize(mask_ref_full, shape_hr) > 0.5
        zratio = zratio_raw / 2 ** layer
        zratio_hr = zratio_hr_raw / 2 ** layer

        if layer == n_layer:
            motion = np.zeros(shape + (3,), dtype=np.float32)
            init = option.get("motion")
            if init is not None:
                init = np.asarray(init, dtype=np.float32)
                for d in range(3):
                    motion[..., d] = imresize(init[..., d], shape) / (sz[d] / shape[d])
        else:
            prev = motion
            motion = np.zeros(shape + (3,), dtype=np.float32)
            for d in range(3):
                up = imresize(prev[..., d], shape, method="bilinear")
                motion[..., d] = up * 2 if d < 2 else up

        phase_init = option.get("phase")
        if phase_init is not None:
            phase_init = np.asarray(phase_init, dtype=np.float32)
            phase_cur = np.zeros(shape + (3,), dtype=np.float32)
            for d in range(3):
                phase_cur[..., d] = imresize(phase_init[..., d], shape) / (sz[d] / shape[d])
        else:
            X, Y, Z = np.indices(shape)
            phase_cur = np.stack([X, Y, Z * zratio / zratio_hr], axis=-1).astype(np.float32)
        sps = sp * (2 * r + 1) ** 2
        forced = None if replay_updates is None else int(replay_updates[layer])
        common = dict(r=r, n_iter=n_iter, sps=sps, mov_range=mov_range, tol=tol, zratio_hr=zratio_hr, lg=lg,
                      noise=noise)
        mask_ref_f = mask_ref_l.astype(np.float32)
        res0 = _optimize_layer(mov_l, ref_l, mask_mov_l, mask_ref_f, phase_cur, motion, forced=forced, **common)
        res = res0
        if wr_enable:
            xg = np.arange(r, x - 1, 2 * r + 1)
            yg = np.arange(r, y - 1, 2 * r + 1)
            err_cp = local_cp_error(res0["residual"], xg, yg, 2 * r + 1, wr_metric)
            bad, nreg = bad_region_mask(err_cp, r, xg, yg, x, y, wr_mad, wr_min)
            decision = {"regions": nreg}
            lg["wrong_region"] = decision
            if nreg > 0:
                if wr_mode == "highresidual":
                    bad = high_residual_refine(bad, res0["error_init"], res0["error_last"], quantile_q)
                bad = bad & res0["valid_mask"]
                trap = trap_mask(bad, res0["phase_new"], ref_l, zratio_hr, expand / (2.0 ** layer), sigma_grad,
                                 intensity_k)
                corrected = (mask_ref_l | trap).astype(np.float32)
                n_old = int(res0["valid_mask"].sum())
                ref_ex = cubic_sample_scipy(corrected, res0["phase_new"][..., 0], res0["phase_new"][..., 1],
                                            res0["phase_new"][..., 2]) > 0.5
                n_new = int((~mask_mov_l & ~ref_ex).sum())
                ratio = n_new / max(n_old, 1)
                decision.update({"trap_voxels": int(trap.sum()), "valid_ratio": ratio})
                if ratio >= 0.4:
                    res1 = _optimize_layer(mov_l, ref_l, mask_mov_l, corrected, phase_cur, motion, **common)
                    res2 = _optimize_layer(mov_l, ref_l, mask_mov_l, mask_ref_f, phase_cur, res1["motion"],
                                           **common)
                    decision.update({"error0": res0["current_error"], "error2": res2["current_error"]})
                    if res2["current_error"] < res0["current_error"]:
                        res = res2
                    decision["accepted"] = res is res2
        motion = res["motion"]

    return res["phase_new"], motion, res["data_ref_sampled"], log


def project_max(values, coords, target_z, xref, yref, ds=1, z_window=1.5, nearest=False, extra=0, fill=0.0):
    """Max splat (calFlowCrossResolution.py:480-569, 878-1141): values (n,),
    coords (n, 3) = (x, y, z); returns (nplanes, xout, yout) float32."""
    values = np.asarray(values, np.float32).ravel()
    coords = np.asarray(coords, np.float32).reshape(-1, 3)
    target_z = np.atleast_1d(np.asarray(target_z, np.float32))
    xout, yout = (xref + ds - 1) // ds, (yref + ds - 1) // ds
    fin = values[np.isfinite(values)]
    shift = np.float32(max(np.float32(-fin.min() + np.float32(1.0)), np.float32(0.0))) if fin.size else np.float32(0.0)
    shifted = (values + shift).astype(np.float32)
    out = np.full((len(target_z), xout, yout), -np.inf, np.float32)
    for i in range(values.size):
        v = shifted[i]
        x, y, z = coords[i]
        if not (np.isfinite(v) and np.isfinite(x) and np.isfinite(y) and np.isfinite(z)):
            continue
        if nearest:
            xs = [int(np.floor(np.float32(x + np.float32(0.5))))]
            ys = [int(np.floor(np.float32(y + np.float32(0.5))))]
        else:
            xf, yf = int(np.floor(x)), int(np.floor(y))
            xs = range(xf - extra, xf + 2 + extra)
            ys = range(yf - extra, yf + 2 + extra)
        for p, z0 in enumerate(target_z):
            if abs(np.float32(z - z0)) > np.float32(z_window):
                continue
            for xi in xs:
                if xi < 0 or xi >= xref or xi // ds >= xout:
                    continue
                for yi in ys:
                    if yi < 0 or yi >= yref or yi // ds >= yout:
                        continue
                    o = out[p, xi // ds, yi // ds]
                    out[p, xi // ds, yi // ds] = max(o, v)
    valid = np.isfinite(out)
    out = np.where(valid, (out - shift).astype(np.float32), out)
    if fill is not None:
        out = np.where(np.isfinite(out), out, np.float32(fill)).astype(np.float32)
    return out


def project_weighted(values, coords, target_z, xref, yref, ds=1, z_window=1.5, z_sigma=None, mode=2, fill=0.0,
                     eps=1e-6):
    """Weighted bilinear splat (calFlowCrossResolution.py:571-660, 700-876);
    returns (planes, summed weights), both (nplanes, xout, yout), float64
    sums (the CUDA kernel accumulates float32 atomically)."""
    values = np.asarray(values, np.float32).ravel()
    coords = np.asarray(coords, np.float32).reshape(-1, 3)
    target_z = np.atleast_1d(np.asarray(target_z, np.float32))
    xout, yout = (xref + ds - 1) // ds, (yref + ds - 1) // ds
    sv = np.zeros((len(target_z), xout, yout))
    sw = np.zeros((len(target_z), xout, yout))
    sigma = np.float32(z_window * 0.5 if z_sigma is None or z_sigma <= 0 else z_sigma)
    for i in range(values.size):
        v = float(values[i])
        x, y, z = (float(c) for c in coords[i])
        if not all(np.isfinite([v, x, y, z])):
            continue
        if x < 0 or x > xref - 1 or y < 0 or y > yref - 1:
            continue
        xo_f, yo_f = x / ds, y / ds
        xo0, yo0 = int(np.floor(xo_f)), int(np.floor(yo_f))
        dx, dy = xo_f - xo0, yo_f - yo0
        for p, z0 in enumerate(target_z):
            dz = abs(z - float(z0))
            if dz > z_window:
                continue
            if mode == 0:
                wz = 1.0
            elif mode == 1:
                wz = max(1.0 - dz / (z_window + 1e-6), 0.0)
            else:
                wz = float(np.exp(-0.5 * dz * dz / (float(sigma) ** 2 + 1e-6)))
            if wz <= 0:
                continue
            for ax in (0, 1):
                xo = xo0 + ax
                if xo < 0 or xo >= xout:
                    continue
                wx = 1.0 - dx if ax == 0 else dx
                for ay in (0, 1):
                    yo = yo0 + ay
                    if yo < 0 or yo >= yout:
                        continue
                    w = wx * (1.0 - dy if ay == 0 else dy) * wz
                    if w <= 0:
                        continue
                    sv[p, xo, yo] += v * w
                    sw[p, xo, yo] += w
    out = np.where(sw > eps, sv / np.maximum(sw, eps), fill)
    return out, sw
