"""CPU oracle for the pyramid patch-wise Lucas-Kanade registration path.

TEST INFRASTRUCTURE ONLY.  This module checks the product: only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may import
it.  The product path (``wholistic_registration_b200``) never calls into it and
fails loudly when its CUDA library is missing.

It restates, in NumPy, the algorithm of the reference package
``wholistic_registration`` (paths relative to ``src/wholistic_registration``):

* ``utils/imresize.py:41-191``       MATLAB-style antialiased resize
* ``utils/interp.py:28-45, 96-100``  trilinear ``map_coordinates`` (mode "nearest")
* ``utils/calculate.py:30-92``       box filters, 3x3 / 2x2 determinants
* ``utils/calFlow3d_Wei_v1.py:37-706`` ``getMotion`` / ``correctMotion`` and helpers
* ``utils/preprocess.py:42-66``      smoothness-penalty normalisation factor

Arrays follow the reference's internal layout: volumes are indexed (x, y, z)
and motion fields are (x, y, z, 3) with component c displacing axis c.

Parity is pinned against fixtures produced by running the reference itself
(``tests/golden/make_golden.py``); ``tests/test_oracle_golden.py`` checks this
module against them.

Two modes for the per-control-point window sums:

* ``window_sums="segmented"`` (default): the (2r+1)x(2r+1)x1 box filter is only
  ever sampled at control points whose windows tile each z-slice, so the sum is
  a reshape-and-sum over edge-replicated tiles.  Mathematically identical to the
  reference, ~100x cheaper.
* ``window_sums="correlate"``: calls ``scipy.ndimage.correlate`` with a ones
  kernel on the full grid, exactly as ``utils/calculate.py:51`` does, so the CPU
  cost matches the reference's NumPy path (used for the timed CPU baseline).
"""

from __future__ import annotations

import math

import numpy as np

__all__ = [
    "cubic",
    "triangle",
    "contributions",
    "imresize",
    "trilinear",
    "box_filter_nearest",
    "get_nei_diff",
    "cal_error",
    "spatial_gradient",
    "solve_flow_with_penalty",
    "get_motion",
    "correct_motion",
    "smooth_penalty_norm_factor",
]


# ----------------------------------------------------------------------------
# imresize (utils/imresize.py)
# ----------------------------------------------------------------------------

def cubic(t):
    """Keys cubic kernel, a = -0.5 (utils/imresize.py:49-57)."""
    a = np.abs(np.asarray(t, dtype=np.float64))
    a2 = a * a
    a3 = a2 * a
    near = (1.5 * a3 - 2.5 * a2 + 1) * (a <= 1)
    far = (-0.5 * a3 + 2.5 * a2 - 4 * a + 2) * ((a > 1) & (a <= 2))
    return near + far


def triangle(t):
    """Linear (tent) kernel (utils/imresize.py:41-46)."""
    t = np.asarray(t, dtype=np.float64)
    left = (t + 1) * ((t >= -1) & (t < 0))
    right = (1 - t) * ((t <= 1) & (t >= 0))
    return left + right


def contributions(in_len, out_len, scale, kernel, kernel_width=4.0):
    """Per-output tap weights and source indices along one axis.

    Follows ``utils/imresize.py:60-82``: antialiasing stretches the kernel by
    1/scale when shrinking, output sample k (1-based) maps to
    u = k/scale + (1 - 1/scale)/2, taps outside [0, in_len) reflect
    symmetrically (-1 -> 0, in_len -> in_len-1), weights are normalised per
    output, and tap columns whose weight is zero for every output are dropped.

    Returns (weights (out_len, T) float64, indices (out_len, T) int64).
    """
    if scale < 1:
        def h(t):
            return scale * kernel(scale * t)
        width = kernel_width / scale
    else:
        h = kernel
        width = kernel_width
    k = np.arange(1, out_len + 1, dtype=np.float64)
    u = k / scale + 0.5 * (1 - 1 / scale)
    left = np.floor(u - width / 2)
    ntaps = int(math.ceil(width)) + 2
    idx = (left[:, None] + np.arange(ntaps) - 1).astype(np.int64)
    w = h(u[:, None] - idx - 1)
    w = w / np.sum(w, axis=1, keepdims=True)
    mirror = np.concatenate([np.arange(in_len), np.arange(in_len - 1, -1, -1)])
    idx = mirror[np.mod(idx, mirror.size)]
    keep = np.any(w != 0, axis=0)
    return w[:, keep], idx[:, keep]


def _resize_axis(vol, axis, w, idx):
    """out[..k..] = sum_t w[k, t] * vol[..idx[k, t]..] along ``axis`` (float64).

    The reference multiplies and reduces over the tap axis
    (utils/imresize.py:121-137); taps are accumulated here in tap order.
    """
    vol = np.moveaxis(np.asarray(vol), axis, 0)
    out = np.zeros((w.shape[0],) + vol.shape[1:], dtype=np.float64)
    shape = (w.shape[0],) + (1,) * (vol.ndim - 1)
    for t in range(w.shape[1]):
        out += w[:, t].reshape(shape) * vol[idx[:, t]].astype(np.float64)
    return np.moveaxis(out, 0, axis)


def imresize(vol, output_shape, method="bicubic"):
    """Separable resize of a 3-D array to ``output_shape`` (float64 result).

    utils/imresize.py:148-191: the axes are processed in increasing order of
    scale; a scale-1 axis has a single unit tap, so it is an exact copy.
    uint8 inputs are rounded and clipped back to uint8 after every axis, as in
    utils/imresize.py:133-135.
    """
    kernel = {"bicubic": cubic, "bilinear": triangle}[method]
    vol = np.asarray(vol)
    scales = [output_shape[k] / vol.shape[k] for k in range(3)]
    tables = [contributions(vol.shape[k], output_shape[k], scales[k], kernel) for k in range(3)]
    out = vol
    for axis in np.argsort(np.asarray(scales), kind="stable"):
        in_dtype = out.dtype
        out = _resize_axis(out, int(axis), *tables[int(axis)])
        if in_dtype == np.uint8:
            out = np.round(np.clip(out, 0, 255)).astype(np.uint8)
    return out


# ----------------------------------------------------------------------------
# interpolation (utils/interp.py, calFlow3d_Wei_v1.py:37-66)
# ----------------------------------------------------------------------------

def trilinear(vol, cx, cy, cz, out_dtype=None):
    """Trilinear sample of ``vol`` at (cx, cy, cz), edge-replicated.

    Equivalent to ``scipy.ndimage.map_coordinates(order=1, mode="nearest")``
    (utils/interp.py:43): taps are clamped to the volume, weights come from the
    unclamped fractional part, arithmetic in float64.  The result is cast to
    ``out_dtype`` (default: ``vol.dtype``), matching scipy's output dtype.
    """
    vol = np.asarray(vol)
    out_dtype = vol.dtype if out_dtype is None else out_dtype
    n = vol.shape
    c = [np.asarray(a, dtype=np.float64) for a in (cx, cy, cz)]
    fl = [np.floor(a) for a in c]
    fr = [a - f for a, f in zip(c, fl)]
    base = [f.astype(np.int64) for f in fl]
    ix = [(np.clip(base[d], 0, n[d] - 1), np.clip(base[d] + 1, 0, n[d] - 1)) for d in range(3)]
    wt = [(1.0 - fr[d], fr[d]) for d in range(3)]
    acc = np.zeros(c[0].shape, dtype=np.float64)
    for a in (0, 1):
        for b in (0, 1):
            for e in (0, 1):
                acc += (wt[0][a] * wt[1][b] * wt[2][e]) * vol[ix[0][a], ix[1][b], ix[2][e]]
    return acc.astype(out_dtype)


def _grid(shape):
    """float32 index grid (calFlow3d_Wei_v1.py:413-419)."""
    return np.meshgrid(*[np.arange(n, dtype=np.float32) for n in shape], indexing="ij")


def _warp_f32(vol, coords):
    """``correctMotionGrid``: cast the volume to float32, then trilinear sample
    (calFlow3d_Wei_v1.py:37-66)."""
    v32 = np.asarray(vol, dtype=np.float32)
    return trilinear(v32, coords[..., 0], coords[..., 1], coords[..., 2])


# ----------------------------------------------------------------------------
# filters (utils/calculate.py, calFlow3d_Wei_v1.py:69-98)
# ----------------------------------------------------------------------------

def box_filter_nearest(a, sx, sy):
    """Centred sx x sy x 1 box correlation with edge replication (float64 sum).

    Same result as ``scipy.ndimage.correlate(a, ones((sx, sy, 1)), mode='nearest')``
    for odd sx, sy (utils/calculate.py:30-64).
    """
    a = np.asarray(a, dtype=np.float64)
    rx, ry = sx // 2, sy // 2
    x, y = a.shape[:2]
    out = np.zeros_like(a)
    for dx in range(-rx, rx + 1):
        ix = np.clip(np.arange(x) + dx, 0, x - 1)
        for dy in range(-ry, ry + 1):
            iy = np.clip(np.arange(y) + dy, 0, y - 1)
            out += a[ix][:, iy]
    return out


def get_nei_diff(cp_motion):
    """Mean of the 8 in-plane neighbours minus the centre, per component and z.

    calFlow3d_Wei_v1.py:69-98 with r=1: a 3x3x1x1 correlation whose outer
    taps are 1/8 and whose centre is -1, edge-replicated.  Evaluated in float64
    and returned as float32 like scipy's correlate on a float32 input.
    """
    m = np.asarray(cp_motion, dtype=np.float64)
    nx, ny = m.shape[:2]
    acc = np.zeros_like(m)
    for dx in (-1, 0, 1):
        ix = np.clip(np.arange(nx) + dx, 0, nx - 1)
        for dy in (-1, 0, 1):
            iy = np.clip(np.arange(ny) + dy, 0, ny - 1)
            wgt = -1.0 if (dx == 0 and dy == 0) else np.float64(np.float32(1.0 / 8.0))
            acc += wgt * m[ix][:, iy]
    return acc.astype(np.float32)


def cal_error(it, nei_diff, smooth_penalty_sum):
    """(diffError, penaltyError) of calFlow3d_Wei_v1.py:101-131.

    diffError = mean(It^2) in float64; the penalty is formed in float32 like the
    reference (float32 neiDiff times a Python float, summed in float32).
    """
    x, y, z = it.shape
    diff = float(np.mean(np.asarray(it, dtype=np.float64) ** 2))
    pen = np.sum(nei_diff.astype(np.float32) ** 2, axis=3) * np.float32(smooth_penalty_sum)
    pen = float(np.sum(pen, dtype=np.float32) / np.float32(x * y * z))
    return diff, pen


def spatial_gradient(vol, coords):
    """Central differences of trilinear samples at c +- e_k, clipped to the
    volume (calFlow3d_Wei_v1.py:134-206).  ``vol`` float64; coords float32."""
    n = vol.shape
    c = [coords[..., k] for k in range(3)]
    grads = []
    for k in range(3):
        hi = list(c)
        lo = list(c)
        hi[k] = np.clip(c[k] + np.float32(1.0), 0, n[k] - 1)
        lo[k] = np.clip(c[k] - np.float32(1.0), 0, n[k] - 1)
        grads.append((trilinear(vol, *hi) - trilinear(vol, *lo)) / 2.0)
    return grads


def solve_flow_with_penalty(s, sps, nei_sum):
    """Regularised 3x3 solve by adjugate / determinant, NaN -> 0.

    calFlow3d_Wei_v1.py:209-262 and utils/calculate.py:67-92.
    ``s`` is a dict of the nine window sums (float64 arrays).
    """
    ixx = s["xx"] + sps
    iyy = s["yy"] + sps
    izz = s["zz"] + sps
    ixy, ixz, iyz = s["xy"], s["xz"], s["yz"]
    ixt = s["xt"] + nei_sum[..., 0]
    iyt = s["yt"] + nei_sum[..., 1]
    izt = s["zt"] + nei_sum[..., 2]
    det = ixx * (iyy * izz - iyz ** 2) - ixy * (ixy * izz - iyz * ixz) + ixz * (ixy * iyz - iyy * ixz)
    m11 = iyy * izz - iyz * iyz
    m12 = -(ixy * izz - iyz * ixz)
    m13 = ixy * iyz - iyy * ixz
    m22 = ixx * izz - ixz * ixz
    m23 = -(ixx * iyz - ixy * ixz)
    m33 = ixx * iyy - ixy * ixy
    with np.errstate(divide="ignore", invalid="ignore"):
        vx = (m11 * ixt + m12 * iyt + m13 * izt) / det
        vy = (m12 * ixt + m22 * iyt + m23 * izt) / det
        vz = (m13 * ixt + m23 * iyt + m33 * izt) / det
    v = np.stack((vx, vy, vz), axis=-1)
    v[np.isnan(v)] = 0
    return v


# ----------------------------------------------------------------------------
# getMotion (calFlow3d_Wei_v1.py:295-673)
# ----------------------------------------------------------------------------

def _window_sums_segmented(p, r, ncx, ncy):
    """Sums of ``p`` over the (2r+1)^2 windows centred on the control points.

    Control point k sits at r + k(2r+1), so windows tile [0, n*(2r+1)); the part
    of the last window past the volume edge replicates the edge voxel
    (mode="nearest"), which the clamped gather below reproduces.
    """
    w = 2 * r + 1
    x, y, z = p.shape
    ix = np.minimum(np.arange(ncx * w), x - 1)
    iy = np.minimum(np.arange(ncy * w), y - 1)
    tiles = np.asarray(p, dtype=np.float64)[ix][:, iy]
    return tiles.reshape(ncx, w, ncy, w, z).sum(axis=(1, 3))


def _window_sums_correlate(p, r, xg, yg):
    """Reference-cost path: full-grid box correlation, then sample at the
    control points (calFlow3d_Wei_v1.py:546-588, utils/calculate.py:51)."""
    from scipy.ndimage import correlate

    k = np.ones((2 * r + 1, 2 * r + 1, 1))
    full = correlate(np.asarray(p, dtype=np.float64), k, mode="nearest")
    return full[xg][:, yg]


def get_motion(dat_mov, dat_ref, option, verbose=False, *, window_sums="segmented",
               replay_updates=None, image_dtype=np.float64):
    """Restatement of ``getMotion`` (calFlow3d_Wei_v1.py:295-673).

    Returns (motion float32 (x,y,z,3), currentError, coords float32 (x,y,z,3),
    error_log) with error_log["layer_l"] holding diffError, penaltyError,
    currentError and max_diff_motion lists, like the reference.

    ``replay_updates`` maps layer -> number of motion updates to perform,
    overriding the stopping rules (used to align iteration counts with a run
    whose stopping decisions were borderline).  ``image_dtype`` lets a test
    run the image math in float32 to estimate the effect of single precision.
    """
    mask_ref_full = np.asarray(option["mask_ref"], dtype=np.float32)
    mask_mov_full = np.asarray(option["mask_mov"], dtype=np.float32)
    n_layer = int(option["layer"])
    n_iter = int(option["iter"])
    r = int(option["r"])
    zratio_raw = float(option["zRatio"])
    mov_range = float(option["movRange"])
    tol = float(option["tol"])
    sz = np.asarray(dat_mov).shape
    error_log = {}
    motion = None
    current_error = None
    shape = None

    for layer in range(n_layer, -1, -1):
        log = {"diffError": [], "penaltyError": [], "currentError": [], "max_diff_motion": []}
        error_log[f"layer_{layer}"] = log
        x = int(sz[0] / (2 ** layer))
        y = int(sz[1] / (2 ** layer))
        z = sz[2]
        shape = (x, y, z)
        mov_l = imresize(dat_mov, shape).astype(image_dtype)
        ref_l = imresize(dat_ref, shape).astype(image_dtype)
        zratio = zratio_raw / (2 ** layer)

        if layer == n_layer:
            motion = np.zeros((x, y, z, 3), dtype=np.float32)
            init = option.get("motion")
            if init is not None:
                init = np.asarray(init, dtype=np.float32)
                for d in range(3):
                    motion[..., d] = imresize(init[..., d], shape) / (sz[d] / shape[d])
        else:
            prev = motion
            motion = np.zeros((x, y, z, 3), dtype=np.float32)
            for d in range(3):
                up = imresize(prev[..., d], shape, method="bilinear")
                motion[..., d] = up * 2 if d < 2 else up

        grid = _grid(shape)
        mask_ref = imresize(mask_ref_full, shape) > 0
        mask_mov = imresize(mask_mov_full, shape)
        old_error = np.full(3, np.inf)
        sps = float(option["smoothPenalty"]) * (2 * r + 1) ** 2
        xg = np.arange(r, x - 1, 2 * r + 1)
        yg = np.arange(r, y - 1, 2 * r + 1)
        ncx, ncy = len(xg), len(yg)
        n_updates = 0
        forced = None if replay_updates is None else int(replay_updates[layer])

        for it_idx in range(n_iter):
            old_motion = motion.copy()
            coords = motion.copy()
            for d in range(3):
                coords[..., d] += grid[d]
            warped = _warp_f32(mov_l, coords)
            mask = (_warp_f32(mask_mov, coords) > 0) | mask_ref
            it = box_filter_nearest(np.asarray(ref_l, dtype=np.float64) - warped, 3, 3) * (1.0 / 9.0)
            it[mask] = 0
            cpm = motion[xg][:, yg]
            nei = get_nei_diff(cpm)
            nei[..., 2] = nei[..., 2] * np.float32(zratio)
            nei_sum = nei * np.float32(sps)
            diff_e, pen_e = cal_error(it, nei, sps)
            current_error = diff_e + pen_e
            log["diffError"].append(diff_e)
            log["penaltyError"].append(pen_e)
            log["currentError"].append(current_error)
            if verbose:
                print(f"layer {layer} iter {it_idx} error {current_error:.6f}")

            if forced is not None:
                if n_updates >= forced:
                    break
            elif it_idx == n_iter - 1:
                break
            elif np.sum(old_error <= current_error) > 1:
                break
            elif abs(old_error[-1] - current_error) < tol:
                break
            else:
                old_error[:-1] = old_error[1:]
                old_error[-1] = current_error

            gx, gy, gz = spatial_gradient(np.asarray(mov_l, dtype=np.float64), coords)
            gx[mask] = 0
            gy[mask] = 0
            gz[mask] = 0
            gz = gz / zratio
            prods = {
                "xx": gx * gx, "xy": gx * gy, "xz": gx * gz, "yy": gy * gy, "yz": gy * gz,
                "zz": gz * gz, "xt": gx * it, "yt": gy * it, "zt": gz * it,
            }
            if window_sums == "segmented":
                sums = {k: _window_sums_segmented(v, r, ncx, ncy) for k, v in prods.items()}
            else:
                sums = {k: _window_sums_correlate(v, r, xg, yg) for k, v in prods.items()}
            v = solve_flow_with_penalty(sums, sps, nei_sum)
            dist = np.maximum(np.sqrt(np.sum(v ** 2, axis=3)) / mov_range, 1.0)
            v = v / dist[..., None]
            v[..., 2] = v[..., 2] / zratio
            cp_new = cpm + v
            gx_n = np.clip((grid[0] - np.float32(r)) / np.float32(2 * r + 1), 0.0, ncx).astype(np.float32)
            gy_n = np.clip((grid[1] - np.float32(r)) / np.float32(2 * r + 1), 0.0, ncy).astype(np.float32)
            for d in range(3):
                motion[..., d] = trilinear(cp_new[..., d], gx_n, gy_n, grid[2], out_dtype=np.float64)
            n_updates += 1
            max_diff = float(np.max(np.abs(motion - old_motion)))
            log["max_diff_motion"].append(max_diff)
            if forced is None and max_diff < 1e-3:
                break

    grid = _grid(shape)
    coords = motion.copy()
    for d in range(3):
        coords[..., d] += grid[d]
    return motion, current_error, coords, error_log


def correct_motion(data_raw, motion_field):
    """``correctMotion`` (calFlow3d_Wei_v1.py:676-706): float32 pull-warp."""
    data_raw = np.asarray(data_raw)
    grid = _grid(data_raw.shape)
    coords = np.asarray(motion_field, dtype=np.float32).copy()
    for d in range(3):
        coords[..., d] += grid[d]
    return _warp_f32(data_raw, coords)


def smooth_penalty_norm_factor(dat_ref, mask_ref):
    """``getSmPnltNormFctr`` (utils/preprocess.py:42-66): half the sum of the
    mean squared x and y central differences over non-excluded voxels."""
    d = np.asarray(dat_ref)
    mask_ref = np.asarray(mask_ref, dtype=bool)
    ix = (d[2:, :, :] - d[:-2, :, :]) / 2
    iy = (d[:, 2:, :] - d[:, :-2, :]) / 2
    ixx = np.mean(ix[~mask_ref[1:-1, :, :]] ** 2)
    iyy = np.mean(iy[~mask_ref[:, 1:-1, :]] ** 2)
    return (ixx + iyy) / 2
