"""CPU oracle for the cross-resolution registration ``getMotion_v2``.

TEST INFRASTRUCTURE ONLY.  This module is the checker: only ``tests/`` may
import it.  The product path (``wholistic_registration_b200``) never calls
into it and fails loudly when its CUDA library is missing.

It restates, in NumPy, the reference's cross-resolution path with the
wrong-region correction switched off (``wrong_region_enable=False``); paths
are relative to ``src/wholistic_registration``:

* ``utils/calFlowCrossResolution.py:2470-2663``  ``getMotion_v2``: pyramid of
  the moving stack on its grid and of the reference stack on its own
  (cross-resolution) grid
* ``utils/calFlowCrossResolution.py:2031-2237``  ``optimize_layer_cross_resolution``
* ``utils/calFlowCrossResolution.py:1904-2028``  phase composition, mask
  resampling (threshold 0.5), motion / phase initialisation (``option["phase"]``
  included), CP grid, valid mask
* ``utils/calFlowCrossResolution.py:463-478, 1144-1154``  the continuous
  reference ``H``: ``map_coordinates(order=3, mode="nearest")``
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
           "project_max", "project_weighted"]

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


def get_motion_v2(dat_mov, dat_ref, option, replay_updates=None, window_noise=None, sample_noise=None):
    """``getMotion_v2`` with ``wrong_region_enable=False``.

    Returns (phase_new float32 (x,y,z,3), motion float32 (x,y,z,3),
    data_ref_sampled float64 (x,y,z), log) where log["layer_l"] holds the
    diffError / penaltyError / currentError lists and the max |motion change|
    of every update.  ``replay_updates`` maps layer -> number of updates to
    perform, overriding the stopping rules.  ``window_noise = (seed, rel)``
    multiplies every window sum by (1 + rel N(0, 1)): a model of
    single-precision accumulation, used by the tests to measure how far the
    reference's own result moves under rounding-level changes (it is chaotic
    where a window is nearly empty or the phase leaves the reference volume).
    ``sample_noise = (seed, rel)`` does the same to every value of the
    reference's spline at the phase (single-precision spline evaluation).
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
    dat_mov = np.asarray(dat_mov, dtype=np.float32)
    dat_ref = np.asarray(dat_ref, dtype=np.float32)
    sz, sz_hr = dat_mov.shape, dat_ref.shape
    motion = None
    log = {}
    phase_new = ref_sampled = None
    noise_rng = np.random.default_rng(window_noise[0]) if window_noise is not None else None
    sample_rng = np.random.default_rng(sample_noise[0]) if sample_noise is not None else None

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
        mask_ref_f = mask_ref_l.astype(np.float32)

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
        xg = np.arange(r, x - 1, 2 * r + 1)
        yg = np.arange(r, y - 1, 2 * r + 1)
        ncx, ncy = len(xg), len(yg)
        grid = _grid(shape)
        box3 = np.ones((3, 3, 1), dtype=np.float32) / 9
        old_error = np.inf * np.ones(3, dtype=np.float32)
        forced = None if replay_updates is None else int(replay_updates[layer])
        n_updates = 0

        def evaluate(motion):
            phase = phase_cur + motion
            sampled = cubic_sample_scipy(ref_l, phase[..., 0], phase[..., 1], phase[..., 2])
            if sample_noise is not None:
                sampled = sampled * (1.0 + sample_noise[1] * sample_rng.standard_normal(sampled.shape))
            ref_ex = cubic_sample_scipy(mask_ref_f, phase[..., 0], phase[..., 1], phase[..., 2]) > 0.5
            valid = ~mask_mov_l & ~ref_ex
            res = ndimage.correlate(mov_l - sampled, box3, mode="nearest")
            res[~valid] = 0
            return phase, sampled, valid, res

        for it_idx in range(n_iter):
            old_motion = motion.copy()
            phase_new, ref_sampled, valid, res = evaluate(motion)
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
            if window_noise is not None:
                for k in sums:
                    sums[k] = sums[k] * (1.0 + window_noise[1] * noise_rng.standard_normal(sums[k].shape))
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

    return phase_new, motion, ref_sampled, log


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
