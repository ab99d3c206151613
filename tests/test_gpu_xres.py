"""Cross-resolution registration (getMotion_v2, with and without the
wrong-region correction) on the GPU against fixtures from the reference's
own runs and against the oracle restatement.

Tolerances: motion and phase within 1e-3 voxel (max abs) wherever the
reference's own result is stable, the sampled reference within 1e-4 relative
to its range (float32 spline coefficients and accumulation against the
reference's float64), and the same number of motion updates per level as the
reference's run (read from the oracle, which reproduces that run exactly).

"Stable": the cross-resolution scheme is chaotic where a window is nearly
empty (masks), where the phase leaves the reference volume (the z = 0 slice
with motion pointing out) and for a single-slice moving stack: there the
reference's own motion moves by more than 1e-3 voxel under perturbations at
the level of single-precision arithmetic.  The oracle measures that spread
per voxel over six runs in which every spline sample of the reference is
scaled by 1 + 1e-6 N(0, 1) (float32 spline evaluation) and every window sum
by 1 + 3e-7 N(0, 1) (float32 accumulation); the bound is 1e-3 + 3 x spread,
and at most 0.1 % of the voxels may exceed it.  A 1 % error in zRatio_HR,
planted in the oracle, breaks the bound in 35-98 % of the voxels of the
cases whose reference stack has more than one slice, except the wide
reference case, which is sensitive almost everywhere (4 %); update counts,
error logs and the sampled reference are checked independently of the bound.
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import (load_xres_case, load_xres_hr_case, load_xres_opt_case, load_xres_wr_case, xres_case_names,
                      xres_hr_case_names, xres_opt_case_names, xres_wr_case_names)

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _updates_per_level(log):
    return {int(k.split("_")[1]): len(v["max_diff_motion"]) for k, v in log.items()}


def _reference_spread(arrays, option, motion_ref):
    """Per-voxel max |motion change| of the oracle when its spline samples and
    window sums are perturbed at single-precision level (six seeds)."""
    from oracle import xres_oracle as X

    spread = np.zeros_like(motion_ref)
    for seed in range(6):
        _, m, _, _ = X.get_motion_v2(arrays["mov"], arrays["ref"], dict(option), window_noise=(seed, 3e-7),
                                     sample_noise=(100 + seed, 1e-6))
        spread = np.maximum(spread, np.abs(m - motion_ref))
    return spread


@pytest.mark.parametrize("name", xres_case_names())
def test_xres_matches_reference_run(name):
    from oracle import xres_oracle as X
    from wholistic_registration_b200 import calFlowCrossResolution as C

    arrays, option = load_xres_case(name)
    phase, motion, sampled = C.getMotion_v2(arrays["mov"], arrays["ref"], dict(option))
    assert phase.shape == arrays["phase"].shape and motion.shape == arrays["motion"].shape
    assert phase.dtype == np.float32 and motion.dtype == np.float32 and sampled.dtype == np.float64
    _, _, _, log = X.get_motion_v2(arrays["mov"], arrays["ref"], dict(option))
    dev_log, _ = C.last_registrar.error_log()
    want = _updates_per_level(log)
    got = {int(k.split("_")[1]): len(v["max_diff_motion"]) for k, v in dev_log.items()}
    assert got == want, f"updates per level {got} vs reference {want}"
    spread = _reference_spread(arrays, option, arrays["motion"])
    bound = 1e-3 + 3.0 * spread
    err_m = np.abs(motion - arrays["motion"])
    err_p = np.abs(phase - arrays["phase"])
    assert (err_m > bound).mean() <= 1e-3, f"motion: max excess {float((err_m - bound).max()):.3g}"
    assert (err_p > bound).mean() <= 1e-3, f"phase: max excess {float((err_p - bound).max()):.3g}"
    assert float(err_m.max()) < 0.5
    # the sampled reference: against the fixture where the motion is stable,
    # and everywhere against the spline evaluated at this run's own phase
    span = float(np.ptp(arrays["ref_sampled"])) or 1.0
    stable = (3.0 * spread).max(axis=-1) <= 1e-3
    np.testing.assert_allclose(sampled[stable], arrays["ref_sampled"][stable], rtol=0, atol=1e-4 * span)
    own = X.cubic_sample_scipy(arrays["ref"].astype(np.float64), phase[..., 0], phase[..., 1], phase[..., 2])
    np.testing.assert_allclose(sampled, own, rtol=0, atol=1e-4 * span)


def test_xres_errors_follow_reference_log():
    """Per-iteration diff / penalty errors of the device run track the
    reference's (oracle) log within float32 accumulation error."""
    from oracle import xres_oracle as X
    from wholistic_registration_b200 import calFlowCrossResolution as C

    arrays, option = load_xres_case("xr_mask_r2_l1")
    C.getMotion_v2(arrays["mov"], arrays["ref"], dict(option))
    dev_log, _ = C.last_registrar.error_log()
    _, _, _, log = X.get_motion_v2(arrays["mov"], arrays["ref"], dict(option))
    for layer, lv in log.items():
        d = dev_log[layer]
        assert len(d["diffError"]) == len(lv["diffError"])
        np.testing.assert_allclose(d["diffError"], lv["diffError"], rtol=2e-4)
        np.testing.assert_allclose(d["penaltyError"], lv["penaltyError"], rtol=2e-3, atol=1e-9)


def test_xres_torch_inputs_stay_on_device():
    from wholistic_registration_b200 import calFlowCrossResolution as C

    arrays, option = load_xres_case("xr_small_r3_l1")
    mov = torch.from_numpy(arrays["mov"]).cuda()
    ref = torch.from_numpy(arrays["ref"]).cuda()
    phase, motion, sampled = C.getMotion_v2(mov, ref, dict(option))
    assert phase.is_cuda and motion.is_cuda and sampled.is_cuda
    np.testing.assert_allclose(motion.cpu().numpy(), arrays["motion"], rtol=0, atol=1e-3)


def test_xres_wrong_region_option_handling():
    """An unknown metric raises ValueError; an exclusion mode other than
    "highresidual" runs the direct exclusion, as the reference's equality test
    (utils/calFlowCrossResolution.py:2340) does: same motion as "direct"."""
    from wholistic_registration_b200 import calFlowCrossResolution as C

    arrays, option = load_xres_case("xr_small_r3_l1")
    opt = dict(option)
    opt["wrong_region_enable"] = True
    opt["wrong_region_exclude_mode"] = "direct"
    _, direct, _ = C.getMotion_v2(arrays["mov"], arrays["ref"], dict(opt))
    opt["wrong_region_exclude_mode"] = "lowresidual"
    _, other, _ = C.getMotion_v2(arrays["mov"], arrays["ref"], dict(opt))
    np.testing.assert_array_equal(other, direct)
    opt["wrong_region_exclude_mode"] = "direct"
    opt["wrong_region_metric"] = "l2"
    with pytest.raises(ValueError):
        C.getMotion_v2(arrays["mov"], arrays["ref"], opt)


@pytest.mark.parametrize("kind,name", [("direct", n) for n in xres_wr_case_names()] +
                         [("highresidual", n) for n in xres_hr_case_names()] +
                         [("options", n) for n in xres_opt_case_names()])
def test_xres_wrong_region_matches_reference_run(kind, name):
    """getMotion_v2 with the wrong-region correction (the reference's
    default): the same bound as without it, the spread measured by the oracle
    running the correction under the same perturbations (a perturbation that
    flips a control point's outlier status or the keep / discard choice shows
    up there as spread).  The device log must hold the updates of every pass
    the oracle ran (one pass, or three when a trap was built).  Both exclusion
    modes: "direct" (the default) and "highresidual", and non-default options
    (metric "mae", thresholds, radii, sigma_grad 0 and 1.6)."""
    from oracle import xres_oracle as X
    from wholistic_registration_b200 import calFlowCrossResolution as C

    loader = {"direct": load_xres_wr_case, "highresidual": load_xres_hr_case, "options": load_xres_opt_case}[kind]
    arrays, option = loader(name)
    phase, motion, sampled = C.getMotion_v2(arrays["mov"], arrays["ref"], dict(option))
    _, _, _, log = X.get_motion_v2(arrays["mov"], arrays["ref"], dict(option))
    dev_log, _ = C.last_registrar.error_log()
    want = _updates_per_level(log)
    got = {int(k.split("_")[1]): len(v["max_diff_motion"]) for k, v in dev_log.items()}
    assert got == want, f"updates per level {got} vs reference {want}"
    spread = _reference_spread(arrays, option, arrays["motion"])
    bound = 1e-3 + 3.0 * spread
    err_m = np.abs(motion - arrays["motion"])
    err_p = np.abs(phase - arrays["phase"])
    assert (err_m > bound).mean() <= 1e-3, f"motion: max excess {float((err_m - bound).max()):.3g}"
    assert (err_p > bound).mean() <= 1e-3, f"phase: max excess {float((err_p - bound).max()):.3g}"
    span = float(np.ptp(arrays["ref_sampled"])) or 1.0
    own = X.cubic_sample_scipy(arrays["ref"].astype(np.float64), phase[..., 0], phase[..., 1], phase[..., 2])
    np.testing.assert_allclose(sampled, own, rtol=0, atol=1e-4 * span)


def _projection_case(seed=5):
    rng = np.random.default_rng(seed)
    X, Y, K = 20, 18, 4
    coords = np.stack([rng.uniform(-2, 22, (X, Y, K)), rng.uniform(-2, 20, (X, Y, K)),
                       rng.uniform(-1, 7, (X, Y, K))], -1).astype(np.float32)
    values = rng.normal(50, 80, (X, Y, K)).astype(np.float32)
    values[0, 0, 0] = np.nan
    coords[1, 1, 1, 0] = np.inf
    ref = rng.normal(100, 20, (21, 19, 6)).astype(np.float32)
    return coords, values, ref


@pytest.mark.parametrize("mode,extra,ds", [("subpixel_footprint", 0, 1), ("subpixel_footprint", 1, 2), ("nearest", 0, 3)])
def test_projection_max_matches_restatement(mode, extra, ds):
    from oracle import xres_oracle as X
    from wholistic_registration_b200 import calFlowCrossResolution as C

    coords, values, ref = _projection_case()
    planes = [0.0, 2.5, 5.0]
    got = C.project_coords_to_fixed_planes_gpu(coords, ref, planes, values_xyk=values, z_window=1.2,
                                               downsample_xy=ds, fill_value=-7.0, return_numpy=True,
                                               output_order="zxy", xy_splat_mode=mode, xy_extra_radius=extra)
    want = X.project_max(values, coords, planes, ref.shape[0], ref.shape[1], ds, 1.2, mode == "nearest", extra, -7.0)
    np.testing.assert_array_equal(got, want)
    zyx = C.project_coords_to_fixed_planes_gpu(coords, ref, planes, values_xyk=values, z_window=1.2,
                                               downsample_xy=ds, fill_value=-7.0, return_numpy=True,
                                               xy_splat_mode=mode, xy_extra_radius=extra)
    np.testing.assert_array_equal(zyx, want.transpose(0, 2, 1))


@pytest.mark.parametrize("wmode", ["hard", "triangular", "gaussian"])
def test_projection_weighted_matches_restatement(wmode):
    from oracle import xres_oracle as X
    from wholistic_registration_b200 import calFlowCrossResolution as C

    coords, values, ref = _projection_case(6)
    planes = [1.0, 3.0]
    out, w = C.project_coords_to_fixed_planes_weighted_gpu(coords, ref, planes, values_xyk=values, z_window=1.5,
                                                           z_weight_mode=wmode, downsample_xy=2, return_numpy=True,
                                                           output_order="zxy")
    want, want_w = X.project_weighted(values, coords, planes, ref.shape[0], ref.shape[1], 2, 1.5, None,
                                      {"hard": 0, "triangular": 1, "gaussian": 2}[wmode])
    np.testing.assert_allclose(w, want_w, rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(out, want, rtol=1e-4, atol=1e-3)


def test_continuous_H_matches_scipy():
    """Spline values H(coords) from the device prefilter and sampler against
    SciPy's map_coordinates (the library call the reference makes)."""
    from oracle import xres_oracle as X
    from wholistic_registration_b200 import calFlowCrossResolution as C

    coords, _, ref = _projection_case(7)
    H = C.generate_continuous_H_gpu(ref, zRatio=2.0)
    got = C.apply_H_to_matrix_gpu(torch.from_numpy(coords).cuda(), H).cpu().numpy()
    want = X.cubic_sample_scipy(ref.astype(np.float64), coords[..., 0], coords[..., 1], coords[..., 2] / 2.0)
    fin = np.isfinite(want)
    np.testing.assert_allclose(got[fin], want[fin], rtol=1e-6, atol=1e-4)


def test_projection_samples_reference_when_values_absent():
    from oracle import xres_oracle as X
    from wholistic_registration_b200 import calFlowCrossResolution as C

    coords, _, ref = _projection_case(8)
    coords[1, 1, 1, 0] = 3.0
    planes = [2.0]
    got = C.project_coords_to_fixed_planes_gpu(coords, ref, planes, z_window=1.0, return_numpy=True,
                                               output_order="zxy")
    vals = X.cubic_sample_scipy(ref.astype(np.float64), coords[..., 0], coords[..., 1], coords[..., 2]).astype(np.float32)
    want = X.project_max(vals, coords, planes, ref.shape[0], ref.shape[1], 1, 1.0, False, 0, 0.0)
    np.testing.assert_allclose(got, want, rtol=1e-5, atol=1e-3)


def test_projection_matches_reference_kernels():
    """The device max and weighted splats against the reference's own
    projection kernels (fixtures from tests/golden/make_projection_golden.py):
    the max splat bit for bit, the weighted one within float32 atomic
    accumulation order (2e-6 of the largest output)."""
    from conftest import projection_ref_cases
    from wholistic_registration_b200 import calFlowCrossResolution as C

    for name, c in projection_ref_cases():
        p = c["params"]
        xr, yr = int(p[0]), int(p[1])
        ref = np.zeros((xr, yr, 6), np.float32)   # only its (x, y) extent is used when values are given
        if name.startswith("max"):
            _, _, zw, near, extra, ds, fill = p
            got = C.project_coords_to_fixed_planes_gpu(c["coords"], ref, c["planes"], values_xyk=c["values"],
                                                       z_window=float(zw), downsample_xy=int(ds), fill_value=float(fill),
                                                       return_numpy=True, output_order="zxy",
                                                       xy_splat_mode="nearest" if near else "subpixel_footprint",
                                                       xy_extra_radius=int(extra))
            np.testing.assert_array_equal(got, c["out"], err_msg=name)
        else:
            _, _, zw, zs, wm, ds, fill, eps = p
            mode = {0: "hard", 1: "triangular", 2: "gaussian"}[int(wm)]
            out, w = C.project_coords_to_fixed_planes_weighted_gpu(
                c["coords"], ref, c["planes"], values_xyk=c["values"], z_window=float(zw),
                z_sigma=None if zs < 0 else float(zs), z_weight_mode=mode, downsample_xy=int(ds),
                fill_value=float(fill), return_numpy=True, output_order="zxy", eps=float(eps))
            np.testing.assert_allclose(out, c["out"], rtol=0, atol=2e-6 * float(np.abs(c["out"]).max()),
                                       err_msg=name)
            np.testing.assert_allclose(w, c["sum_w"], rtol=0, atol=2e-6 * float(c["sum_w"].max()), err_msg=name)


def _impulse_pair(mov_shape, ref_shape, zr, zr_hr, seed):
    """Moving and reference stacks cut at z spacings zr and zr_hr from one
    blurred random-impulse field (physical z step 0.5), the moving one shifted
    by a smooth in-plane field and Poisson-noised.  (x, y, z) float32."""
    from scipy import ndimage

    rng = np.random.default_rng(seed)
    nzf = int(max(mov_shape[2] * zr, ref_shape[2] * zr_hr) / 0.5) + 8
    field = np.zeros((mov_shape[0] + 8, mov_shape[1] + 8, nzf), np.float64)
    k = field.size // 60
    field.flat[rng.choice(field.size, k, replace=False)] = rng.uniform(2e3, 2e4, k)
    field = ndimage.gaussian_filter(field, (2.0, 2.0, 3.0)) + 100.0

    def cut(shape, zs, dx=0.0, dy=0.0):
        X, Y, Z = np.meshgrid(*[np.arange(n, dtype=np.float64) for n in shape], indexing="ij")
        pts = np.stack([X + 4 + dx, Y + 4 + dy, Z * zs / 0.5 + 4])
        return ndimage.map_coordinates(field, pts, order=1, mode="nearest")

    X, Y = np.meshgrid(np.arange(mov_shape[0]), np.arange(mov_shape[1]), indexing="ij")
    dx = (1.2 * np.sin(2 * np.pi * Y / 37.0 + 0.3) + 0.5)[..., None]
    dy = (1.0 * np.cos(2 * np.pi * X / 41.0) - 0.4)[..., None]
    mov = rng.poisson(cut(mov_shape, zr, dx, dy)).astype(np.float32)
    ref = rng.poisson(cut(ref_shape, zr_hr)).astype(np.float32)
    return mov, ref


def test_xres_wrong_region_many_control_points():
    """More control points per slice (80 x 80 at r 1) than the detection's
    shared-memory working set holds: the per-slice median / MAD and
    components run on global scratch.  Against the oracle with the spread
    bound; the oracle must have built a trap (regions found, re-runs done)."""
    from oracle import xres_oracle as X
    from wholistic_registration_b200 import calFlowCrossResolution as C

    mov, ref = _impulse_pair((240, 240, 3), (240, 240, 5), 2.0, 1.0, 11)
    option = {"mask_ref": np.zeros(ref.shape, np.uint8), "mask_mov": np.zeros(mov.shape, np.uint8), "layer": 0,
              "iter": 6, "r": 1, "zRatio": 2.0, "zRatio_HR": 1.0, "smoothPenalty": 0.05, "movRange": 5.0, "tol": 1e-3,
              "motion": None, "wrong_region_enable": True}
    phase_o, motion_o, _, log = X.get_motion_v2(mov, ref, dict(option))
    assert log["layer_0"]["wrong_region"]["regions"] > 0 and "error2" in log["layer_0"]["wrong_region"]
    phase, motion, _ = C.getMotion_v2(mov, ref, dict(option))
    dev_log, _ = C.last_registrar.error_log()
    assert len(dev_log["layer_0"]["max_diff_motion"]) == len(log["layer_0"]["max_diff_motion"])
    spread = _reference_spread({"mov": mov, "ref": ref}, option, motion_o)
    bound = 1e-3 + 3.0 * spread
    err = np.abs(motion - motion_o)
    assert (err > bound).mean() <= 1e-3, f"motion: max excess {float((err - bound).max()):.3g}"
