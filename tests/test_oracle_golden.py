"""The CPU oracle against fixtures produced by running the reference itself."""

from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import (GOLDEN, load_motion_case, load_xres_case, load_xres_hr_case, load_xres_opt_case,
                      load_xres_wr_case, motion_case_names, option_from_case, xres_case_names, xres_hr_case_names,
                      xres_opt_case_names, xres_wr_case_names)
from oracle import lk_oracle as O

PRIM = os.path.join(GOLDEN, "primitives.npz")


@pytest.fixture(scope="module")
def prim():
    return dict(np.load(PRIM))


def test_imresize_bicubic_matches_reference(prim):
    vol = prim["resize_in"]
    for i, shp in enumerate([(18, 25, 5), (9, 12, 5), (4, 6, 5), (37, 50, 5)]):
        np.testing.assert_allclose(O.imresize(vol, shp), prim[f"resize_bicubic_{i}"], rtol=0, atol=1e-9)


def test_imresize_integer_and_mask_inputs(prim):
    np.testing.assert_allclose(O.imresize(prim["resize_u16_in"], (16, 10, 4)), prim["resize_u16_out"], atol=1e-9)
    out8 = O.imresize(prim["resize_u8_in"], (10, 9, 3))
    assert out8.dtype == np.uint8
    np.testing.assert_array_equal(out8, prim["resize_u8_out"])
    m = O.imresize(prim["resize_mask_in"], (10, 9, 4))
    np.testing.assert_allclose(m, prim["resize_mask_out"], atol=1e-12)
    np.testing.assert_array_equal(m > 0, prim["resize_mask_out"] > 0)


def test_imresize_bilinear_upsample(prim):
    out = O.imresize(prim["resize_bilinear_in"], (37, 50, 5), method="bilinear")
    np.testing.assert_allclose(out, prim["resize_bilinear_out"], atol=1e-12)


def test_correct_motion_matches_reference(prim):
    out = O.correct_motion(prim["warp_in"], prim["warp_motion"])
    assert out.dtype == np.float32
    np.testing.assert_array_equal(out, prim["warp_out"])


def test_solve_and_neighbour_difference(prim):
    comps = [prim[f"solve_in_{i}"] for i in range(9)]
    keys = ["xx", "xy", "xz", "yy", "yz", "zz", "xt", "yt", "zt"]
    v = O.solve_flow_with_penalty(dict(zip(keys, comps)), 0.7, prim["solve_nei"])
    np.testing.assert_allclose(v, prim["solve_out"], rtol=1e-10, atol=1e-12)
    # the adjugate solve is a linear solve: check against numpy on one CP
    a = np.array([[comps[0][0, 0, 0] + 0.7, comps[1][0, 0, 0], comps[2][0, 0, 0]],
                  [comps[1][0, 0, 0], comps[3][0, 0, 0] + 0.7, comps[4][0, 0, 0]],
                  [comps[2][0, 0, 0], comps[4][0, 0, 0], comps[5][0, 0, 0] + 0.7]])
    b = np.array([comps[6][0, 0, 0], comps[7][0, 0, 0], comps[8][0, 0, 0]]) + prim["solve_nei"][0, 0, 0]
    np.testing.assert_allclose(v[0, 0, 0], np.linalg.solve(a, b), rtol=1e-9)
    nd = O.get_nei_diff(prim["neidiff_in"])
    np.testing.assert_allclose(nd, prim["neidiff_out"], rtol=0, atol=2e-7)


def test_box_filter(prim):
    np.testing.assert_allclose(O.box_filter_nearest(prim["box_in"], 5, 3), prim["box_out_5x3"], atol=1e-12)


@pytest.mark.parametrize("name", motion_case_names())
def test_get_motion_matches_reference(name):
    arrays, meta = load_motion_case(name)
    option = option_from_case(arrays, meta)
    motion, err, coords, log = O.get_motion(arrays["mov"], arrays["ref"], option)
    for l in range(meta["layer"] + 1):
        key = f"layer_{l}"
        assert len(log[key]["currentError"]) == len(arrays[f"{key}/currentError"]), key
        np.testing.assert_allclose(log[key]["currentError"], arrays[f"{key}/currentError"], rtol=1e-6)
        np.testing.assert_allclose(log[key]["max_diff_motion"], arrays[f"{key}/max_diff_motion"], atol=1e-5)
    assert np.abs(motion - arrays["motion"]).max() < 1e-4
    np.testing.assert_allclose(err, float(arrays["current_error"]), rtol=1e-6)
    warped = O.correct_motion(arrays["mov"].astype(np.float32), arrays["motion"])
    # float64 trilinear rounded to float32: summation order may move 1 ulp
    np.testing.assert_allclose(warped, arrays["warped"], rtol=1e-6, atol=0)


@pytest.mark.parametrize("name", ["c0slab_8x256x256_l2", "c1slab_4x512x512_l3"])
def test_oracle_matches_reference_at_benchmarked_configuration(name):
    """r = 16 (33 x 33 patches), 70 % ellipsoid mask, 3 and 4 levels: the
    oracle reproduces the reference's run (the two smaller benchmarked-
    configuration fixtures; the GPU tests use all four)."""
    import sys

    sys.path.insert(0, GOLDEN)
    from bench_cases import BENCH_CASES, bench_inputs, bench_option

    d = dict(np.load(os.path.join(GOLDEN, f"bench_{name}.npz")))
    tmpl, mov, excl, digest = bench_inputs(name)
    assert digest == str(d["sha256"])
    layer = BENCH_CASES[name][4]
    option = bench_option(name, float(d["smooth_penalty"]))
    option["mask_ref"], option["mask_mov"] = excl.copy(), excl.copy()
    motion, err, _, log = O.get_motion(mov, tmpl, option)
    for l in range(layer + 1):
        key = f"layer_{l}"
        assert len(log[key]["currentError"]) == len(d[f"{key}/currentError"]), key
        np.testing.assert_allclose(log[key]["currentError"], d[f"{key}/currentError"], rtol=1e-6)
    s = int(d["stride"])
    assert np.abs(motion[::s, ::s] - d["motion_sub"]).max() < 1e-4
    np.testing.assert_allclose(err, float(d["current_error"]), rtol=1e-6)


def test_penalty_factor():
    arrays, meta = load_motion_case("mask_r3_l1_z2")
    f = O.smooth_penalty_norm_factor(arrays["ref"].astype(np.float64), arrays["mask_ref"])
    np.testing.assert_allclose(f, float(arrays["penalty_factor"]), rtol=1e-12)


MASK_CASES = ("mask_a", "mask_b", "mask_c")


@pytest.mark.parametrize("name", MASK_CASES)
def test_mask_oracle_matches_reference_fixture(name):
    from oracle import mask_oracle as M

    d = np.load(os.path.join(GOLDEN, "masks.npz"))
    vol = d[f"{name}_vol"]
    thres, lo, hi = d[f"{name}_params"]
    mu, sg = M.robust_mean_std(vol.astype(np.float32))
    np.testing.assert_array_equal(np.array([mu, sg], np.float32), d[f"{name}_musig"])
    m = M.get_mask(vol, float(thres))
    np.testing.assert_array_equal(m, d[f"{name}_mask"])
    f, _ = M.bwareafilt3(m, (lo, hi))
    np.testing.assert_array_equal(f, d[f"{name}_filtered"])


@pytest.mark.parametrize("name", xres_case_names())
def test_xres_oracle_matches_reference(name):
    """The getMotion_v2 restatement reproduces the reference's run on the
    same inputs (phase, motion, sampled reference)."""
    from oracle import xres_oracle as X

    arrays, option = load_xres_case(name)
    phase, motion, sampled, _ = X.get_motion_v2(arrays["mov"], arrays["ref"], option)
    np.testing.assert_allclose(motion, arrays["motion"], rtol=0, atol=1e-6)
    np.testing.assert_allclose(phase, arrays["phase"], rtol=0, atol=1e-6)
    np.testing.assert_allclose(sampled, arrays["ref_sampled"], rtol=1e-12, atol=1e-9)


def test_xres_spline_restatement_matches_scipy():
    """Edge padding + recursive cubic B-spline prefilter + 64-tap evaluation
    (the CUDA path's algorithm) against scipy's map_coordinates(order=3,
    mode="nearest") for coordinates inside, near and beyond the faces."""
    from oracle import xres_oracle as X

    rng = np.random.default_rng(3)
    vol = rng.normal(100.0, 30.0, size=(13, 9, 6))
    coef = X.bspline_coefficients(vol)
    # inside and a few voxels beyond the faces the two agree to rounding; more
    # than the 12-voxel padding beyond a face only the prefilter's start-up at
    # the padded ends differs, damped by 0.268^12 (relative 1e-7)
    for lo, hi, tol in ((0.0, 0.0, 1e-11), (-4.0, 4.0, 1e-11), (-40.0, 40.0, 3e-7)):
        pts = [rng.uniform(lo, n - 1 + hi, 3000) for n in vol.shape]
        got = X.cubic_sample(coef, *pts)
        want = X.cubic_sample_scipy(vol, *pts)
        np.testing.assert_allclose(got, want, rtol=0, atol=tol * np.abs(vol).max())


@pytest.mark.parametrize("name", xres_wr_case_names())
def test_xres_wrong_region_oracle_matches_reference(name):
    """getMotion_v2 with the wrong-region correction: the restatement
    reproduces the reference's run (detection, trap mask, re-runs, choice)."""
    from oracle import xres_oracle as X

    arrays, option = load_xres_wr_case(name)
    phase, motion, sampled, _ = X.get_motion_v2(arrays["mov"], arrays["ref"], option)
    np.testing.assert_allclose(motion, arrays["motion"], rtol=0, atol=1e-6)
    np.testing.assert_allclose(phase, arrays["phase"], rtol=0, atol=1e-6)
    np.testing.assert_allclose(sampled, arrays["ref_sampled"], rtol=1e-12, atol=1e-9)


@pytest.mark.parametrize("name", xres_hr_case_names())
def test_xres_high_residual_oracle_matches_reference(name):
    """getMotion_v2 with the "highresidual" exclusion mode: the restatement
    reproduces the reference's run.  Its bad-voxel and trap masks equal the
    reference's; in one case the re-runs differ from the reference's by
    summation-order rounding (motion <= 7.2e-7 in 4 % of the voxels, phase one
    float32 ulp), hence 1e-5 here against 1e-6 for the other fixtures."""
    from oracle import xres_oracle as X

    arrays, option = load_xres_hr_case(name)
    phase, motion, sampled, log = X.get_motion_v2(arrays["mov"], arrays["ref"], option)
    np.testing.assert_allclose(motion, arrays["motion"], rtol=0, atol=1e-5)
    np.testing.assert_allclose(phase, arrays["phase"], rtol=0, atol=1e-5)
    # the sampled reference moves by its gradient times that phase ulp
    span = float(np.ptp(arrays["ref_sampled"]))
    np.testing.assert_allclose(sampled, arrays["ref_sampled"], rtol=0, atol=1e-6 * span)


def test_projection_oracle_matches_reference_kernels():
    """The oracle's max and weighted splats against the reference's own
    projection kernels (compiled from its source, run with its wrappers'
    steps): the max splat bit for bit, the weighted one within float32
    atomic-accumulation order (2e-6 of the largest output; the oracle sums in
    float64)."""
    from conftest import projection_ref_cases
    from oracle import xres_oracle as X

    cases = projection_ref_cases()
    assert len(cases) == 8
    for name, c in cases:
        p = c["params"]
        if name.startswith("max"):
            xr, yr, zw, near, extra, ds, fill = p
            got = X.project_max(c["values"], c["coords"], c["planes"], int(xr), int(yr), int(ds), float(zw),
                                bool(near), int(extra), float(fill))
            np.testing.assert_array_equal(got, c["out"], err_msg=name)
        else:
            xr, yr, zw, zs, wm, ds, fill, eps = p
            got, w = X.project_weighted(c["values"], c["coords"], c["planes"], int(xr), int(yr), int(ds), float(zw),
                                        None if zs < 0 else float(zs), int(wm), float(fill), float(eps))
            np.testing.assert_allclose(got, c["out"], rtol=0, atol=2e-6 * float(np.abs(c["out"]).max()),
                                       err_msg=name)
            np.testing.assert_allclose(w, c["sum_w"], rtol=0, atol=2e-6 * float(c["sum_w"].max()), err_msg=name)


@pytest.mark.parametrize("name", xres_opt_case_names())
def test_xres_wrong_region_options_oracle_matches_reference(name):
    """getMotion_v2 with the wrong-region correction at non-default options
    (metric "mae", MAD threshold, minimum component size, expand radius,
    intensity_k, sigma_grad 0 and 1.6): the restatement reproduces the
    reference's run."""
    from oracle import xres_oracle as X

    arrays, option = load_xres_opt_case(name)
    phase, motion, sampled, _ = X.get_motion_v2(arrays["mov"], arrays["ref"], option)
    np.testing.assert_allclose(motion, arrays["motion"], rtol=0, atol=1e-5)
    np.testing.assert_allclose(phase, arrays["phase"], rtol=0, atol=1e-5)
    span = float(np.ptp(arrays["ref_sampled"]))
    np.testing.assert_allclose(sampled, arrays["ref_sampled"], rtol=0, atol=1e-6 * span)
