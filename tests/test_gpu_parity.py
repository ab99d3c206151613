"""Parity of the CUDA path (through the C ABI) with the reference's outputs.

Bars (see the package docs): displacement within 1e-3 voxel max-abs and
warped volumes within 1e-4 relative L2 of the reference; when the stopping
rules flip on a borderline decision the per-level update counts of the
reference run are replayed (``forced_updates``) and the same bars apply.
"""

from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import GOLDEN, load_motion_case, motion_case_names, option_from_case, updates_per_layer

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

FLOW_TOL = 1e-3     # voxel, max-abs
WARP_TOL = 1e-4     # relative L2


def _cf3():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from wholistic_registration_b200 import calFlow3d_Wei_v1

    return calFlow3d_Wei_v1


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.parametrize("name", motion_case_names())
def test_get_motion_matches_reference_fixture(name):
    cf3 = _cf3()
    arrays, meta = load_motion_case(name)
    option = option_from_case(arrays, meta)
    motion, err, coords, log = cf3.getMotion(arrays["mov"], arrays["ref"], option)
    ref_counts = {l: len(arrays[f"layer_{l}/currentError"]) for l in range(meta["layer"] + 1)}
    counts = {l: len(log[f"layer_{l}"]["currentError"]) for l in range(meta["layer"] + 1)}
    if counts != ref_counts:
        option = option_from_case(arrays, meta)
        option["forced_updates"] = updates_per_layer(arrays, meta)
        motion, err, coords, log = cf3.getMotion(arrays["mov"], arrays["ref"], option)
    assert motion.shape == arrays["motion"].shape and motion.dtype == np.float32
    dmax = float(np.abs(motion - arrays["motion"]).max())
    assert dmax <= FLOW_TOL, f"{name}: max |dflow| {dmax:.3g} (counts {counts} vs {ref_counts})"
    for l in range(meta["layer"] + 1):
        np.testing.assert_allclose(log[f"layer_{l}"]["currentError"][:len(arrays[f"layer_{l}/currentError"])],
                                   arrays[f"layer_{l}/currentError"][:len(log[f"layer_{l}"]["currentError"])],
                                   rtol=1e-4)
    warped = cf3.correctMotion(arrays["mov"].astype(np.float32), motion)
    assert rel_l2(warped, arrays["warped"]) <= WARP_TOL


def test_stopping_rules_reach_reference_counts():
    """Without replay, the device-side stopping rules give the reference's
    per-level iteration counts on most fixtures."""
    cf3 = _cf3()
    same = 0
    names = motion_case_names()
    for name in names:
        arrays, meta = load_motion_case(name)
        _, _, _, log = cf3.getMotion(arrays["mov"], arrays["ref"], option_from_case(arrays, meta))
        same += all(len(log[f"layer_{l}"]["currentError"]) == len(arrays[f"layer_{l}/currentError"])
                    for l in range(meta["layer"] + 1))
    assert same >= len(names) - 1


def test_correct_motion_matches_reference_fixture():
    cf3 = _cf3()
    prim = dict(np.load(os.path.join(GOLDEN, "primitives.npz")))
    out = cf3.correctMotion(prim["warp_in"], prim["warp_motion"])
    assert out.dtype == np.float32
    np.testing.assert_allclose(out, prim["warp_out"], rtol=2e-7, atol=1e-4)
    u16 = np.clip(prim["warp_in"], 0, 65535).astype(np.uint16)
    np.testing.assert_allclose(cf3.correctMotion(u16, prim["warp_motion"]),
                               cf3.correctMotion(u16.astype(np.float32), prim["warp_motion"]), rtol=0, atol=0)


def test_penalty_factor_matches_reference_fixture():
    _cf3()
    from wholistic_registration_b200 import penalty_factor

    arrays, _ = load_motion_case("mask_r3_l1_z2")
    ref = torch.from_numpy(np.ascontiguousarray(arrays["ref"].astype(np.float32).transpose(2, 1, 0))).cuda()
    mref = torch.from_numpy(np.ascontiguousarray(arrays["mask_ref"].transpose(2, 1, 0))).cuda()
    f = float(penalty_factor(ref, mref))
    np.testing.assert_allclose(f, float(arrays["penalty_factor"]), rtol=1e-12)


def _oracle_case(shape_zyx, seed, r, layer, zratio=1.0, mask=False, max_disp=(3.0, 3.0, 1.0), blobs=600):
    from oracle import lk_oracle as O
    from wholistic_registration_b200 import synthetic

    tmpl, mov, field = synthetic.make_pair(shape_zyx, seed, n_blobs=blobs, max_disp=max_disp)
    t = tmpl.to(torch.int32).numpy().astype(np.uint16).transpose(2, 1, 0)
    m = mov.to(torch.int32).numpy().astype(np.uint16).transpose(2, 1, 0)
    shape = t.shape
    if mask:
        excl = ~synthetic.ellipsoid_inclusion(shape_zyx, 0.7).numpy().transpose(2, 1, 0)
    else:
        excl = np.zeros(shape, bool)
    factor = O.smooth_penalty_norm_factor(t.astype(np.float64), excl)
    option = {"mask_ref": excl, "mask_mov": excl, "layer": layer, "iter": 10, "r": r, "zRatio": zratio,
              "movRange": 5.0, "motion": None, "smoothPenalty": float(factor * 0.08), "tol": 1e-3, "save_ite": 100}
    return t, m, option


@pytest.mark.parametrize("shape,r,layer,zr,mask", [
    ((16, 128, 128), 8, 2, 1.0, False),
    ((12, 96, 160), 5, 2, 2.0, True),
])
def test_against_oracle_medium(shape, r, layer, zr, mask):
    cf3 = _cf3()
    from oracle import lk_oracle as O

    t, m, option = _oracle_case(shape, 11, r, layer, zr, mask)
    om, oe, _, olog = O.get_motion(m, t, dict(option))
    gm, ge, _, glog = cf3.getMotion(m, t, dict(option))
    ocounts = {l: len(olog[f"layer_{l}"]["max_diff_motion"]) for l in range(layer + 1)}
    gcounts = {l: len(glog[f"layer_{l}"]["max_diff_motion"]) for l in range(layer + 1)}
    if ocounts != gcounts:
        opt = dict(option)
        opt["forced_updates"] = ocounts
        gm, ge, _, glog = cf3.getMotion(m, t, opt)
    assert float(np.abs(gm - om).max()) <= FLOW_TOL
    w_o = O.correct_motion(m.astype(np.float32), om)
    w_g = cf3.correctMotion(m.astype(np.float32), gm)
    assert rel_l2(w_g, w_o) <= WARP_TOL


def test_deterministic_and_torch_path():
    cf3 = _cf3()
    arrays, meta = load_motion_case("r5_l2_big")
    option = option_from_case(arrays, meta)
    a = cf3.getMotion(arrays["mov"], arrays["ref"], dict(option))[0]
    b = cf3.getMotion(arrays["mov"], arrays["ref"], dict(option))[0]
    np.testing.assert_array_equal(a, b)
    mov = torch.from_numpy(arrays["mov"].astype(np.float32)).cuda()
    ref = torch.from_numpy(arrays["ref"].astype(np.float32)).cuda()
    c, err, coords, _ = cf3.getMotion(mov, ref, dict(option))
    assert isinstance(c, torch.Tensor) and c.is_cuda and tuple(c.shape) == a.shape
    np.testing.assert_array_equal(c.cpu().numpy(), a)
    grid = np.stack(np.meshgrid(*[np.arange(n, dtype=np.float32) for n in a.shape[:3]], indexing="ij"), -1)
    np.testing.assert_allclose(np.asarray(coords), a + grid)


def test_argument_errors_raise_value_error():
    cf3 = _cf3()
    arrays, meta = load_motion_case("tiny_r1_l0")
    option = option_from_case(arrays, meta)
    with pytest.raises(ValueError):
        cf3.getMotion(arrays["mov"][:-1], arrays["ref"], dict(option))
    bad = dict(option)
    bad["r"] = 0
    with pytest.raises(ValueError):
        cf3.getMotion(arrays["mov"], arrays["ref"], bad)
    big = dict(option)
    big["layer"] = 4
    with pytest.raises(ValueError):
        cf3.getMotion(arrays["mov"], arrays["ref"], big)


def test_reuse_reference_matches_fresh_registration():
    """Registering a second frame with the template pyramid kept from the
    first call gives the same field as a fresh registration."""
    _cf3()
    from wholistic_registration_b200 import LKParams, LKRegistrar, synthetic

    shape = (8, 96, 80)
    tmpl, mov1, _ = synthetic.make_pair(shape, 21, n_blobs=300, max_disp=(2.5, 2.5, 0.8))
    _, mov2, _ = synthetic.make_pair(shape, 22, n_blobs=300, max_disp=(2.5, 2.5, 0.8), template=tmpl.float())
    excl = (~synthetic.ellipsoid_inclusion(shape, 0.75)).to(torch.uint8)
    t, m1, m2, e = (x.cuda().contiguous() for x in (tmpl, mov1, mov2, excl))
    p = LKParams(layer=2, iter=10, r=4, zRatio=1.0, movRange=5.0, smoothPenalty=200.0, tol=1e-3)
    a = LKRegistrar(shape, p)
    a.register(m1, t, e, e)
    kept = a.register(m2, t, e, e, reuse_reference=True).clone()
    b = LKRegistrar(shape, p)
    fresh = b.register(m2, t, e, e)
    torch.testing.assert_close(kept, fresh, rtol=0, atol=0)


@pytest.mark.parametrize("shape,layer", [((8, 96, 80), 2), ((6, 70, 66), 0)])
def test_register_and_warp_in_one_call_matches_two_calls(shape, layer):
    """wr_lk_register_warp gives exactly the motion of wr_lk_register and the
    volume of wr_warp_trilinear on that motion (correctMotion)."""
    _cf3()
    from wholistic_registration_b200 import LKParams, LKRegistrar, synthetic, warp

    tmpl, mov, _ = synthetic.make_pair(shape, 31, n_blobs=300, max_disp=(2.5, 2.5, 0.8))
    excl = (~synthetic.ellipsoid_inclusion(shape, 0.75)).to(torch.uint8)
    t, m, e = (x.cuda().contiguous() for x in (tmpl, mov, excl))
    p = LKParams(layer=layer, iter=1 if layer == 0 else 10, r=4, zRatio=1.0, movRange=5.0, smoothPenalty=200.0,
                 tol=1e-3)
    reg = LKRegistrar(shape, p)
    motion = reg.register(m, t, e, e).clone()
    warped = warp(m, motion)
    warped_fused = torch.empty(shape, dtype=torch.float32, device="cuda")
    motion_fused = reg.register(m, t, e, e, warped_out=warped_fused).clone()
    torch.testing.assert_close(motion_fused, motion, rtol=0, atol=0)
    torch.testing.assert_close(warped_fused, warped, rtol=0, atol=0)


@pytest.mark.parametrize("precision,rms_tol", [(1, 2.5e-3), (2, 1.5e-2)])   # about twice the B200 errors
def test_mixed_precision_error_against_fp64_oracle(precision, rms_tol):
    """Levels and gradients stored in float16 (1) or bfloat16 (2), sums and
    solves in float32: flow error against the float64 oracle of the method."""
    cf3 = _cf3()
    from oracle import lk_oracle as O

    t, m, option = _oracle_case((16, 128, 128), 11, 8, 2, 1.0, True)
    om, _, _, olog = O.get_motion(m, t, dict(option))
    opt = dict(option)
    opt["precision"] = precision
    opt["forced_updates"] = {l: len(olog[f"layer_{l}"]["max_diff_motion"]) for l in range(3)}
    gm, _, _, _ = cf3.getMotion(m, t, opt)
    err = gm - om
    rms = float(np.sqrt(np.mean(err ** 2)))
    print(f"precision {precision}: flow RMS {rms:.3e} vox, max {np.abs(err).max():.3e} vox")
    assert rms <= rms_tol
    w_o = O.correct_motion(m.astype(np.float32), om)
    w_g = cf3.correctMotion(m.astype(np.float32), gm)
    assert rel_l2(w_g, w_o) <= 10 * rms_tol


def test_fp64_fallback_for_ill_conditioned_patches():
    """Without smoothness penalty a near-uniform slab makes the structure
    tensor singular: the mixed path re-solves those patches in float64."""
    _cf3()
    from wholistic_registration_b200 import LKParams, LKRegistrar, synthetic

    shape = (8, 96, 96)
    tmpl, mov, _ = synthetic.make_pair(shape, 31, n_blobs=200, max_disp=(2.0, 2.0, 0.5))
    t, mv = tmpl.cuda().float(), mov.cuda().float()
    t[:, 40:60, :] = 100.0
    mv[:, 40:60, :] = 100.0
    p = LKParams(layer=1, iter=6, r=4, zRatio=1.0, movRange=5.0, smoothPenalty=0.0, tol=1e-3,
                 precision=1, forced_updates={0: 5, 1: 5})
    reg = LKRegistrar(shape, p)
    out = reg.register(mv.contiguous(), t.contiguous())
    st = reg.stats()
    assert st.fp64_solves > 0
    assert bool(torch.isfinite(out).all())
