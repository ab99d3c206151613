"""The per-batch wrappers on the device: wbi_registration_3d's masks are the
mask oracle's, its motions and corrected frames those of LKRegistrar with
those masks, its errors NumPy's; template picking follows the reference's
pick_initial_reference restated in NumPy; wbi_registration_2d is the stacked
3-D registration."""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _need():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _config(pick=False, dual=False):
    return {
        "channels": {"dual_channel": dual, "function": "log10", "k": 30},
        "reference": {"pick_reference_auto": pick, "chunk_size": 2},
        "mask": {"thresFactor": 3.0, "maskRange": [5, 4000]},
        "pyramid": {"layer": 1, "iter": 10, "r": 4, "smoothPenalty": 0.08, "tolerance": 1e-3},
        "MetaData": {"zRatio": 1.0},
    }


def _batch(n=3, shape=(6, 64, 64), seed=7):
    from wholistic_registration_b200 import synthetic

    tmpl, _, _ = synthetic.make_pair(shape, seed, n_blobs=250, max_disp=(2.0, 2.0, 0.6))
    frames = [synthetic.make_pair(shape, seed + 1 + k, n_blobs=250, max_disp=(2.0, 2.0, 0.6),
                                  template=tmpl.float())[1] for k in range(n)]
    to_np = lambda t: t.to(torch.int32).numpy().astype(np.uint16)
    return to_np(tmpl), np.stack([to_np(f) for f in frames])


def test_wrapper_matches_its_parts():
    _need()
    from oracle import mask_oracle as M
    from wholistic_registration_b200 import LKParams, LKRegistrar, penalty_factor
    from wholistic_registration_b200.registration import wbi_registration_3d

    ref, frames = _batch()
    cfg = _config()
    mem_out, ca_out, dat_ref, errors, motions = wbi_registration_3d(frames, cfg, reference_image=ref, verbose=False)
    assert mem_out.shape == frames.shape and motions.shape == frames.shape + (3,) and ca_out.size == 0
    np.testing.assert_array_equal(dat_ref, ref.transpose(2, 1, 0))
    rng = tuple(cfg["mask"]["maskRange"])
    mref = M.bwareafilt3(M.get_mask(ref.transpose(2, 1, 0), 3.0), rng)[0].transpose(2, 1, 0)
    t = torch.from_numpy(ref).cuda()
    mref_t = torch.from_numpy(np.ascontiguousarray(mref)).cuda()
    factor = float(penalty_factor(t, mref_t).item())
    p = LKParams(layer=1, iter=10, r=4, zRatio=1.0, movRange=5.0, smoothPenalty=factor * 0.08, tol=1e-3)
    for i in range(len(frames)):
        mmov = M.bwareafilt3(M.get_mask(frames[i].transpose(2, 1, 0), 3.0), rng)[0].transpose(2, 1, 0)
        m = torch.from_numpy(frames[i]).cuda()
        w = torch.empty(frames[i].shape, dtype=torch.float32, device="cuda")
        mot = LKRegistrar(frames[i].shape, p).register(
            m, t, torch.from_numpy(np.ascontiguousarray(mmov)).cuda(), mref_t, warped_out=w)
        np.testing.assert_array_equal(motions[i], mot.cpu().numpy())
        np.testing.assert_array_equal(mem_out[i], w.cpu().numpy())
        init = np.mean((frames[i] - ref) ** 2)                       # uint16 arithmetic, as the reference
        fin = np.mean((w.cpu().numpy().astype(np.float64) - ref.astype(np.float64)) ** 2)
        assert errors[i]["initial_error"] == pytest.approx(float(init), rel=1e-12)
        assert errors[i]["eventual_error"] == pytest.approx(float(fin), rel=1e-9)


def _pick_numpy(frames, max_corr_frames, spatial_ds=4):
    """utils/reference.py:19-99 restated in NumPy (float32)."""
    T, Z = frames.shape[:2]
    used = frames[:, Z // 2 - 1:Z // 2 + 2] if Z >= 3 else frames
    small = np.ascontiguousarray(used[:, :, ::spatial_ds, ::spatial_ds], dtype=np.float32)
    flat = small.reshape(T, -1)
    dem = flat - flat.mean(axis=1, keepdims=True)
    cc = dem @ dem.T
    d = np.sqrt(np.diag(cc)) + 1e-12
    cc = cc / (d[:, None] * d[None, :])
    n = min(max_corr_frames, T - 1)
    best = (-np.sort(-cc, axis=1))[:, 1:n + 1].mean(axis=1)
    imax = int(np.argmax(best))
    top = np.argsort(-cc[imax], kind="stable")[:n]
    return frames[top].mean(axis=0), top


def test_pick_initial_reference_and_dual_channel():
    _need()
    from wholistic_registration_b200.registration import pick_initial_reference, wbi_registration_3d

    _, frames = _batch(n=6, seed=21)
    ref_np, top_np = _pick_numpy(frames, 3)
    ref_t, top_t = pick_initial_reference(torch.from_numpy(frames).cuda(), 3)
    assert sorted(top_t.cpu().tolist()) == sorted(top_np.tolist())
    np.testing.assert_allclose(ref_t.cpu().numpy(), ref_np, rtol=1e-12)
    ca = (frames.astype(np.float32) * 0.5).astype(np.uint16)
    cfg = _config(pick=True, dual=True)
    cfg["reference"]["chunk_size"] = 3
    mem_out, ca_out, dat_ref, errors, motions = wbi_registration_3d(frames, cfg, moving_Ca_image=ca, verbose=False)
    assert ca_out.shape == frames.shape and np.isfinite(ca_out).all() and np.isfinite(mem_out).all()
    assert all(np.isfinite(e["eventual_error"]) for e in errors)


def test_2d_wrapper_is_the_stacked_3d_registration():
    """wbi_registration_2d registers each image as a two-plane volume whose
    x axis is the image's first axis (utils/registration.py:41-189)."""
    _need()
    from wholistic_registration_b200.registration import DEFAULT_ZRATIO, wbi_registration_2d, wbi_registration_3d

    ref, frames = _batch(n=2, shape=(1, 80, 72), seed=33)
    ref2, frames2 = ref[0], frames[:, 0]                   # (d0, d1) images
    mem, ca, dat_ref, errors, motions = wbi_registration_2d(frames2, _config(), reference_image=ref2, verbose=False)
    assert mem.shape == frames2.shape and motions.shape == frames2.shape + (3,) and dat_ref.shape == ref2.shape + (2,)
    vol = lambda im: np.ascontiguousarray(np.stack([im.T] * 2, axis=-3))
    cfg3 = _config()
    cfg3["MetaData"]["zRatio"] = DEFAULT_ZRATIO
    mem3, _, _, errors3, motions3 = wbi_registration_3d(np.stack([vol(f) for f in frames2]), cfg3,
                                                        reference_image=vol(ref2), verbose=False)
    np.testing.assert_array_equal(motions, motions3[:, 0].transpose(0, 2, 1, 3))
    np.testing.assert_array_equal(mem, mem3[:, 0].transpose(0, 2, 1))
    assert [e["initial_error"] for e in errors] == [e["initial_error"] for e in errors3]
