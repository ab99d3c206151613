"""Batched registration (wr_lk_register_batch): frames of uneven shapes run
together must give exactly the motion, warped volume and error log of
registering each frame alone; the CUDA-graph form replays the same."""

from __future__ import annotations

import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

SHAPES = [(8, 96, 80), (6, 70, 66), (8, 64, 64)]


def _need():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _frames(seed, shapes=SHAPES):
    from wholistic_registration_b200 import synthetic

    out = []
    for k, s in enumerate(shapes):
        tmpl, mov, _ = synthetic.make_pair(s, seed + k, n_blobs=300, max_disp=(2.5, 2.5, 0.8))
        excl = (~synthetic.ellipsoid_inclusion(s, 0.75)).to(torch.uint8)
        out.append(tuple(x.cuda().contiguous() for x in (tmpl, mov, excl)))
    return out


def _params(**kw):
    from wholistic_registration_b200 import LKParams

    base = dict(layer=2, iter=10, r=4, zRatio=1.0, movRange=5.0, smoothPenalty=200.0, tol=1e-3)
    base.update(kw)
    return LKParams(**base)


def _alone(frames, p, warp=False):
    from wholistic_registration_b200 import LKRegistrar

    motions, warps, evals = [], [], []
    for t, m, e in frames:
        reg = LKRegistrar(tuple(t.shape), p)
        w = torch.empty(t.shape, dtype=torch.float32, device="cuda") if warp else None
        motions.append(reg.register(m, t, e, e, warped_out=w).clone())
        warps.append(w)
        st = reg.stats()
        evals.append([st.evals[l] for l in range(p.layer + 1)])
    return motions, warps, evals


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_equals_frames_alone(precision):
    _need()
    from wholistic_registration_b200.batch import BatchRegistrar

    frames = _frames(40)
    p = _params(precision=precision)
    ref_m, ref_w, ref_e = _alone(frames, p, warp=True)
    br = BatchRegistrar(SHAPES, p, warp=True)
    motions, warps = br.register([f[1] for f in frames], [f[0] for f in frames], [f[2] for f in frames],
                                 [f[2] for f in frames])
    for i in range(len(SHAPES)):
        torch.testing.assert_close(motions[i], ref_m[i], rtol=0, atol=0)
        torch.testing.assert_close(warps[i], ref_w[i], rtol=0, atol=0)
    st = br.stats()
    assert [[s.evals[l] for l in range(p.layer + 1)] for s in st] == ref_e


def test_batch_without_masks_and_with_initial_field():
    _need()
    from wholistic_registration_b200 import LKRegistrar
    from wholistic_registration_b200.batch import BatchRegistrar

    frames = _frames(50)
    p = _params(layer=1)
    inits = [torch.full(tuple(t.shape) + (3,), 0.25, dtype=torch.float32, device="cuda") for t, _, _ in frames]
    br = BatchRegistrar(SHAPES, p, mask_mov=False, mask_ref=False, init=True)
    motions = br.register([f[1] for f in frames], [f[0] for f in frames], inits=inits)
    for i, (t, m, _) in enumerate(frames):
        alone = LKRegistrar(tuple(t.shape), p).register(m, t, motion_init=inits[i])
        torch.testing.assert_close(motions[i], alone, rtol=0, atol=0)


def test_batch_graph_replays_series():
    """A series against fixed templates: eager first call, captured second
    call, replays after; every call equals the frames registered alone."""
    _need()
    from wholistic_registration_b200 import LKRegistrar
    from wholistic_registration_b200.batch import BatchRegistrar
    from wholistic_registration_b200 import synthetic

    p = _params()
    frames = _frames(60)
    br = BatchRegistrar(SHAPES, p, graph=True)
    for call in range(4):
        movs = []
        for k, (t, _, _) in enumerate(frames):
            _, m, _ = synthetic.make_pair(SHAPES[k], 100 * call + k, n_blobs=300, max_disp=(2.5, 2.5, 0.8),
                                          template=t.float().cpu())
            movs.append(m.cuda().contiguous())
        motions = br.register(movs, [f[0] for f in frames], [f[2] for f in frames], [f[2] for f in frames],
                              reuse_reference=call > 0)
        got = [x.clone() for x in motions]
        for k, (t, _, e) in enumerate(frames):
            alone = LKRegistrar(SHAPES[k], p).register(movs[k], t, e, e)
            torch.testing.assert_close(got[k], alone, rtol=0, atol=0)
    assert br._graph is not None


def test_batch_argument_errors():
    _need()
    from wholistic_registration_b200.batch import BatchRegistrar

    with pytest.raises(ValueError):
        BatchRegistrar([(8, 64, 64)] * 65, _params())
    with pytest.raises(ValueError):
        BatchRegistrar(SHAPES, [_params()] * 2)          # one parameter set per frame, or one for all
    with pytest.raises(RuntimeError, match="precision"):
        BatchRegistrar(SHAPES, [_params(), _params(precision=1), _params()])
    br = BatchRegistrar(SHAPES, _params())
    frames = _frames(70)
    with pytest.raises(ValueError):
        br.register([f[1] for f in frames][:2], [f[0] for f in frames][:2])


def test_launch_shapes_do_not_change_results():
    """Every autotuner candidate (tile order, CTAs per SM) gives the same
    motion, bit for bit, single and batched."""
    _need()
    from wholistic_registration_b200 import LKRegistrar, autotune
    from wholistic_registration_b200.batch import BatchRegistrar

    frames = _frames(80)
    p = _params()
    t, m, e = frames[0]
    reg = LKRegistrar(tuple(t.shape), p)
    base = reg.register(m, t, e, e).clone()
    br = BatchRegistrar(SHAPES, p)
    bbase = [x.clone() for x in br.register([f[1] for f in frames], [f[0] for f in frames], [f[2] for f in frames],
                                            [f[2] for f in frames])]
    for flags in autotune.candidates():
        reg.tune_flags = flags
        torch.testing.assert_close(reg.register(m, t, e, e), base, rtol=0, atol=0)
        br.tune_flags = flags
        got = br.register([f[1] for f in frames], [f[0] for f in frames], [f[2] for f in frames],
                          [f[2] for f in frames])
        for a, b in zip(got, bbase):
            torch.testing.assert_close(a, b, rtol=0, atol=0)


def test_autotune_picks_and_caches(tmp_path, monkeypatch):
    _need()
    from wholistic_registration_b200 import LKRegistrar, autotune

    monkeypatch.setenv("WR_B200_CACHE", str(tmp_path))
    p = _params()
    reg = LKRegistrar((8, 96, 80), p)
    report = {}
    flags = reg.autotune(report=report)
    assert flags in autotune.candidates()
    assert len(report) == len(autotune.candidates())
    assert (tmp_path / "autotune.json").exists()
    again = {}
    assert reg.autotune(report=again) == flags and again == report


@pytest.mark.parametrize("init", [False, True])
def test_batch_with_parameters_per_frame(init):
    """Each frame with its own option dict (wr_lk_register_batch_each): patch
    radius, levels, iterations, zRatio and penalty differ between frames, so
    frames with fewer levels join the batch at their own top level; every
    frame's motion, warped volume and evaluations equal its call alone."""
    _need()
    from wholistic_registration_b200 import LKRegistrar
    from wholistic_registration_b200.batch import BatchRegistrar

    shapes = [(8, 96, 80), (6, 70, 66), (8, 64, 64), (5, 120, 96), (7, 80, 90)]
    frames = _frames(60, shapes)
    plist = [_params(r=4, layer=2), _params(r=3, layer=1, iter=6, zRatio=2.0),
             _params(r=2, layer=0, iter=4, smoothPenalty=50.0), _params(r=8, layer=2, tol=1e-4),
             _params(r=5, layer=1, iter=8, movRange=2.0)]
    inits = [torch.full(tuple(t.shape) + (3,), 0.3, dtype=torch.float32, device="cuda") for t, _, _ in frames] \
        if init else None
    br = BatchRegistrar(shapes, plist, warp=True, init=init)
    motions, warps = br.register([f[1] for f in frames], [f[0] for f in frames], [f[2] for f in frames],
                                 [f[2] for f in frames], inits=inits)
    st = br.stats()
    for i, ((t, m, e), p) in enumerate(zip(frames, plist)):
        reg = LKRegistrar(tuple(t.shape), p)
        w = torch.empty(t.shape, dtype=torch.float32, device="cuda")
        alone = reg.register(m, t, e, e, motion_init=inits[i] if init else None, warped_out=w).clone()
        torch.testing.assert_close(motions[i], alone, rtol=0, atol=0)
        torch.testing.assert_close(warps[i], w, rtol=0, atol=0)
        s = reg.stats()
        assert [st[i].evals[l] for l in range(p.layer + 1)] == [s.evals[l] for l in range(p.layer + 1)]


def test_batch_holds_64_frames():
    """The batch cap is 64 frames (WR_MAX_BATCH); 48 small frames with their
    own radii in one call equal their calls alone."""
    _need()
    from wholistic_registration_b200 import LKRegistrar
    from wholistic_registration_b200 import _lib
    from wholistic_registration_b200.batch import BatchRegistrar

    assert _lib.MAX_BATCH == 64
    shapes = [(4, 48 + 4 * (k % 5), 40 + 4 * (k % 7)) for k in range(48)]
    frames = _frames(80, shapes)
    plist = [_params(r=2 + k % 4, layer=1, iter=5) for k in range(48)]
    br = BatchRegistrar(shapes, plist)
    motions = br.register([f[1] for f in frames], [f[0] for f in frames], [f[2] for f in frames],
                          [f[2] for f in frames])
    for i in (0, 17, 33, 47):
        t, m, e = frames[i]
        alone = LKRegistrar(tuple(t.shape), plist[i]).register(m, t, e, e)
        torch.testing.assert_close(motions[i], alone, rtol=0, atol=0)
    with pytest.raises(ValueError):
        BatchRegistrar([(4, 48, 40)] * 65, plist[0])


def test_batch_mixing_own_launches_and_shared_launches():
    """A frame-level with enough tiles takes its own launch of the
    single-volume kernel inside the batched call, smaller ones share the
    batched launch (level 0 of the first frame: 16 x 52 x 52 tiles of 5 x 5);
    both give exactly the frames' results alone."""
    _need()
    from wholistic_registration_b200.batch import BatchRegistrar

    shapes = [(16, 256, 256), (8, 64, 64), (12, 128, 96)]
    frames = _frames(90, shapes)
    plist = [_params(r=2, layer=2, iter=6), _params(r=4, layer=1, iter=6), _params(r=3, layer=2, iter=5)]
    br = BatchRegistrar(shapes, plist, warp=True)
    motions, warps = br.register([f[1] for f in frames], [f[0] for f in frames], [f[2] for f in frames],
                                 [f[2] for f in frames])
    for i, (f, p) in enumerate(zip(frames, plist)):
        ref_m, ref_w, ref_e = _alone([f], p, warp=True)
        torch.testing.assert_close(motions[i], ref_m[0], rtol=0, atol=0)
        torch.testing.assert_close(warps[i], ref_w[0], rtol=0, atol=0)
        assert [br.stats()[i].evals[l] for l in range(p.layer + 1)] == ref_e[0]
