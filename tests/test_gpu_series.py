"""Time-series registration from host memory (series.SeriesRegistrar): the
host motion and warped volumes of every frame equal registering the frame
alone on the device (utils/registration.py:299-346 registers frame by frame),
for several buffer depths."""

from __future__ import annotations

import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("depth", [1, 2, 3])
def test_series_matches_frames_alone(depth):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from wholistic_registration_b200 import LKParams, LKRegistrar, synthetic
    from wholistic_registration_b200.series import SeriesRegistrar

    shape = (9, 64, 72)
    dev = torch.device("cuda")
    tmpl, _, _ = synthetic.make_pair(shape, 3, n_blobs=300, max_disp=(2.0, 2.0, 0.5), device=dev)
    tmpl = tmpl.contiguous()
    excl = (~synthetic.ellipsoid_inclusion(shape, 0.75, device=dev)).to(torch.uint8).contiguous()
    frames = []
    for k in range(5):
        _, mov, _ = synthetic.make_pair(shape, 10 + k, n_blobs=300, max_disp=(2.0, 2.0, 0.5), device=dev,
                                        template=tmpl.float())
        frames.append(mov.contiguous())
    p = LKParams(layer=2, iter=6, r=3, zRatio=1.0, movRange=5.0, smoothPenalty=100.0, tol=1e-3)

    host_in = [f.cpu().pin_memory() for f in frames]
    host_m = [torch.empty(shape + (3,), dtype=torch.float32).pin_memory() for _ in frames]
    host_w = [torch.empty(shape, dtype=torch.float32).pin_memory() for _ in frames]
    series = SeriesRegistrar(tmpl, p, mask_ref=excl, mask_mov=excl, depth=depth)
    series.run(host_in, host_m, host_w)
    series.done()

    reg = LKRegistrar(shape, p, dev)
    for k, f in enumerate(frames):
        w = torch.empty(shape, dtype=torch.float32, device=dev)
        m = reg.register(f, tmpl, excl, excl, warped_out=w)
        torch.cuda.synchronize()
        assert torch.equal(host_m[k], m.cpu()), k
        assert torch.equal(host_w[k], w.cpu()), k

