"""The trained warm-start network: what it gains over the method without it.

On a held-out synthetic pair the network's field alone must be much closer
to the full plain pyramid's (which matches the reference to 1e-3 voxel) than
no field, and a 2-level, 4-iteration refinement started from it must end
closer than the same short refinement started from zero.  The distances are
printed; the short refinement does not reach the plain pyramid's field to
0.1 voxel, so the registrar keeps its plain-pyramid fallback.  The whole
network forward pass is also checked against a torch CPU restatement.
"""

from __future__ import annotations

import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
WEIGHTS = os.path.join(ROOT, "wholistic_registration_b200", "weights", "warmstart.npz")


def _need():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    if not os.path.exists(WEIGHTS):
        pytest.skip("no trained weights")


def _pair(shape, seed):
    from wholistic_registration_b200 import penalty_factor, synthetic

    tmpl, mov, field = synthetic.make_pair(shape, seed, n_blobs=2000, max_disp=(6.0, 6.0, 2.0), device="cuda")
    t = tmpl.float().contiguous()
    m = mov.float().contiguous()
    return t, m, float(penalty_factor(t))


def test_warm_start_beats_short_refinement_from_zero():
    _need()
    from wholistic_registration_b200 import LKParams, LKRegistrar
    from wholistic_registration_b200.warmstart import WarmStartNet

    shape = (64, 256, 256)
    t, m, factor = _pair(shape, 91357)
    plain = LKParams(layer=2, iter=10, r=16, zRatio=1.0, movRange=5.0, smoothPenalty=0.08 * factor, tol=1e-3)
    short = LKParams(layer=1, iter=4, r=16, zRatio=1.0, movRange=5.0, smoothPenalty=0.08 * factor, tol=1e-3)
    ref_field = LKRegistrar(shape, plain).register(m, t).clone()
    net = WarmStartNet()
    net.load(WEIGHTS)
    init = net.predict(t, m).clone()
    warm = LKRegistrar(shape, short).register(m, t, motion_init=init).clone()
    cold = LKRegistrar(shape, short).register(m, t).clone()
    rms = lambda a: float(torch.sqrt(((a - ref_field) ** 2).mean()))
    r_warm, r_cold, r_init = rms(warm), rms(cold), rms(init)
    r_zero = float(torch.sqrt((ref_field ** 2).mean()))
    print(f"RMS vs plain: warm {r_warm:.4f}, cold {r_cold:.4f}, network alone {r_init:.4f}, zero {r_zero:.4f}")
    assert r_init < 0.5 * r_zero
    assert r_warm < r_cold


def test_network_forward_matches_torch_restatement():
    _need()
    from wholistic_registration_b200.warmstart import LAYERS, WarmStartNet

    net = WarmStartNet()
    net.load(WEIGHTS)
    shape = (12, 64, 48)
    gen = torch.Generator(device="cuda").manual_seed(3)
    t = torch.rand(shape, generator=gen, device="cuda") * 1000 + 100
    m = torch.rand(shape, generator=gen, device="cuda") * 1000 + 100
    net.prepare(t, m)
    out = net.forward().float().cpu()
    # torch CPU restatement on the same bf16 input and bf16-rounded weights
    acts = {"in": net.act["in"].float().cpu().reshape(1, *net.gs[0], 16).permute(0, 4, 1, 2, 3)}
    for name, s1, s2, c1, c2, up1, cout, stride, act, lvl in LAYERS:
        x1 = acts[s1]
        if up1:
            g = net.gs[lvl]
            x1 = x1.repeat_interleave(2, 2).repeat_interleave(2, 3).repeat_interleave(2, 4)[:, :, :g[0], :g[1], :g[2]]
        x = torch.cat([x1, acts[s2]], 1) if s2 else x1
        w = net.wf[name].float().cpu()[:, :cout, :].reshape(3, 3, 3, cout, c1 + c2).permute(3, 4, 0, 1, 2)
        y = torch.nn.functional.conv3d(x, w, net.b[name].cpu(), stride=stride, padding=1)
        if act:
            y = torch.nn.functional.leaky_relu(y, 0.1).to(torch.bfloat16).float()
        acts[name] = y
    ref = acts["out"].permute(0, 2, 3, 4, 1).reshape(-1, 3)
    err = float((out - ref).abs().max() / ref.abs().max())
    assert err < 5e-2, err
