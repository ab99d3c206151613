"""Convolution kernels of the warm-start network against torch CPU autograd.

The CUDA kernels (BF16 tensor cores, float32 accumulation) are checked
against float32 CPU convolutions on the same bfloat16-rounded operands; the
tolerance covers bfloat16 rounding of the kernels' outputs and gradients.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = 2e-2   # relative to the largest magnitude of the reference


def _lib():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from wholistic_registration_b200 import _lib

    return _lib, _lib.load()


def _geom(_lib, n, o, i, stride, c1, c2, up1, cout, act):
    return _lib.WrConvGeom(n, *o, *i, stride, c1, c2, up1, cout, act)


def _to_torch_w(w, cout, cin):
    # [27][cout_p][cin] -> [cout][cin][3][3][3]
    return torch.from_numpy(w[:, :cout, :].reshape(3, 3, 3, cout, cin).transpose(3, 4, 0, 1, 2).copy())


def _close(a, b, tol=TOL):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    scale = max(np.abs(b).max(), 1e-6)
    err = np.abs(a - b).max() / scale
    assert err <= tol, f"relative error {err:.3e}"


CASES = [
    # n, input grid, stride, c1, c2, up1, cout, act
    (2, (6, 10, 12), 1, 16, 0, 0, 32, 1),
    (1, (7, 9, 11), 2, 32, 0, 0, 48, 1),
    (2, (6, 10, 12), 1, 32, 16, 1, 16, 1),
    (1, (5, 8, 6), 1, 16, 0, 0, 3, 0),
    # several 128-row tiles, the widest operands (112 input, 64 output channels)
    (1, (8, 16, 16), 1, 64, 48, 1, 48, 1),
    (1, (8, 16, 18), 2, 64, 0, 0, 64, 1),
]


@pytest.mark.parametrize("case", CASES)
def test_conv_forward_and_gradients(case):
    _l, lib = _lib()
    n, ig, stride, c1, c2, up1, cout, act = case
    rng = np.random.default_rng(sum(ig) + cout)
    og = tuple((d - 1) // stride + 1 for d in ig)
    cg = tuple((d + 1) // 2 for d in ig)
    cin = c1 + c2
    cout_p = (cout + 15) // 16 * 16
    bf = lambda a: torch.from_numpy(a).to(torch.bfloat16)
    x1 = bf(rng.normal(size=(n,) + (cg if up1 else ig) + (c1,)).astype(np.float32))
    x2 = bf(rng.normal(size=(n,) + ig + (c2,)).astype(np.float32)) if c2 else None
    w = rng.normal(size=(27, cout_p, cin)).astype(np.float32) * 0.1
    w[:, cout:, :] = 0
    w32 = torch.from_numpy(w).to(torch.bfloat16).float().numpy()
    b = rng.normal(size=cout).astype(np.float32)
    dev = "cuda"
    d_w = torch.from_numpy(w).to(dev)
    d_wf = torch.empty(w.shape, dtype=torch.bfloat16, device=dev)
    d_wt = torch.empty((27, cin, cout_p), dtype=torch.bfloat16, device=dev)
    s = torch.cuda.current_stream().cuda_stream
    _l.check("wr_net_weights_to_bf16", lib.wr_net_weights_to_bf16(d_w.data_ptr(), d_wf.data_ptr(), d_wt.data_ptr(),
                                                                  cout, cin, s))
    g = _geom(_l, n, og, ig, stride, c1, c2, up1, cout, act)
    d_x1 = x1.to(dev)
    d_x2 = x2.to(dev) if x2 is not None else None
    d_b = torch.from_numpy(b).to(dev)
    nvo = n * int(np.prod(og))
    if cout % 2 == 1:
        y = torch.empty((nvo, cout), dtype=torch.float32, device=dev)
        _l.check("fwd", lib.wr_net_conv3d_fwd(ctypes.byref(g), d_x1.data_ptr(), d_x2.data_ptr() if d_x2 is not None else None,
                                              d_wf.data_ptr(), d_b.data_ptr(), None, y.data_ptr(), s))
    else:
        y = torch.empty((nvo, cout), dtype=torch.bfloat16, device=dev)
        _l.check("fwd", lib.wr_net_conv3d_fwd(ctypes.byref(g), d_x1.data_ptr(), d_x2.data_ptr() if d_x2 is not None else None,
                                              d_wf.data_ptr(), d_b.data_ptr(), y.data_ptr(), None, s))
    # torch reference (NCDHW)
    t1 = x1.float().permute(0, 4, 1, 2, 3)
    if up1:
        t1 = t1.repeat_interleave(2, 2).repeat_interleave(2, 3).repeat_interleave(2, 4)[:, :, :ig[0], :ig[1], :ig[2]]
    tin = torch.cat([t1, x2.float().permute(0, 4, 1, 2, 3)], 1) if c2 else t1
    tin = tin.detach().requires_grad_(True)
    tw = _to_torch_w(w32, cout, cin).requires_grad_(True)
    tb = torch.from_numpy(b).requires_grad_(True)
    pre = torch.nn.functional.conv3d(tin, tw, tb, stride=stride, padding=1)
    ref = torch.nn.functional.leaky_relu(pre, 0.1) if act else pre
    _close(y.float().cpu().reshape((n,) + og + (cout,)).numpy(), ref.detach().permute(0, 2, 3, 4, 1).numpy())

    # backward with a random upstream gradient on the activation output
    up = torch.randn(ref.shape, generator=torch.Generator().manual_seed(3))
    ref.backward(up)
    grad = up.permute(0, 2, 3, 4, 1).reshape(nvo, cout).contiguous().to(dev)
    dpre = torch.empty((nvo, cout_p), dtype=torch.bfloat16, device=dev)
    _l.check("act", lib.wr_net_act_backward(grad.data_ptr(), y.data_ptr() if y.dtype == torch.bfloat16 else None,
                                            act, dpre.data_ptr(), nvo, cout, s))
    nvi = n * int(np.prod(ig))
    dxv = torch.empty((nvi, cin), dtype=torch.float32, device=dev)
    _l.check("dgrad", lib.wr_net_conv3d_dgrad(ctypes.byref(g), dpre.data_ptr(), d_wt.data_ptr(), dxv.data_ptr(), s))
    _close(dxv.cpu().reshape((n,) + ig + (cin,)).numpy(), tin.grad.permute(0, 2, 3, 4, 1).numpy())
    dw = torch.zeros((27, cout_p, cin), dtype=torch.float32, device=dev)
    db = torch.zeros(cout, dtype=torch.float32, device=dev)
    _l.check("wgrad", lib.wr_net_conv3d_wgrad(ctypes.byref(g), d_x1.data_ptr(),
                                              d_x2.data_ptr() if d_x2 is not None else None, dpre.data_ptr(),
                                              dw.data_ptr(), db.data_ptr(), s))
    ref_dw = tw.grad.permute(2, 3, 4, 0, 1).reshape(27, cout, cin).numpy()
    _close(dw.cpu().numpy()[:, :cout, :], ref_dw)
    _close(db.cpu().numpy(), tb.grad.numpy())
    if up1:
        g1 = torch.zeros((n,) + cg + (c1,), dtype=torch.float32, device=dev)
        g2 = torch.zeros((n,) + ig + (c2,), dtype=torch.float32, device=dev)
        _l.check("split", lib.wr_net_split_grad(ctypes.byref(g), dxv.data_ptr(), g1.data_ptr(), g2.data_ptr(), s))
        tg = tin.grad.permute(0, 2, 3, 4, 1).numpy()
        ref_g2 = tg[..., c1:]
        up_part = tg[..., :c1]
        ref_g1 = np.zeros((n,) + cg + (c1,), np.float64)
        for z in range(ig[0]):
            for yy in range(ig[1]):
                for x in range(ig[2]):
                    ref_g1[:, z // 2, yy // 2, x // 2] += up_part[:, z, yy, x]
        _close(g2.cpu().numpy(), ref_g2)
        _close(g1.cpu().numpy(), ref_g1)
    # the tensor-core convolutions finished without a wait running out
    flag = ctypes.c_int(-1)
    _l.check("wr_net_tc_error", lib.wr_net_tc_error(ctypes.byref(flag)))
    assert flag.value == 0
