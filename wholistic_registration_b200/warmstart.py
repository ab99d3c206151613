"""Learned warm start for the pyramid Lucas-Kanade registration.

A 3-D convolutional encoder-decoder (4 scales, 16/32/48/64 channels, 3x3x3
kernels, LeakyReLU, bfloat16 weights and activations, float32 accumulation)
reads the template and moving volumes pooled 4x in x and y and predicts the
displacement field on that grid.  Every operation is a kernel of the
project's library (``include/wr_net.h``): implicit-GEMM convolutions on BF16
tensor cores for the forward pass and both backward passes, Adam, the loss.

The network learns the plain method's own converged fields (``train``); its
prediction, up-sampled to full resolution, enters the registration through
the reference's warm-start channel ``option["motion"]``
(utils/calFlow3d_Wei_v1.py:362-377) for a short refinement (2 levels, 4
iterations).  ``WarmStartRegistrar`` falls back to the full plain pyramid
when the refined field's masked residual exceeds the plain method's by more
than a margin.
"""

from __future__ import annotations

import ctypes
import math
import os
import time

import numpy as np
import torch

from . import _lib
from .registrar import LKParams, LKRegistrar, warp

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_WEIGHTS = os.path.join(HERE, "weights", "warmstart.npz")
POOL = 4   # network grid: x and y pooled by 4, z kept

# name, source 1, source 2, c1, c2, source 1 at half resolution, cout, stride, activation, output scale
LAYERS = [
    ("e0a", "in", None, 16, 0, 0, 16, 1, 1, 0),
    ("e0b", "e0a", None, 16, 0, 0, 16, 1, 1, 0),
    ("e1a", "e0b", None, 16, 0, 0, 32, 2, 1, 1),
    ("e1b", "e1a", None, 32, 0, 0, 32, 1, 1, 1),
    ("e2a", "e1b", None, 32, 0, 0, 48, 2, 1, 2),
    ("e2b", "e2a", None, 48, 0, 0, 48, 1, 1, 2),
    ("e3a", "e2b", None, 48, 0, 0, 64, 2, 1, 3),
    ("e3b", "e3a", None, 64, 0, 0, 64, 1, 1, 3),
    ("d2", "e3b", "e2b", 64, 48, 1, 48, 1, 1, 2),
    ("d1", "d2", "e1b", 48, 32, 1, 32, 1, 1, 1),
    ("d0", "d1", "e0b", 32, 16, 1, 16, 1, 1, 0),
    ("out", "d0", None, 16, 0, 0, 3, 1, 0, 0),
]


def _pad16(c):
    return (c + 15) // 16 * 16


def grids(g0):
    out = [tuple(g0)]
    for _ in range(3):
        out.append(tuple((d + 1) // 2 for d in out[-1]))
    return out


class WarmStartNet:
    """Parameters, buffers and the forward / backward passes."""

    def __init__(self, device=None, seed=0):
        self.lib = _lib.load()
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        gen = np.random.default_rng(seed)
        self.w, self.b, self.wf, self.wt, self.gw, self.gb = {}, {}, {}, {}, {}, {}
        self.adam = {}
        for name, s1, s2, c1, c2, up1, cout, stride, act, lvl in LAYERS:
            cin = c1 + c2
            cout_p = _pad16(cout)
            fan_in = 27 * (2 if name == "e0a" else cin)
            std = math.sqrt(2.0 / fan_in) * (0.1 if name == "out" else 1.0)
            w = np.zeros((27, cout_p, cin), np.float32)
            w[:, :cout, :] = gen.normal(0.0, std, size=(27, cout, cin))
            self.w[name] = torch.from_numpy(w).to(self.device)
            self.b[name] = torch.zeros(cout, dtype=torch.float32, device=self.device)
            self.wf[name] = torch.empty((27, cout_p, cin), dtype=torch.bfloat16, device=self.device)
            self.wt[name] = torch.empty((27, cin, cout_p), dtype=torch.bfloat16, device=self.device)
            self.gw[name] = torch.zeros_like(self.w[name])
            self.gb[name] = torch.zeros_like(self.b[name])
            self.adam[name] = [torch.zeros_like(self.w[name]), torch.zeros_like(self.w[name]),
                               torch.zeros_like(self.b[name]), torch.zeros_like(self.b[name])]
        self.step_count = 0
        self._buf_key = None
        self._refresh_bf16()

    # -- parameters ---------------------------------------------------------
    def _stream(self):
        return torch.cuda.current_stream(self.device).cuda_stream

    def _refresh_bf16(self):
        for name, s1, s2, c1, c2, up1, cout, stride, act, lvl in LAYERS:
            _lib.check("wr_net_weights_to_bf16", self.lib.wr_net_weights_to_bf16(
                self.w[name].data_ptr(), self.wf[name].data_ptr(), self.wt[name].data_ptr(), cout, c1 + c2,
                self._stream()))

    def state(self):
        out = {}
        for name in self.w:
            out[f"{name}.w"] = self.w[name].cpu().numpy()
            out[f"{name}.b"] = self.b[name].cpu().numpy()
        return out

    def save(self, path=DEFAULT_WEIGHTS, **meta):
        os.makedirs(os.path.dirname(path), exist_ok=True)
        np.savez_compressed(path, **self.state(), **{f"meta.{k}": np.asarray(v) for k, v in meta.items()})

    def load(self, path=DEFAULT_WEIGHTS):
        d = np.load(path)
        for name in self.w:
            self.w[name].copy_(torch.from_numpy(d[f"{name}.w"]))
            self.b[name].copy_(torch.from_numpy(d[f"{name}.b"]))
        self._refresh_bf16()
        return {k[5:]: d[k] for k in d.files if k.startswith("meta.")}

    def parameter_count(self):
        return sum(27 * L[6] * (L[3] + L[4]) + L[6] for L in LAYERS)

    # -- buffers ------------------------------------------------------------
    def _buffers(self, n, g0):
        key = (n, tuple(g0))
        if key == self._buf_key:
            return
        gs = grids(g0)
        dev = self.device
        self.gs = gs
        self.n = n
        self.act = {"in": torch.zeros((n * int(np.prod(gs[0])), 16), dtype=torch.bfloat16, device=dev)}
        self.grad = {}
        for name, s1, s2, c1, c2, up1, cout, stride, act, lvl in LAYERS:
            nv = n * int(np.prod(gs[lvl]))
            if name == "out":
                self.act[name] = torch.empty((nv, 3), dtype=torch.float32, device=dev)
            else:
                self.act[name] = torch.empty((nv, cout), dtype=torch.bfloat16, device=dev)
            self.grad[name] = torch.zeros((nv, cout), dtype=torch.float32, device=dev)
        maxv = n * int(np.prod(gs[0]))
        self.dpre = torch.empty(maxv * 64, dtype=torch.bfloat16, device=dev)
        self.dxv = torch.empty(maxv * 112, dtype=torch.float32, device=dev)
        self._buf_key = key

    def _geom(self, layer):
        name, s1, s2, c1, c2, up1, cout, stride, act, lvl = layer
        go = self.gs[lvl]
        if stride == 2:
            gi = self.gs[lvl - 1]
        else:
            gi = go
        return _lib.WrConvGeom(self.n, *go, *gi, stride, c1, c2, up1, cout, act)

    # -- passes -------------------------------------------------------------
    def forward(self):
        """Runs the layers on ``self.act['in']``; returns the flow (nvox, 3) float32."""
        s = self._stream()
        for layer in LAYERS:
            name, s1, s2, c1, c2, up1, cout, stride, act, lvl = layer
            g = self._geom(layer)
            x2 = self.act[s2].data_ptr() if s2 else None
            y = self.act[name]
            if name == "out":
                rc = self.lib.wr_net_conv3d_fwd(ctypes.byref(g), self.act[s1].data_ptr(), x2, self.wf[name].data_ptr(),
                                                self.b[name].data_ptr(), None, y.data_ptr(), s)
            else:
                rc = self.lib.wr_net_conv3d_fwd(ctypes.byref(g), self.act[s1].data_ptr(), x2, self.wf[name].data_ptr(),
                                                self.b[name].data_ptr(), y.data_ptr(), None, s)
            _lib.check("wr_net_conv3d_fwd", rc)
        return self.act["out"]

    def backward(self):
        """Back-propagates ``self.grad['out']`` (set by the loss) into gw, gb."""
        s = self._stream()
        for t in self.grad.values():
            if t is not self.grad["out"]:
                t.zero_()
        for layer in reversed(LAYERS):
            name, s1, s2, c1, c2, up1, cout, stride, act, lvl = layer
            g = self._geom(layer)
            nvo = self.n * int(np.prod(self.gs[lvl]))
            y = self.act[name] if act else None
            _lib.check("wr_net_act_backward", self.lib.wr_net_act_backward(
                self.grad[name].data_ptr(), y.data_ptr() if y is not None else None, act, self.dpre.data_ptr(), nvo,
                cout, s))
            x2 = self.act[s2].data_ptr() if s2 else None
            _lib.check("wr_net_conv3d_wgrad", self.lib.wr_net_conv3d_wgrad(
                ctypes.byref(g), self.act[s1].data_ptr(), x2, self.dpre.data_ptr(), self.gw[name].data_ptr(),
                self.gb[name].data_ptr(), s))
            if s1 == "in":
                continue
            _lib.check("wr_net_conv3d_dgrad", self.lib.wr_net_conv3d_dgrad(
                ctypes.byref(g), self.dpre.data_ptr(), self.wt[name].data_ptr(), self.dxv.data_ptr(), s))
            _lib.check("wr_net_split_grad", self.lib.wr_net_split_grad(
                ctypes.byref(g), self.dxv.data_ptr(), self.grad[s1].data_ptr(),
                self.grad[s2].data_ptr() if s2 else None, s))

    def zero_grad(self):
        for name in self.gw:
            self.gw[name].zero_()
            self.gb[name].zero_()

    def adam_step(self, lr, b1=0.9, b2=0.999, eps=1e-8, decay=0.0):
        self.step_count += 1
        s = self._stream()
        for name in self.w:
            m, v, mb, vb = self.adam[name]
            _lib.check("wr_net_adam", self.lib.wr_net_adam(self.w[name].data_ptr(), self.gw[name].data_ptr(),
                                                           m.data_ptr(), v.data_ptr(), self.w[name].numel(), lr, b1,
                                                           b2, eps, self.step_count, decay, s))
            _lib.check("wr_net_adam", self.lib.wr_net_adam(self.b[name].data_ptr(), self.gb[name].data_ptr(),
                                                           mb.data_ptr(), vb.data_ptr(), self.b[name].numel(), lr, b1,
                                                           b2, eps, self.step_count, 0.0, s))
        self._refresh_bf16()

    # -- inputs -------------------------------------------------------------
    def prepare(self, tmpl, mov, keep_fp32=False):
        """Pools a (z, y, x) pair into the network input; returns the grid."""
        z, y, x = tmpl.shape
        g0 = (z, y // POOL, x // POOL)
        self._buffers(1, g0)
        if not hasattr(self, "_mean") or self._mean.device != self.device:
            self._mean = torch.zeros(2, dtype=torch.float64, device=self.device)
        dt = {torch.uint16: _lib.WR_U16, torch.float32: _lib.WR_F32}[tmpl.dtype]
        vt, vm = _lib.volume(tmpl.data_ptr(), dt, tmpl.shape), _lib.volume(mov.data_ptr(), dt, mov.shape)
        t4 = m4 = None
        if keep_fp32:
            nq = int(np.prod(g0))
            if getattr(self, "_t4", None) is None or self._t4.numel() != nq:
                self._t4 = torch.empty(nq, dtype=torch.float32, device=self.device)
                self._m4 = torch.empty(nq, dtype=torch.float32, device=self.device)
            t4, m4 = self._t4.data_ptr(), self._m4.data_ptr()
        _lib.check("wr_net_prepare_input", self.lib.wr_net_prepare_input(
            ctypes.byref(vt), ctypes.byref(vm), POOL, self._mean.data_ptr(), self.act["in"].data_ptr(), t4, m4,
            self._stream()))
        return g0

    def predict(self, tmpl, mov, out=None):
        """Full-resolution (z, y, x, 3) initial field for a (z, y, x) pair."""
        z, y, x = tmpl.shape
        self.prepare(tmpl, mov)
        fq = self.forward()
        if out is None:
            out = torch.empty((z, y, x, 3), dtype=torch.float32, device=self.device)
        _lib.check("wr_net_upsample_flow", self.lib.wr_net_upsample_flow(fq.data_ptr(), z, y, x, POOL, out.data_ptr(),
                                                                         self._stream()))
        return out


def masked_mse(warped, ref, excl=None):
    """Mean (warped - ref)^2 over voxels not excluded (device float64 pair)."""
    lib = _lib.load()
    out = torch.zeros(2, dtype=torch.float64, device=warped.device)
    dt = {torch.uint16: _lib.WR_U16, torch.float32: _lib.WR_F32}[ref.dtype]
    v = _lib.volume(ref.data_ptr(), dt, ref.shape)
    _lib.check("wr_net_masked_sse", lib.wr_net_masked_sse(warped.data_ptr(), ctypes.byref(v),
                                                         excl.data_ptr() if excl is not None else None,
                                                         out.data_ptr(), torch.cuda.current_stream().cuda_stream))
    return out


# ---------------------------------------------------------------------------
# training
# ---------------------------------------------------------------------------

def train(steps=20000, shape=(64, 256, 256), templates=48, seed=0, lr=1e-3, res_weight=1.0, log_every=500,
          device=None, net=None, time_limit=None):
    """Train on ``steps`` synthetic pairs at ``shape`` (z, y, x): a template
    from a pool rendered with the blob generator, a random sinusoid field of
    up to 8 voxels in x / y and 3 in z, and as target the plain method's own
    converged field (layer 2, r 16, iter 10), pooled onto the network grid."""
    from . import synthetic
    from .registrar import penalty_factor

    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    rng = np.random.default_rng(seed)
    net = net or WarmStartNet(dev, seed)
    pool = []
    for k in range(templates):
        clean = synthetic.render_blobs(shape, 2000, rng, device=dev)
        gen = torch.Generator(device=dev)
        gen.manual_seed(seed * 1000 + k)
        t = torch.poisson(clean, generator=gen)
        pool.append((t, float(penalty_factor(t.contiguous()))))
    reg = None
    z, y, x = shape
    g0 = (z, y // POOL, x // POOL)
    target = torch.empty((int(np.prod(g0)), 3), dtype=torch.float32, device=dev)
    loss_acc = torch.zeros(1, dtype=torch.float64, device=dev)
    history = []
    t_start = time.time()
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed + 17)
    for step in range(steps):
        tmpl_f, factor = pool[int(rng.integers(templates))]
        md = rng.uniform(0.0, 8.0)
        field = synthetic.sinusoid_field(shape, rng, max_disp=(md, rng.uniform(0.0, 8.0), rng.uniform(0.0, 3.0)),
                                         device=dev)
        mov = torch.poisson(synthetic.warp_pull(tmpl_f, -field).clamp_min(0), generator=gen)
        tmpl = tmpl_f.contiguous()
        if reg is None:
            reg = LKRegistrar(shape, LKParams(layer=2, iter=10, r=16, zRatio=1.0, movRange=5.0,
                                              smoothPenalty=0.08 * factor, tol=1e-3), dev)
        reg._cp.smoothPenalty = 0.08 * factor
        flow = reg.register(mov, tmpl)
        _lib.check("wr_net_pool_flow", net.lib.wr_net_pool_flow(flow.data_ptr(), z, y, x, POOL, target.data_ptr(),
                                                                 net._stream()))
        net.prepare(tmpl, mov, keep_fp32=True)
        pred = net.forward()
        net.zero_grad()
        frac = step / max(steps - 1, 1)
        cur_lr = 1e-4 + 0.5 * (lr - 1e-4) * (1 + math.cos(math.pi * frac))
        _lib.check("wr_net_flow_loss", net.lib.wr_net_flow_loss(
            pred.data_ptr(), target.data_ptr(), net._t4.data_ptr(), net._m4.data_ptr(), net.grad["out"].data_ptr(),
            loss_acc.data_ptr(), 1, *g0, float(POOL), 1.0, res_weight, net._stream()))
        net.backward()
        net.adam_step(cur_lr)
        if (step + 1) % log_every == 0 or step == steps - 1:
            mean_loss = float(loss_acc) / ((step % log_every) + 1)
            loss_acc.zero_()
            history.append((step + 1, mean_loss, time.time() - t_start))
            print(f"step {step + 1}: loss {mean_loss:.4f} lr {cur_lr:.2e} ({time.time() - t_start:.0f} s)", flush=True)
        if time_limit is not None and time.time() - t_start > time_limit:
            print(f"time limit reached at step {step + 1}", flush=True)
            history.append((step + 1, float("nan"), time.time() - t_start))
            break
    return net, history


# ---------------------------------------------------------------------------
# warm-started registration
# ---------------------------------------------------------------------------

class WarmStartRegistrar:
    """Registration warm-started by the network, with the plain pyramid as fallback.

    The network's field initialises a ``refine_layer``-level,
    ``refine_iter``-iteration registration (levels stored in ``precision``).
    Every ``calibrate_every``-th frame also runs the plain pyramid and records
    the ratio of its masked residual (after / before registration); a frame
    whose warm-started ratio exceeds that by more than ``margin`` is
    registered again with the plain pyramid.
    """

    def __init__(self, shape_zyx, plain: LKParams, net: WarmStartNet, refine_layer=1, refine_iter=4,
                 precision=_lib.WR_PREC_F16, margin=0.05, calibrate_every=16, device=None):
        self.shape = tuple(shape_zyx)
        self.net = net
        self.plain = LKRegistrar(self.shape, plain, device)
        fast = LKParams(layer=refine_layer, iter=refine_iter, r=plain.r, zRatio=plain.zRatio,
                        movRange=plain.movRange, smoothPenalty=plain.smoothPenalty, tol=plain.tol,
                        precision=precision)
        self.fast = LKRegistrar(self.shape, fast, device)
        self.device = self.plain.device
        self.init = torch.empty(self.shape + (3,), dtype=torch.float32, device=self.device)
        self.warped = torch.empty(self.shape, dtype=torch.float32, device=self.device)
        self.margin = margin
        self.calibrate_every = calibrate_every
        self.plain_ratio = None
        self.frames = 0
        self.fallbacks = 0
        self.ref_ready = False

    def _ratio(self, mov, ref, motion, excl):
        warp(mov, motion, out=self.warped)
        after = masked_mse(self.warped, ref, excl)
        before = masked_mse(mov.float() if mov.dtype != torch.float32 else mov, ref, excl)
        return after, before

    def register(self, mov, ref, mask_mov=None, mask_ref=None, out=None):
        calibrate = self.plain_ratio is None or self.frames % self.calibrate_every == 0
        self.frames += 1
        self.net.predict(ref, mov, out=self.init)
        motion = self.fast.register(mov, ref, mask_mov, mask_ref, self.init, out=out,
                                    reuse_reference=self.ref_ready)
        self.ref_ready = True
        a, b = self._ratio(mov, ref, motion, mask_ref)
        r_fast = float(a[0]) / max(float(b[0]), 1e-30)
        if calibrate:
            plain_motion = self.plain.register(mov, ref, mask_mov, mask_ref)
            pa, pb = self._ratio(mov, ref, plain_motion, mask_ref)
            self.plain_ratio = float(pa[0]) / max(float(pb[0]), 1e-30)
        if r_fast > (1.0 + self.margin) * self.plain_ratio:
            self.fallbacks += 1
            motion = self.plain.register(mov, ref, mask_mov, mask_ref, out=out)
        return motion


def time_network(shape=(128, 1024, 1024), train_shape=(64, 256, 256), reps=5, device=None, net=None):
    """Milliseconds (CUDA events) of the network's inference on a (z, y, x)
    pair of ``shape`` (pooling, forward, up-sampling of the field) and of one
    training step at ``train_shape`` (pooling, forward, loss, backward, Adam;
    the target field is zero here, so no registration is timed)."""
    from . import synthetic

    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    if net is None:
        net = WarmStartNet(dev)
        if os.path.exists(DEFAULT_WEIGHTS):
            net.load()

    def ev(fn, n):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(n):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / n

    out = {}
    blobs = max(200, int(20000 * np.prod(shape) / (128 * 1024 * 1024)))
    t, m, _ = synthetic.make_pair(shape, 3, n_blobs=blobs, max_disp=(8.0, 8.0, 3.0), device=dev)
    t, m = t.contiguous(), m.contiguous()
    field = torch.empty(shape + (3,), dtype=torch.float32, device=dev)
    out[f"inference {'x'.join(map(str, shape))}"] = ev(lambda: net.predict(t, m, out=field), reps)
    t, m, _ = synthetic.make_pair(train_shape, 4, n_blobs=2000, max_disp=(8.0, 8.0, 3.0), device=dev)
    t, m = t.float().contiguous(), m.float().contiguous()
    z, y, x = train_shape
    g0 = (z, y // POOL, x // POOL)
    target = torch.zeros((int(np.prod(g0)), 3), dtype=torch.float32, device=dev)
    loss = torch.zeros(1, dtype=torch.float64, device=dev)

    def step():
        net.prepare(t, m, keep_fp32=True)
        pred = net.forward()
        net.zero_grad()
        _lib.check("wr_net_flow_loss", net.lib.wr_net_flow_loss(
            pred.data_ptr(), target.data_ptr(), net._t4.data_ptr(), net._m4.data_ptr(), net.grad["out"].data_ptr(),
            loss.data_ptr(), 1, *g0, float(POOL), 1.0, 1.0, net._stream()))
        net.backward()
        net.adam_step(1e-6)

    out[f"training step {'x'.join(map(str, train_shape))}"] = ev(step, reps)
    flag = ctypes.c_int(-1)
    _lib.check("wr_net_tc_error", net.lib.wr_net_tc_error(ctypes.byref(flag)))
    if flag.value:
        raise RuntimeError("a tensor-core convolution gave up waiting for its MMAs")
    return out


SWEEP_REFINE = ((0, 2), (0, 4), (0, 10), (1, 2), (1, 4), (1, 6), (2, 4), (2, 6), (2, 10), (3, 4))
SWEEP_STARTS = ("zero", "network", "truth", "plain")


def sweep(shape=(128, 1024, 1024), frames=3, refine=SWEEP_REFINE, starts=SWEEP_STARTS, net=None, seed=500,
          precision=_lib.WR_PREC_F32, device=None):
    """What a warm start can buy: short refinements (levels ``layer`` .. 0,
    ``iter`` iterations) started from the zero field, the network's
    prediction, the true synthetic deformation (the best any predictor could
    give) and the plain pyramid's own result, against the plain pyramid
    (layer 3, r 16, iter 10) on config-1-like frames (20k blobs per
    128 x 1024 x 1024, fields up to 8 / 8 / 3 voxels, 70 % ellipsoid mask).

    Returns (rows, plain_ms): per (start, layer, iter) the flow RMS from the
    plain field over all voxels and inside the mask, its max, and the
    milliseconds per frame (CUDA events; the network's prediction included),
    and the plain pyramid's milliseconds per frame."""
    from . import penalty_factor, synthetic

    device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    rng = np.random.default_rng(seed)
    blobs = max(200, int(20000 * np.prod(shape) / (128 * 1024 * 1024)))
    clean = synthetic.render_blobs(shape, blobs, rng, device=device)
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    tmpl_f = torch.poisson(clean, generator=gen)
    del clean
    tmpl = tmpl_f.clamp(0, 65535).round().to(torch.int32).to(torch.uint16).contiguous()
    excl = (~synthetic.ellipsoid_inclusion(shape, 0.7, device=device)).to(torch.uint8).contiguous()
    inside = excl == 0
    pen = 0.08 * float(penalty_factor(tmpl, excl))
    movs, truths = [], []
    for t in range(frames):
        _, mov, field = synthetic.make_pair(shape, seed + 1 + t, max_disp=(8.0, 8.0, 3.0), device=device,
                                            template=tmpl_f)
        movs.append(mov.contiguous())
        truths.append(field.contiguous())
    del tmpl_f
    if net is None and "network" in starts:
        net = WarmStartNet(device)
        net.load()

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        out = fn()
        e1.record()
        torch.cuda.synchronize()
        return out, e0.elapsed_time(e1)

    base = dict(r=16, zRatio=1.0, movRange=5.0, smoothPenalty=pen, tol=1e-3)
    plain = LKRegistrar(shape, LKParams(layer=3, iter=10, precision=_lib.WR_PREC_F32, **base), device)
    plain.register(movs[0], tmpl, excl, excl)                       # warm-up
    plain_m, plain_ms = [], []
    for mov in movs:
        m, ms = timed(lambda: plain.register(mov, tmpl, excl, excl, reuse_reference=True).clone())
        plain_m.append(m)
        plain_ms.append(ms)
    del plain
    torch.cuda.empty_cache()
    init = torch.empty(shape + (3,), dtype=torch.float32, device=device)
    rows = []
    for layer, iters in refine:
        reg = LKRegistrar(shape, LKParams(layer=layer, iter=iters, precision=precision, **base), device)
        reg.register(movs[0], tmpl, excl, excl, motion_init=plain_m[0])   # warm-up, builds the template levels
        for start in starts:
            rms, rms_in, mx, ms = [], [], [], []
            for k, mov in enumerate(movs):
                def run():
                    if start == "network":
                        net.predict(tmpl, mov, out=init)
                    elif start == "truth":
                        init.copy_(truths[k])
                    elif start == "plain":
                        init.copy_(plain_m[k])
                    else:
                        init.zero_()
                    return reg.register(mov, tmpl, excl, excl, motion_init=init, reuse_reference=True)
                m, t_ms = timed(run)
                d = (m - plain_m[k]).float()
                rms.append(float(d.square().mean().sqrt()))
                rms_in.append(float(d[inside].square().mean().sqrt()))
                mx.append(float(d.abs().max()))
                ms.append(t_ms)
            rows.append({"start": start, "layer": layer, "iter": iters, "rms": float(np.mean(rms)),
                         "rms_inside": float(np.mean(rms_in)), "max": float(np.max(mx)),
                         "ms_per_frame": float(np.median(ms))})
        del reg
        torch.cuda.empty_cache()
    return rows, float(np.median(plain_ms))


def main(argv=None):
    import argparse
    import sys

    argv = sys.argv[1:] if argv is None else argv
    if argv[:1] == ["time"]:
        ap = argparse.ArgumentParser(description="time the network: inference on a pair, one training step")
        ap.add_argument("--shape", default="128x1024x1024", help="z x y x x of the inference pair")
        ap.add_argument("--train-shape", default="64x256x256")
        ap.add_argument("--reps", type=int, default=5)
        args = ap.parse_args(argv[1:])
        for name, ms in time_network(tuple(int(v) for v in args.shape.split("x")),
                                     tuple(int(v) for v in args.train_shape.split("x")), args.reps).items():
            print(f"{name}: {ms:.3f} ms")
        return
    if argv[:1] == ["sweep"]:
        ap = argparse.ArgumentParser(description="what a warm start can buy (see sweep())")
        ap.add_argument("--shape", default="128x1024x1024")
        ap.add_argument("--frames", type=int, default=3)
        args = ap.parse_args(argv[1:])
        shape = tuple(int(v) for v in args.shape.split("x"))
        rows, plain_ms = sweep(shape, args.frames)
        print(f"plain pyramid (layer 3, 10 iterations): {plain_ms:.2f} ms per frame")
        print("start     layer iter   RMS all  RMS mask      max   ms/frame  speed-up")
        for r in rows:
            print(f"{r['start']:8s}  {r['layer']:5d} {r['iter']:4d}  {r['rms']:8.4f}  {r['rms_inside']:8.4f}  "
                  f"{r['max']:7.3f}  {r['ms_per_frame']:9.2f}  {plain_ms / r['ms_per_frame']:8.2f}")
        return
    import argparse

    ap = argparse.ArgumentParser(description="train the warm-start network on synthetic pairs")
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--shape", default="64x256x256")
    ap.add_argument("--templates", type=int, default=48)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--res-weight", type=float, default=1.0)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--time-limit", type=float, default=None)
    ap.add_argument("--out", default=DEFAULT_WEIGHTS)
    args = ap.parse_args(argv)
    shape = tuple(int(v) for v in args.shape.split("x"))
    net, hist = train(args.steps, shape, args.templates, args.seed, args.lr, args.res_weight,
                      time_limit=args.time_limit)
    net.save(args.out, steps=hist[-1][0], shape=np.asarray(shape), loss=np.asarray([h[1] for h in hist]),
             wall_s=hist[-1][2])
    print(f"saved {args.out} ({net.parameter_count()} parameters)")


if __name__ == "__main__":
    main()
