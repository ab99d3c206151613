"""Device-level entry point: (z, y, x) CUDA tensors in, (z, y, x, 3) motion out.

``LKRegistrar`` owns a workspace for one volume shape and parameter set and
calls the C ABI (``wr_lk_register``, ``wr_warp_trilinear``) on the current
torch CUDA stream.  ``getMotion`` / ``correctMotion`` in
``calFlow3d_Wei_v1`` wrap it with the reference's NumPy calling convention.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import torch

from . import _lib

_DTYPES = {
    torch.uint16: _lib.WR_U16,
    torch.uint8: _lib.WR_U8,
    torch.float32: _lib.WR_F32,
}


@dataclass
class LKParams:
    """The getMotion option keys (utils/calFlow3d_Wei_v1.py:318-324,429-431).

    ``forced_updates`` (layer -> count) replays another run's per-level update
    counts instead of applying the stopping rules.
    """

    layer: int = 3
    iter: int = 10
    r: int = 5
    zRatio: float = 27.693
    movRange: float = 5.0
    smoothPenalty: float = 0.0
    tol: float = 1e-4
    precision: int = _lib.WR_PREC_F32
    forced_updates: dict = field(default_factory=dict)

    @classmethod
    def from_option(cls, option) -> "LKParams":
        return cls(
            layer=int(option["layer"]), iter=int(option["iter"]), r=int(option["r"]),
            zRatio=float(option["zRatio"]), movRange=float(option.get("movRange", 5.0)),
            smoothPenalty=float(option["smoothPenalty"]), tol=float(option["tol"]),
            precision=int(option.get("precision", _lib.WR_PREC_F32)),
            forced_updates=dict(option.get("forced_updates") or {}),
        )

    def to_c(self) -> _lib.WrLKParams:
        p = _lib.WrLKParams()
        p.layer, p.iter, p.r = self.layer, self.iter, self.r
        p.zRatio, p.movRange = self.zRatio, self.movRange
        p.smoothPenalty, p.tol = self.smoothPenalty, self.tol
        p.precision = self.precision
        for i in range(_lib.MAX_LEVELS):
            p.forced_updates[i] = int(self.forced_updates.get(i, -1))
        return p


def _stream_ptr(stream=None) -> int:
    s = stream if stream is not None else torch.cuda.current_stream()
    return int(s.cuda_stream)


def _require_cuda(t: torch.Tensor, name: str):
    if not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous (z, y, x)")


def _vol(t: torch.Tensor, name: str) -> _lib.WrVolume:
    _require_cuda(t, name)
    if t.dim() != 3:
        raise ValueError(f"{name} must be a 3-D (z, y, x) volume")
    if t.dtype not in _DTYPES:
        raise ValueError(f"{name}: dtype {t.dtype} not supported (uint8, uint16, float32)")
    return _lib.volume(t.data_ptr(), _DTYPES[t.dtype], t.shape)


def stats_to_log(st: _lib.WrLKStats, layers: int) -> tuple[dict, float]:
    """error_log dict in the reference's shape (utils/calFlow3d_Wei_v1.py:329-335)."""
    log = {}
    for layer in range(layers - 1, -1, -1):
        # the device keeps at most WR_MAX_ITERS entries per level
        e, u = min(st.evals[layer], _lib.MAX_ITERS), min(st.updates[layer], _lib.MAX_ITERS)
        diff = [st.diff_error[layer][i] for i in range(e)]
        pen = [st.penalty_error[layer][i] for i in range(e)]
        log[f"layer_{layer}"] = {
            "diffError": diff,
            "penaltyError": pen,
            "currentError": [a + b for a, b in zip(diff, pen)],
            "max_diff_motion": [st.max_diff_motion[layer][i] for i in range(u)],
            "motion_current": [],
            "data_mov_corrected": [],
        }
    return log, float(st.current_error)


class LKRegistrar:
    """Pyramid Lucas-Kanade registration of (z, y, x) volumes on one GPU."""

    def __init__(self, shape_zyx, params: LKParams, device=None):
        self.lib = _lib.load()
        self.shape = tuple(int(s) for s in shape_zyx)
        self.params = params
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self._cp = params.to_c()
        nbytes = ctypes.c_size_t(0)
        _lib.check("wr_lk_workspace_size",
                   self.lib.wr_lk_workspace_size(*self.shape, ctypes.byref(self._cp), ctypes.byref(nbytes)))
        self.workspace_bytes = int(nbytes.value)
        self.workspace = torch.empty(self.workspace_bytes + 256, dtype=torch.uint8, device=self.device)
        base = self.workspace.data_ptr()
        self._ws_ptr = (base + 255) // 256 * 256
        self.stats_dev = torch.zeros(ctypes.sizeof(_lib.WrLKStats), dtype=torch.uint8, device=self.device)
        # launch-shape bits of WrLKParams.flags (tile order, CTAs per SM); results do not depend on them
        self.tune_flags = 0

    def set_params(self, params: LKParams) -> None:
        """Use other solver parameters from the next call on; the workspace
        must still suffice (ValueError otherwise), which it does for the same
        patch radius and number of levels."""
        cp = params.to_c()
        nbytes = ctypes.c_size_t(0)
        _lib.check("wr_lk_workspace_size",
                   self.lib.wr_lk_workspace_size(*self.shape, ctypes.byref(cp), ctypes.byref(nbytes)))
        if int(nbytes.value) > self.workspace_bytes:
            raise ValueError("these parameters need a larger workspace than this registrar holds")
        self.params, self._cp = params, cp

    def autotune(self, dtype=torch.uint16, mask=True, use_cache=True, report=None) -> int:
        """Pick the fused kernel's launch shape for this registrar's shape and
        parameters (``autotune.tune``, cached) and use it from now on."""
        from . import autotune

        self.tune_flags = autotune.tune(self.shape, self.params, dtype=dtype, mask=mask, device=self.device,
                                        use_cache=use_cache, report=report)
        return self.tune_flags

    def register(self, mov: torch.Tensor, ref: torch.Tensor, mask_mov=None, mask_ref=None,
                 motion_init=None, out=None, stream=None, profile=None, reuse_reference=False,
                 warped_out=None, snapshots=None) -> torch.Tensor:
        """Motion (z, y, x, 3) float32 registering ``mov`` onto ``ref``.

        Masks are (z, y, x) uint8/bool exclusion masks (True = excluded) or
        None; ``motion_init`` is a (z, y, x, 3) float32 initial field or None.
        ``reuse_reference`` keeps the reference pyramid and reference mask
        built by the previous call on this registrar (same ``ref`` and
        ``mask_ref``), as when registering a time series to one template.
        ``warped_out`` (float32 (z, y, x)) also receives ``mov`` warped by the
        motion (correctMotion), written in the same pass as the motion.
        """
        if tuple(mov.shape) != self.shape or tuple(ref.shape) != self.shape:
            raise ValueError(f"volumes must have shape {self.shape}")
        vm, vr = _vol(mov, "mov"), _vol(ref, "ref")
        ptrs = []
        for m, name in ((mask_mov, "mask_mov"), (mask_ref, "mask_ref")):
            if m is None:
                ptrs.append(None)
                continue
            _require_cuda(m, name)
            if tuple(m.shape) != self.shape:
                raise ValueError(f"{name} must have shape {self.shape}")
            if m.dtype == torch.bool:
                m = m.view(torch.uint8)
            if m.dtype != torch.uint8:
                raise ValueError(f"{name} must be bool or uint8")
            ptrs.append(m.data_ptr())
        init_ptr = None
        if motion_init is not None:
            _require_cuda(motion_init, "motion_init")
            if tuple(motion_init.shape) != self.shape + (3,) or motion_init.dtype != torch.float32:
                raise ValueError("motion_init must be float32 (z, y, x, 3)")
            init_ptr = motion_init.data_ptr()
        if out is None:
            out = torch.empty(self.shape + (3,), dtype=torch.float32, device=self.device)
        self._cp.flags = self.tune_flags | (_lib.WR_LK_REUSE_REFERENCE if reuse_reference else 0)
        args = (ctypes.byref(vm), ctypes.byref(vr), ptrs[0], ptrs[1], ctypes.byref(self._cp), init_ptr,
                out.data_ptr(), self.stats_dev.data_ptr(), self._ws_ptr, self.workspace_bytes, _stream_ptr(stream))
        prof = ctypes.byref(profile.begin_call()) if profile is not None else None
        if snapshots is not None:
            # getMotion's error_log snapshots (a _lib.WrSnapshots of device buffers)
            if warped_out is not None or profile is not None:
                raise ValueError("snapshots cannot be combined with warped_out or profile")
            _lib.check("wr_lk_register_snapshots",
                       self.lib.wr_lk_register_snapshots(*args, ctypes.byref(snapshots)))
            return out
        if warped_out is not None:
            _require_cuda(warped_out, "warped_out")
            if tuple(warped_out.shape) != self.shape or warped_out.dtype != torch.float32 \
                    or not warped_out.is_contiguous():
                raise ValueError("warped_out must be contiguous float32 (z, y, x)")
            _lib.check("wr_lk_register_warp",
                       self.lib.wr_lk_register_warp(*args[:7], warped_out.data_ptr(), *args[7:], prof))
        elif profile is None:
            _lib.check("wr_lk_register", self.lib.wr_lk_register(*args))
        else:
            _lib.check("wr_lk_register_profiled", self.lib.wr_lk_register_profiled(*args, prof))
        return out

    def stats(self) -> _lib.WrLKStats:
        """Statistics of the last call (synchronises the stream)."""
        host = self.stats_dev.cpu().numpy().tobytes()
        return _lib.WrLKStats.from_buffer_copy(host)

    def error_log(self):
        return stats_to_log(self.stats(), self.params.layer + 1)


class KernelProfile:
    """CUDA events around every launch of the fused iteration kernel.

    ``begin_call`` hands a fresh slice of events to one registration call;
    ``durations_ms`` (after a synchronize) returns one list per call.
    """

    def __init__(self, calls: int, per_call: int):
        self.per_call = per_call
        self.begin = [torch.cuda.Event(enable_timing=True) for _ in range(calls * per_call)]
        self.end = [torch.cuda.Event(enable_timing=True) for _ in range(calls * per_call)]
        for e in self.begin + self.end:
            e.record()  # creates the underlying cudaEvent_t
        torch.cuda.synchronize()
        self._bh = (ctypes.c_void_p * len(self.begin))(*[e.cuda_event for e in self.begin])
        self._eh = (ctypes.c_void_p * len(self.end))(*[e.cuda_event for e in self.end])
        self.calls = 0
        self.launches = []
        self.recorded = []
        self._prof = None

    def begin_call(self) -> _lib.WrProfile:
        if self._prof is not None:
            self.recorded.append(self._prof.recorded)
            self.launches.append(self._prof.launches)
        off = self.calls * self.per_call
        if off + self.per_call > len(self.begin):
            raise RuntimeError("KernelProfile: out of events")
        p = _lib.WrProfile()
        p.acc_begin = ctypes.cast(ctypes.byref(self._bh, off * ctypes.sizeof(ctypes.c_void_p)),
                                  ctypes.POINTER(ctypes.c_void_p))
        p.acc_end = ctypes.cast(ctypes.byref(self._eh, off * ctypes.sizeof(ctypes.c_void_p)),
                                ctypes.POINTER(ctypes.c_void_p))
        p.capacity = self.per_call
        self.calls += 1
        self._prof = p
        return p

    def finish(self):
        if self._prof is not None:
            self.recorded.append(self._prof.recorded)
            self.launches.append(self._prof.launches)
            self._prof = None

    def durations_ms(self):
        self.finish()
        out = []
        for c in range(self.calls):
            base = c * self.per_call
            out.append([self.begin[base + i].elapsed_time(self.end[base + i]) for i in range(self.recorded[c])])
        return out


def warp(src: torch.Tensor, motion: torch.Tensor, out=None, stream=None) -> torch.Tensor:
    """correctMotion on the device: out(p) = src(p + motion(p)), float32."""
    lib = _lib.load()
    vs = _vol(src, "src")
    _require_cuda(motion, "motion")
    if tuple(motion.shape) != tuple(src.shape) + (3,) or motion.dtype != torch.float32:
        raise ValueError("motion must be float32 (z, y, x, 3) matching src")
    if out is None:
        out = torch.empty(tuple(src.shape), dtype=torch.float32, device=src.device)
    _lib.check("wr_warp_trilinear", lib.wr_warp_trilinear(ctypes.byref(vs), motion.data_ptr(), out.data_ptr(),
                                                         _stream_ptr(stream)))
    return out


def penalty_factor(ref: torch.Tensor, mask_ref=None, stream=None) -> torch.Tensor:
    """getSmPnltNormFctr (utils/preprocess.py:42-66) on the device; returns a
    0-d float64 CUDA tensor."""
    lib = _lib.load()
    vr = _vol(ref, "ref")
    nbytes = ctypes.c_size_t(0)
    _lib.check("wr_penalty_factor_scratch", lib.wr_penalty_factor_scratch(*ref.shape, ctypes.byref(nbytes)))
    scratch = torch.empty(int(nbytes.value), dtype=torch.uint8, device=ref.device)
    out = torch.empty((), dtype=torch.float64, device=ref.device)
    mptr = None
    if mask_ref is not None:
        _require_cuda(mask_ref, "mask_ref")
        mptr = (mask_ref.view(torch.uint8) if mask_ref.dtype == torch.bool else mask_ref).data_ptr()
    _lib.check("wr_penalty_factor", lib.wr_penalty_factor(ctypes.byref(vr), mptr, out.data_ptr(),
                                                         scratch.data_ptr(), int(nbytes.value), _stream_ptr(stream)))
    return out
