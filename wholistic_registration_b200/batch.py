"""Batched registration: many frames, one launch per LK iteration.

The reference registers the frames of a batch one after another with the same
option dict (``utils/registration.py:299-346``).  ``BatchRegistrar`` runs up
to 64 of them together through ``wr_lk_register_batch_each``: every pyramid level
advances all frames with one persistent launch of the fused iteration kernel
per LK iteration (and one launch each of the decision, solve and bookkeeping
kernels), each frame keeping its own stopping state, so each frame's motion
equals a ``LKRegistrar.register`` call on it alone.  Frames may have
different shapes and, with a list of ``LKParams`` (one per frame), their own
patch radius, levels, iterations and penalties; they share the storage
precision.  Small volumes, which leave most of the GPU idle when
registered one by one, gain the most.

``graph=True`` captures the whole batched call into a CUDA graph on the
second call (the first runs eagerly and, with ``reuse_reference``, builds the
template pyramids) and replays it afterwards; the inputs are then copied into
the registrar's own device buffers, and the returned tensors are those
buffers (valid until the next call).
"""

from __future__ import annotations

import ctypes

import torch

from . import _lib
from .registrar import _DTYPES, LKParams, _require_cuda, _stream_ptr


class BatchRegistrar:
    def __init__(self, shapes, params: LKParams, device=None, dtype=torch.uint16, mask_mov=True, mask_ref=True,
                 init=False, warp=False, graph=False):
        self.lib = _lib.load()
        self.shapes = [tuple(int(v) for v in s) for s in shapes]
        self.n = len(self.shapes)
        if not 1 <= self.n <= _lib.MAX_BATCH:
            raise ValueError(f"a batch holds 1..{_lib.MAX_BATCH} frames")
        if dtype not in _DTYPES:
            raise ValueError(f"dtype {dtype} not supported (uint8, uint16, float32)")
        plist = list(params) if isinstance(params, (list, tuple)) else [params] * self.n
        if len(plist) != self.n:
            raise ValueError(f"params: one LKParams for the batch or one per frame ({self.n})")
        self.params = plist
        self.dtype = dtype
        self.has_mmov, self.has_mref, self.has_init, self.has_warp = bool(mask_mov), bool(mask_ref), bool(init), bool(warp)
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self._cps = (_lib.WrLKParams * self.n)(*[q.to_c() for q in plist])
        self._items = (_lib.WrLKItem * self.n)()
        one = ctypes.c_void_p(1)   # placeholder pointers: the size query reads shapes and presence only
        for i, s in enumerate(self.shapes):
            it = self._items[i]
            it.mov = _lib.volume(1, _DTYPES[dtype], s)
            it.ref = _lib.volume(1, _DTYPES[dtype], s)
            it.excl_mask_mov = one if self.has_mmov else None
            it.excl_mask_ref = one if self.has_mref else None
            it.motion_init = one if self.has_init else None
        nbytes = ctypes.c_size_t(0)
        _lib.check("wr_lk_batch_each_workspace_size",
                   self.lib.wr_lk_batch_each_workspace_size(self._items, self._cps, self.n, ctypes.byref(nbytes)))
        self.workspace_bytes = int(nbytes.value)
        self.workspace = torch.empty(self.workspace_bytes + 256, dtype=torch.uint8, device=self.device)
        self._ws_ptr = (self.workspace.data_ptr() + 255) // 256 * 256
        self.stats_dev = torch.zeros((self.n, ctypes.sizeof(_lib.WrLKStats)), dtype=torch.uint8, device=self.device)
        self.motion = [torch.empty(s + (3,), dtype=torch.float32, device=self.device) for s in self.shapes]
        self.warped = [torch.empty(s, dtype=torch.float32, device=self.device) for s in self.shapes] if warp else None
        # launch-shape bits of WrLKParams.flags (autotune.candidates()); results do not depend on them
        self.tune_flags = 0
        self.graph = graph
        self._graph = None
        self._calls = 0
        if graph:
            self._in = {
                "mov": [torch.empty(s, dtype=dtype, device=self.device) for s in self.shapes],
                "ref": [torch.empty(s, dtype=dtype, device=self.device) for s in self.shapes],
                "mask_mov": [torch.empty(s, dtype=torch.uint8, device=self.device) for s in self.shapes]
                if self.has_mmov else None,
                "mask_ref": [torch.empty(s, dtype=torch.uint8, device=self.device) for s in self.shapes]
                if self.has_mref else None,
                "init": [torch.empty(s + (3,), dtype=torch.float32, device=self.device) for s in self.shapes]
                if self.has_init else None,
            }

    # -- checks --------------------------------------------------------------------------------------------------
    def _check(self, ts, name, shape_of, dtype, present):
        if not present:
            if ts is not None:
                raise ValueError(f"{name} given to a registrar built without it")
            return None
        if ts is None or len(ts) != self.n:
            raise ValueError(f"{name}: one tensor per frame expected ({self.n})")
        out = []
        for i, t in enumerate(ts):
            _require_cuda(t, name)
            if tuple(t.shape) != shape_of(i):
                raise ValueError(f"{name}[{i}] must have shape {shape_of(i)}")
            if dtype is torch.uint8 and t.dtype == torch.bool:
                t = t.view(torch.uint8)
            if t.dtype != dtype:
                raise ValueError(f"{name}[{i}] must be {dtype}")
            out.append(t)
        return out

    def _launch(self, movs, refs, mmovs, mrefs, inits, flags, stream):
        for i in range(self.n):
            it = self._items[i]
            it.mov = _lib.volume(movs[i].data_ptr(), _DTYPES[self.dtype], self.shapes[i])
            it.ref = _lib.volume(refs[i].data_ptr(), _DTYPES[self.dtype], self.shapes[i])
            it.excl_mask_mov = mmovs[i].data_ptr() if mmovs else None
            it.excl_mask_ref = mrefs[i].data_ptr() if mrefs else None
            it.motion_init = inits[i].data_ptr() if inits else None
            it.motion_out = self.motion[i].data_ptr()
            it.warped_out = self.warped[i].data_ptr() if self.warped else None
            it.stats = self.stats_dev[i].data_ptr()
        for i in range(self.n):
            self._cps[i].flags = flags
        _lib.check("wr_lk_register_batch_each",
                   self.lib.wr_lk_register_batch_each(self._items, self._cps, self.n, self._ws_ptr,
                                                      self.workspace_bytes, stream))

    # -- API -------------------------------------------------------------------------------------------------------
    def register(self, movs, refs, masks_mov=None, masks_ref=None, inits=None, reuse_reference=False):
        """Motions (list of (z, y, x, 3) float32) of the frames; with ``warp``
        also the warped frames.  ``reuse_reference`` keeps each frame's
        template pyramid from the previous call (a series against fixed
        templates)."""
        shape_of = lambda i: self.shapes[i]
        movs = self._check(movs, "movs", shape_of, self.dtype, True)
        refs = self._check(refs, "refs", shape_of, self.dtype, True)
        mmovs = self._check(masks_mov, "masks_mov", shape_of, torch.uint8, self.has_mmov)
        mrefs = self._check(masks_ref, "masks_ref", shape_of, torch.uint8, self.has_mref)
        inits = self._check(inits, "inits", lambda i: self.shapes[i] + (3,), torch.float32, self.has_init)
        flags = self.tune_flags | (_lib.WR_LK_REUSE_REFERENCE if reuse_reference else 0)
        if not self.graph:
            self._launch(movs, refs, mmovs, mrefs, inits, flags, _stream_ptr())
            return (self.motion, self.warped) if self.warped else self.motion
        src = {"mov": movs, "ref": refs, "mask_mov": mmovs, "mask_ref": mrefs, "init": inits}
        for k, ts in src.items():
            if ts is not None:
                for d, t in zip(self._in[k], ts):
                    d.copy_(t)
        if self._graph is None and self._calls >= 1:
            # capture on a side stream (torch.cuda.graph's requirement); the eager first call did the warm-up
            self._graph = torch.cuda.CUDAGraph()
            self._graph_flags = flags
            with torch.cuda.graph(self._graph):
                self._launch(self._in["mov"], self._in["ref"], self._in["mask_mov"], self._in["mask_ref"],
                             self._in["init"], flags, _stream_ptr())
        if self._graph is not None:
            if flags != self._graph_flags:
                raise ValueError("a captured batch replays with the flags it was captured with")
            self._graph.replay()
        else:
            self._launch(self._in["mov"], self._in["ref"], self._in["mask_mov"], self._in["mask_ref"],
                         self._in["init"], flags, _stream_ptr())
        self._calls += 1
        return (self.motion, self.warped) if self.warped else self.motion

    def stats(self):
        host = self.stats_dev.cpu().numpy()
        return [_lib.WrLKStats.from_buffer_copy(host[i].tobytes()) for i in range(self.n)]
