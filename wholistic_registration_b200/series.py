"""Time-series registration from host memory.

The reference registers a batch of frames against one template frame by frame
(utils/registration.py:299-346): for each frame, getMotion then correctMotion,
with the volumes copied to the device and the results copied back.
``SeriesRegistrar`` does the same on one GPU with the copies overlapped with
compute: frame t+1 is copied in and frame t-1's motion and warped volume are
copied out while frame t registers.
"""

from __future__ import annotations

import torch

from .registrar import LKParams, LKRegistrar


class SeriesRegistrar:
    """Register host (z, y, x) frames onto a device-resident template.

    Host buffers should be pinned (``torch.empty(..., pin_memory=True)``) for
    the copies to overlap.  ``depth`` device buffers of each kind are cycled.
    """

    def __init__(self, template: torch.Tensor, params: LKParams, mask_ref=None, mask_mov=None, depth: int = 2,
                 frame_dtype=torch.uint16):
        self.template = template
        self.shape = tuple(template.shape)
        self.device = template.device
        self.params = params
        self.mask_ref = mask_ref
        self.mask_mov = mask_mov
        self.reg = LKRegistrar(self.shape, params, self.device)
        self.depth = depth
        self.s_in = torch.cuda.Stream(self.device)
        self.s_run = torch.cuda.Stream(self.device)
        self.s_out = torch.cuda.Stream(self.device)
        self.d_in = [torch.empty(self.shape, dtype=frame_dtype, device=self.device) for _ in range(depth)]
        self.d_motion = [torch.empty(self.shape + (3,), dtype=torch.float32, device=self.device) for _ in range(depth)]
        self.d_warp = [torch.empty(self.shape, dtype=torch.float32, device=self.device) for _ in range(depth)]
        self.in_free = [torch.cuda.Event() for _ in range(depth)]
        self.in_ready = [torch.cuda.Event() for _ in range(depth)]
        self.out_ready = [torch.cuda.Event() for _ in range(depth)]
        self.out_free = [torch.cuda.Event() for _ in range(depth)]
        self.started = [False] * depth
        self.ref_ready = False   # the registrar's workspace holds the template pyramid

    def bytes_per_frame(self):
        n = 1
        for s in self.shape:
            n *= s
        esize = self.d_in[0].element_size()
        return n * esize, n * 12 + n * 4

    def run(self, frames, motion_out, warped_out, mask_mov=None):
        """Register ``frames[t]`` (host) into ``motion_out[t]`` (z,y,x,3) and
        ``warped_out[t]`` (z,y,x) (host, float32).  Returns when all copies
        are queued; synchronise (or use ``done``) before reading outputs."""
        mask_mov = self.mask_mov if mask_mov is None else mask_mov
        # the template and masks were written on the caller's stream
        self.s_run.wait_stream(torch.cuda.current_stream(self.device))
        for t, frame in enumerate(frames):
            k = t % self.depth
            with torch.cuda.stream(self.s_in):
                if self.started[k]:
                    self.s_in.wait_event(self.in_free[k])
                self.d_in[k].copy_(frame, non_blocking=True)
                self.in_ready[k].record(self.s_in)
            with torch.cuda.stream(self.s_run):
                self.s_run.wait_event(self.in_ready[k])
                if self.started[k]:
                    self.s_run.wait_event(self.out_free[k])
                # motion and the frame warped by it (correctMotion) in one call
                self.reg.register(self.d_in[k], self.template, mask_mov, self.mask_ref, None,
                                  out=self.d_motion[k], stream=self.s_run, reuse_reference=self.ref_ready,
                                  warped_out=self.d_warp[k])
                self.ref_ready = True
                self.in_free[k].record(self.s_run)
                self.out_ready[k].record(self.s_run)
            with torch.cuda.stream(self.s_out):
                self.s_out.wait_event(self.out_ready[k])
                motion_out[t].copy_(self.d_motion[k], non_blocking=True)
                warped_out[t].copy_(self.d_warp[k], non_blocking=True)
                self.out_free[k].record(self.s_out)
            self.started[k] = True
        return self.s_out

    def done(self):
        self.s_out.synchronize()
