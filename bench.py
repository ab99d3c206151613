"""Benchmark of the pyramid Lucas-Kanade registration path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
    python -m torch.distributed.run --nproc-per-node N ... bench.py --gpus N   (one rank per GPU)

A step registers one synthetic time-series frame (128 x 1024 x 1024 uint16,
70 % ellipsoid inclusion mask, 4 pyramid levels, 33 x 33 patches, up to 10
iterations per level) onto the template and warps it (getMotion +
correctMotion).  Frames are independent, so N ranks each register their own
frames (weak scaling, no collective on the data path).

``value`` is volumes/s with the frames resident in HBM; ``e2e`` is the same
metric through the host-memory time-series API (pinned host frames in,
motion + warped volume out, copies overlapped with compute).
``--impl reference`` times the CPU oracle port of the reference algorithm
(the reference's scipy correlate cost) on all host cores over a bounded sample
and extrapolates to volumes/s.
"""

from __future__ import annotations

import argparse
import json
import math
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}
# DRAM bytes (read + write) per level voxel of one k_lk_accumulate launch, measured with
# ncu (dram__bytes_read.sum + dram__bytes_write.sum) on a level-0 launch of the
# 64x512x512 workload (366.7 MB for 16.78 M voxels); the traffic of a launch grows with
# the voxels it processes, so the bench scales it to its own launches.
TRAFFIC_BYTES_PER_VOXEL = 21.86

WORKLOADS = {
    # z, y, x, frames, blobs, max displacement (x, y, z), drift, mask coverage, layer, r, iter
    "series-128x1024x1024": dict(shape=(128, 1024, 1024), frames=32, blobs=20000, max_disp=(8.0, 8.0, 3.0),
                                 drift=0.05, coverage=0.70, layer=3, r=16, iter=10),
    "profile-64x512x512": dict(shape=(64, 512, 512), frames=2, blobs=5000, max_disp=(8.0, 8.0, 3.0),
                               drift=0.05, coverage=0.70, layer=3, r=16, iter=10),
    "single-64x256x256": dict(shape=(64, 256, 256), frames=4, blobs=2000, max_disp=(4.0, 4.0, 1.5),
                              drift=0.0, coverage=None, layer=2, r=16, iter=10),
}
METRIC = "volumes/s on 1 B200: warm-start+mixed-precision vs plain at ≤0.1 vox RMS error"
CPU_SLAB = (8, 256, 256)   # z, y, x voxels of one CPU sample (one LK iteration at full resolution)


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            d = json.load(fh)
        return {"hbm_gbs": float(d["hbm_gbs"]), "bf16_tflops": float(d["bf16_tflops"])}, "measured"
    except Exception:
        return dict(PEAKS_FALLBACK), "fallback"


# ---------------------------------------------------------------------------
# CPU baseline: the oracle port with the reference's correlate cost
# ---------------------------------------------------------------------------

def _cpu_sample(seed):
    """One LK iteration (warp, It, gradients, nine (2r+1)^2 correlations,
    solve, update) plus two error evaluations at full resolution on one slab."""
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    import numpy as np

    from oracle import lk_oracle as O

    rng = np.random.default_rng(seed)
    z, y, x = CPU_SLAB
    ref = rng.uniform(100, 1000, size=(x, y, z))
    mov = np.roll(ref, 1, axis=0)
    excl = np.zeros((x, y, z), bool)
    opt = {"mask_ref": excl, "mask_mov": excl, "layer": 0, "iter": 2, "r": 16, "zRatio": 1.0, "movRange": 5.0,
           "motion": None, "smoothPenalty": 1.0, "tol": 1e-3}
    t = time.perf_counter()
    O.get_motion(mov, ref, opt, window_sums="correlate")
    return time.perf_counter() - t


def cpu_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def cpu_rate(pool, cores, reps=1):
    """Seconds per voxel-iteration per core (median over the cores' samples)."""
    times = []
    for r in range(reps):
        times += pool.map(_cpu_sample, [1000 * r + i for i in range(cores)])
    n = CPU_SLAB[0] * CPU_SLAB[1] * CPU_SLAB[2]
    return statistics.median(times) / n, times


def voxel_iters_per_volume(wl, updates=None):
    z, y, x = wl["shape"]
    tot = 0.0
    for l in range(wl["layer"] + 1):
        u = updates[l] if updates is not None else wl["iter"] - 1
        tot += z * int(y / 2 ** l) * int(x / 2 ** l) * u
    return tot


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------

class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 100 ms."""

    FIELDS = ("timestamp,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.proc = None
        self.rows = []
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100",
                 "-i", str(gpu_index)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out, _ = self.proc.communicate()
        for line in out.splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) == 9:
                self.rows.append(parts)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        def num(v):
            try:
                return float(v)
            except ValueError:
                return None
        sm = [num(r[1]) for r in self.rows if num(r[1]) is not None]
        mx = [num(r[2]) for r in self.rows if num(r[2]) is not None]
        pw = [num(r[3]) for r in self.rows if num(r[3]) is not None]
        busy = [num(r[1]) for r in self.rows if num(r[3]) is not None and num(r[3]) > 300 and num(r[1]) is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(busy or sm) if (busy or sm) else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(self.rows),
                "samples_under_load": len(busy), "power_w_max": max(pw) if pw else None}


def make_workload(wl, device, n_frames, seed0):
    import torch

    from wholistic_registration_b200 import penalty_factor, synthetic
    import numpy as np

    shape = wl["shape"]
    rng = np.random.default_rng(seed0)
    clean = synthetic.render_blobs(shape, wl["blobs"], rng, device=device)
    gen = torch.Generator(device=device)
    gen.manual_seed(seed0)
    tmpl_f = torch.poisson(clean, generator=gen)
    del clean
    template = tmpl_f.clamp(0, 65535).round().to(torch.int32).to(torch.uint16)
    if wl["coverage"] is not None:
        excl = ~synthetic.ellipsoid_inclusion(shape, wl["coverage"], device=device)
        excl = excl.to(torch.uint8).contiguous()
    else:
        excl = None
    frames = []
    total = wl["frames"]
    for t in range(n_frames):
        drift = wl["drift"] * (t % total) / max(total - 1, 1)
        _, mov, _ = synthetic.make_pair(shape, seed0 + 1 + t, max_disp=wl["max_disp"], drift=drift, device=device,
                                        template=tmpl_f)
        frames.append(mov)
        torch.cuda.empty_cache()
    factor = float(penalty_factor(template, excl))
    return template, excl, frames, factor


def run_ours(args, wl, rank, world, local_rank):
    import torch
    import torch.distributed as dist

    from wholistic_registration_b200 import LKParams, LKRegistrar
    from wholistic_registration_b200.registrar import KernelProfile
    from wholistic_registration_b200.series import SeriesRegistrar

    torch.cuda.set_device(local_rank)
    device = torch.device("cuda", local_rank)
    n_frames = min(wl["frames"], max(args.frames, 1))
    template, excl, frames, factor = make_workload(wl, device, n_frames, seed0=1000 + 97 * rank)
    prec = {"f32": 0, "f16": 1, "bf16": 2}[args.precision]
    params = LKParams(layer=wl["layer"], iter=wl["iter"], r=wl["r"], zRatio=1.0, movRange=5.0,
                      smoothPenalty=0.08 * factor, tol=1e-3, precision=prec)
    reg = LKRegistrar(wl["shape"], params, device)
    motion = torch.empty(wl["shape"] + (3,), dtype=torch.float32, device=device)
    warped = torch.empty(wl["shape"], dtype=torch.float32, device=device)
    stats_hist = torch.zeros((args.steps, reg.stats_dev.numel()), dtype=torch.uint8, device=device)

    ref_ready = [False]

    def step(k, prof=None, keep_stats=False):
        f = frames[k % len(frames)]
        # the template's pyramid is built by the first call and reused for the series
        # registration and correctMotion of the frame in one call
        reg.register(f, template, excl, excl, None, out=motion, profile=prof, reuse_reference=ref_ready[0],
                     warped_out=warped)
        ref_ready[0] = True
        if keep_stats:
            stats_hist[k].copy_(reg.stats_dev, non_blocking=True)

    tune_report = {}
    if not args.no_autotune:
        # launch shape of the fused kernel for this workload (results do not depend on it)
        reg.autotune(dtype=frames[0].dtype, mask=True, use_cache=False, report=tune_report)
    for k in range(args.warmup):
        step(k)
    torch.cuda.synchronize()
    prof = KernelProfile(args.steps, wl["iter"] * (wl["layer"] + 1))
    clocks = ClockSampler(local_rank) if rank == 0 else None
    time.sleep(0.3)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for k in range(args.steps):
        step(k, prof, keep_stats=True)
    e1.record()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    if clocks:
        clocks.stop()
    ms = e0.elapsed_time(e1)
    if world > 1:
        t = torch.tensor([ms], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())

    # roofline of the fused iteration kernel over its active launches
    from wholistic_registration_b200 import _lib

    durs = prof.durations_ms()
    bpv = 10.0 if args.precision == "f32" else 6.0
    st_bytes = stats_hist.cpu().numpy()
    z, y, x = wl["shape"]
    levels = wl["layer"] + 1
    alg_bytes = 0.0
    act_ms = 0.0
    idle_ms = 0.0
    active_launches = 0
    updates_sum = [0] * levels
    evals_sum = [0] * levels
    for k in range(args.steps):
        st = _lib.WrLKStats.from_buffer_copy(st_bytes[k].tobytes())
        i = 0
        for l in range(levels - 1, -1, -1):
            n_l = z * int(y / 2 ** l) * int(x / 2 ** l)
            evals_sum[l] += st.evals[l]
            updates_sum[l] += st.updates[l]
            for it in range(wl["iter"]):
                d = durs[k][i]
                i += 1
                if it < st.evals[l]:
                    alg_bytes += n_l * bpv   # ref + moving level (storage precision) + two 1-byte masks
                    act_ms += d
                    active_launches += 1
                else:
                    idle_ms += d
    launches_per_step = prof.launches[0] + 1 if prof.launches else None
    pk, pk_kind = peaks()
    achieved = alg_bytes / (act_ms * 1e-3) / 1e9 if act_ms > 0 else None
    n_vox = z * y * x
    b_vol = n_vox * 5.0 + sum(z * int(y / 2 ** l) * int(x / 2 ** l) * 10.0 for l in range(levels))
    b_vol += sum(z * int(y / 2 ** l) * int(x / 2 ** l) * 10.0 * evals_sum[l] / args.steps for l in range(levels))
    b_vol += n_vox * 18.0
    vps = world * args.steps / (ms * 1e-3)
    res = {
        "metric": METRIC, "value": round(vps, 3), "unit": "volumes/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": args.precision, "data": "synthetic",
        "config": {
            "workload": args.workload, "shape_zyx": list(wl["shape"]), "frames_resident": n_frames,
            "layer": wl["layer"], "r": wl["r"], "iter": wl["iter"],
            "path": {"f32": "plain-fp32", "f16": "plain, levels in float16", "bf16": "plain, levels in bfloat16"}[args.precision],
            "mask": f"ellipsoid inclusion {wl['coverage']}" if wl["coverage"] else "none",
            "l2": (f"inputs larger than L2: each frame {n_vox * 2 / 1e6:.0f} MB, its level-0 moving level "
                   f"(m, Gx, Gy, Gz) {n_vox * 16 / 1e6:.0f} MB, L2 126 MB"),
            "parallelism": f"frames sharded over {world} rank(s), no collective",
            "evals_per_level_mean": [round(evals_sum[l] / args.steps, 2) for l in range(levels)],
            "updates_per_level_mean": [round(updates_sum[l] / args.steps, 2) for l in range(levels)],
            "gvox_per_s": round(vps * n_vox / 1e9, 3),
            "pipeline_hbm_frac": round(b_vol * vps / world / 1e9 / pk["hbm_gbs"], 4),
            "algorithmic_bytes_per_volume": round(b_vol),
        },
        "roofline": {
            "kernel": "k_lk_accumulate (fused warp + It + gradients + window sums)",
            "bound": "hbm", "achieved": round(achieved, 1) if achieved else None, "peak": pk["hbm_gbs"],
            "unit": "GB/s", "frac": round(achieved / pk["hbm_gbs"], 4) if achieved else None,
            "peak_kind": pk_kind,
            "traffic": round(alg_bytes / bpv * TRAFFIC_BYTES_PER_VOXEL / active_launches) if active_launches else None,
            "traffic_note": "bytes per active launch: ncu-measured DRAM bytes per voxel x voxels per launch",
            "active_launches": active_launches,
            "active_ms_per_step": round(act_ms / args.steps, 4), "idle_launch_ms_per_step": round(idle_ms / args.steps, 4),
            "bytes_per_voxel": bpv,
        },
        "gpu_launches": (launches_per_step * args.steps) if launches_per_step else None,
        "clocks": clocks.summary() if clocks else None,
    }
    res["config"]["autotune"] = {"flags": reg.tune_flags, "ms_per_candidate": tune_report} if tune_report else None
    if not args.no_batch:
        res["config"]["batched_small_frames"] = run_batched_small(device)
        res["config"]["uneven_batch"] = run_uneven_batch(device)
    if not args.no_xres:
        res["config"]["cross_resolution"] = run_cross_resolution(device, args.xres_shape)
        res["config"]["cross_resolution_wrong_region"] = run_cross_resolution(device, args.xres_shape,
                                                                              wrong_region=True)

    # float16 levels on the same frames (flow checked against the float32 result), and what a
    # learned warm start can buy at <= 0.1 voxel RMS (the sweep of warmstart.sweep)
    if args.precision == "f32" and not args.no_mixed:
        res["config"]["mixed_precision_f16"] = run_mixed_f16(args, wl, template, excl, frames, params, device, world,
                                                             res["value"])
    weights = os.path.join(ROOT, "wholistic_registration_b200", "weights", "warmstart.npz")
    if not args.no_warmstart and world == 1 and os.path.exists(weights):
        res["config"]["warm_start"] = run_warmstart_sweep(device, weights)

    # e2e through the host-memory series API
    if not args.no_e2e:
        n_host = min(4, n_frames)
        host_frames = [frames[i].cpu().pin_memory() for i in range(n_host)]
        host_motion = [torch.empty(wl["shape"] + (3,), dtype=torch.float32).pin_memory() for _ in range(2)]
        host_warp = [torch.empty(wl["shape"], dtype=torch.float32).pin_memory() for _ in range(2)]
        series = SeriesRegistrar(template, params, mask_ref=excl, mask_mov=excl)
        series.reg.tune_flags = reg.tune_flags
        ek = max(4, args.steps)   # one pass of the pipeline: fill and drain amortised over the timed steps
        seq = [host_frames[i % n_host] for i in range(ek)]
        outs_m = [host_motion[i % 2] for i in range(ek)]
        outs_w = [host_warp[i % 2] for i in range(ek)]
        series.run(seq[:2], outs_m[:2], outs_w[:2])
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(series.s_in)
        series.s_in.wait_stream(torch.cuda.current_stream())
        series.run(seq, outs_m, outs_w)
        t1.record(series.s_out)
        torch.cuda.synchronize()
        e_ms = t0.elapsed_time(t1)
        if world > 1:
            t = torch.tensor([e_ms], dtype=torch.float64, device=device)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e_ms = float(t.item())
        h2d, d2h = series.bytes_per_frame()
        res["e2e"] = {"value": round(world * ek / (e_ms * 1e-3), 3), "unit": "volumes/s", "h2d_bytes_per_step": h2d,
                      "d2h_bytes_per_step": d2h, "steps": ek,
                      "api": "SeriesRegistrar.run (pinned host frames -> host motion + warped volume)"}
        res["gpu_launches_e2e_per_step"] = launches_per_step
    return res, [updates_sum[l] / args.steps for l in range(levels)]


def run_batched_small(device, n=16, reps=3):
    """Frames small enough to leave most of the GPU idle one by one (the
    64x256x256 configuration, layer 2, r 16): registration + warp of n frames
    one call each, and as one batched call replayed from a CUDA graph."""
    import torch

    from wholistic_registration_b200 import LKParams, LKRegistrar, penalty_factor, synthetic
    from wholistic_registration_b200.batch import BatchRegistrar

    shape = (64, 256, 256)
    tmpl, _, _ = synthetic.make_pair(shape, 4242, n_blobs=2000, max_disp=(4.0, 4.0, 1.5), device=device)
    movs = [synthetic.make_pair(shape, 4300 + k, n_blobs=2000, max_disp=(4.0, 4.0, 1.5), device=device,
                                template=tmpl.float())[1].contiguous() for k in range(n)]
    tmpl = tmpl.contiguous()
    excl = (~synthetic.ellipsoid_inclusion(shape, 0.7, device=device)).to(torch.uint8)
    factor = float(penalty_factor(tmpl.float().contiguous()))
    p = LKParams(layer=2, iter=10, r=16, zRatio=1.0, movRange=5.0, smoothPenalty=0.08 * factor, tol=1e-3)
    reg = LKRegistrar(shape, p, device)
    motion = torch.empty(shape + (3,), dtype=torch.float32, device=device)
    warped = torch.empty(shape, dtype=torch.float32, device=device)

    def one_by_one():
        for k in range(n):
            reg.register(movs[k], tmpl, excl, excl, out=motion, warped_out=warped, reuse_reference=True)

    br = BatchRegistrar([shape] * n, p, device, warp=True, graph=True)
    tm, ex = [tmpl] * n, [excl] * n
    br.register(movs, tm, ex, ex)

    def batched():
        br.register(movs, tm, ex, ex, reuse_reference=True)

    out = {"frames": n, "shape_zyx": list(shape), "layer": 2, "r": 16}
    reg.register(movs[0], tmpl, excl, excl, out=motion, warped_out=warped)
    for name, fn in (("one_call_per_frame", one_by_one), ("batched_cuda_graph", batched)):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        out[name + "_volumes_per_s"] = round(n * reps / (e0.elapsed_time(e1) * 1e-3), 2)
    out["speedup"] = round(out["batched_cuda_graph_volumes_per_s"] / out["one_call_per_frame_volumes_per_s"], 3)
    return out


def run_uneven_batch(device, reps=3, seed=777):
    """Uneven batch: 48 volume pairs, 16 each at 32x256x256, 64x512x512 and
    96x768x1024 (config-0 blob density and sinusoid fields), each with its
    own random ellipsoid exclusion mask (40-90 % coverage) and patch radius
    r in 4..16 (patches 9x9 .. 33x33), as many levels (up to 4) as the radius
    leaves a CP on the coarsest, 10 iterations.  Timed: registering each
    volume with its own parameters one call after another (registrars built
    beforehand, one per shape and radius) against one per-frame-parameter
    batched call (wr_lk_register_batch_each) replayed from a CUDA graph."""
    import numpy as np
    import torch

    from wholistic_registration_b200 import LKParams, LKRegistrar, penalty_factor, synthetic
    from wholistic_registration_b200.batch import BatchRegistrar

    rng = np.random.default_rng(seed)
    shapes = [(32, 256, 256)] * 16 + [(64, 512, 512)] * 16 + [(96, 768, 1024)] * 16
    radii = [4, 6, 8, 10, 12, 14, 16]
    movs, refs, masks, plist = [], [], [], []
    for k, shape in enumerate(shapes):
        nb = max(200, int(2000 * np.prod(shape) / (64 * 256 * 256)))
        tmpl, mov, _ = synthetic.make_pair(shape, seed + k, n_blobs=nb, max_disp=(4.0, 4.0, 1.5), device=device)
        cov = float(rng.uniform(0.4, 0.9))
        excl = (~synthetic.ellipsoid_inclusion(shape, cov, device=device)).to(torch.uint8).contiguous()
        r = int(radii[k % len(radii)])
        layer = 0
        while layer < 3 and min(shape[1], shape[2]) // 2 ** (layer + 1) >= 2 * r + 1:
            layer += 1
        factor = float(penalty_factor(tmpl.float().contiguous(), excl))
        plist.append(LKParams(layer=layer, iter=10, r=r, zRatio=1.0, movRange=5.0, smoothPenalty=0.08 * factor,
                              tol=1e-3))
        movs.append(mov.contiguous())
        refs.append(tmpl.contiguous())
        masks.append(excl)
        del tmpl, mov
    torch.cuda.synchronize()
    regs = {}
    for shape, p in zip(shapes, plist):
        key = (shape, p.r, p.layer)
        if key not in regs:
            regs[key] = (LKRegistrar(shape, p, device), torch.empty(shape + (3,), dtype=torch.float32, device=device))

    def one_by_one():
        for k, (shape, p) in enumerate(zip(shapes, plist)):
            reg, out = regs[(shape, p.r, p.layer)]
            reg.set_params(p)
            reg.register(movs[k], refs[k], masks[k], masks[k], out=out)

    br = BatchRegistrar(shapes, plist, device, graph=True)
    br.register(movs, refs, masks, masks)

    def batched():
        br.register(movs, refs, masks, masks)

    nvox = float(sum(np.prod(s) for s in shapes))
    out = {"volumes": len(shapes), "shapes_zyx": [[32, 256, 256], [64, 512, 512], [96, 768, 1024]],
           "radii": sorted({p.r for p in plist}), "layers": sorted({p.layer for p in plist}),
           "mask_coverage": "uniform 0.4-0.9 per volume"}
    for name, fn in (("one_call_per_volume", one_by_one), ("batched_cuda_graph", batched)):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        sec = e0.elapsed_time(e1) * 1e-3 / reps
        out[name + "_volumes_per_s"] = round(len(shapes) / sec, 2)
        out[name + "_gvox_per_s"] = round(nvox / sec * 1e-9, 3)
    out["speedup"] = round(out["batched_cuda_graph_volumes_per_s"] / out["one_call_per_volume_volumes_per_s"], 3)
    del br, regs, movs, refs, masks
    torch.cuda.empty_cache()
    return out


def run_cross_resolution(device, shape="32x1024x1024:128", reps=4, wrong_region=False):
    """getMotion_v2: by default a 32x1024x1024 moving stack (z spacing 4)
    onto a 128x1024x1024 reference (z spacing 1), layer 3, r 16, iter 10, its
    own stopping rules; the moving stack is every (nzh / nz)-th reference
    slice shifted by one voxel in x and y.  wrong_region: with the
    wrong-region correction at the reference's default options."""
    import torch

    from wholistic_registration_b200 import synthetic
    from wholistic_registration_b200.calFlowCrossResolution import XresRegistrar
    from wholistic_registration_b200 import _lib
    from wholistic_registration_b200.registrar import LKParams

    zyx, nzh = shape.split(":")
    nz, ny, nx = (int(v) for v in zyx.split("x"))
    nzh = int(nzh)
    if nzh % nz:
        raise ValueError("--xres-shape: the reference's z extent must be a multiple of the moving stack's")
    tmpl, _, _ = synthetic.make_pair((nzh, ny, nx), 77, n_blobs=max(200, 20000 * nzh * ny * nx // (128 << 20)),
                                     device=device)
    ref = tmpl.float().contiguous()
    mov = torch.roll(ref[::nzh // nz], shifts=(1, -1), dims=(1, 2)).contiguous()
    excl = torch.zeros((nz, ny, nx), dtype=torch.uint8, device=device)
    p = LKParams(layer=3, iter=10, r=16, zRatio=float(nzh // nz), movRange=5.0, smoothPenalty=0.05, tol=1e-3)
    wr = _lib.WrXresWrongRegion(1, 0, 3.0, 2, 2.0, 1.0, 2.0, 0, 0.8) if wrong_region else None
    reg = XresRegistrar((nz, ny, nx), (nzh, ny, nx), p, 1.0, has_mask_ref=False, device=device, wrong_region=wr)
    reg.register(mov, ref, mask_mov=excl)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        reg.register(mov, ref, mask_mov=excl)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    log, _ = reg.error_log()
    return {"shape_mov_zyx": [nz, ny, nx], "shape_ref_zyx": [nzh, ny, nx], "zRatio": float(nzh // nz), "zRatio_HR": 1.0,
            "layer": 3, "r": 16, "iter": 10, "ms_per_volume": round(ms, 3), "volumes_per_s": round(1e3 / ms, 3),
            "updates_per_level": {k: len(v["max_diff_motion"]) for k, v in log.items()},
            "wrong_region_correction": "on (reference defaults, direct mode)" if wrong_region else "off",
            "api": "XresRegistrar.register (device-resident stacks)"}


def run_mixed_f16(args, wl, template, excl, frames, params, device, world, f32_value):
    """The plain path with its levels stored in float16 (interpolated in half2),
    timed like `value` on the same frames, and its flow RMS / max against the
    float32 path on the first frame."""
    import torch
    import torch.distributed as dist

    from wholistic_registration_b200 import LKParams, LKRegistrar

    p16 = LKParams(layer=params.layer, iter=params.iter, r=params.r, zRatio=params.zRatio, movRange=params.movRange,
                   smoothPenalty=params.smoothPenalty, tol=params.tol, precision=1)
    p32 = LKParams(layer=params.layer, iter=params.iter, r=params.r, zRatio=params.zRatio, movRange=params.movRange,
                   smoothPenalty=params.smoothPenalty, tol=params.tol)
    m32 = LKRegistrar(wl["shape"], p32, device).register(frames[0], template, excl, excl).clone()
    reg = LKRegistrar(wl["shape"], p16, device)
    m16 = reg.register(frames[0], template, excl, excl).clone()
    d = (m16 - m32).float()
    rms, mx = float(d.square().mean().sqrt()), float(d.abs().max())
    del m32, m16, d
    motion = torch.empty(wl["shape"] + (3,), dtype=torch.float32, device=device)
    warped = torch.empty(wl["shape"], dtype=torch.float32, device=device)
    steps = max(4, min(args.steps, 16))
    for k in range(args.warmup):
        reg.register(frames[k % len(frames)], template, excl, excl, out=motion, warped_out=warped,
                     reuse_reference=True)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for k in range(steps):
        reg.register(frames[k % len(frames)], template, excl, excl, out=motion, warped_out=warped,
                     reuse_reference=True)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    if world > 1:
        t = torch.tensor([ms], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    v = world * steps / (ms * 1e-3)
    return {"value": round(v, 3), "ms_per_step": round(ms / steps, 4), "steps": steps,
            "speedup_vs_f32": round(v / f32_value, 3), "flow_rms_vs_f32": round(rms, 6), "flow_max_vs_f32": round(mx, 5),
            "storage": "levels and gradients float16 (half of each value), sums and solves float32, "
                       "float64 re-solve above condition 1e6"}


def run_warmstart_sweep(device, weights):
    """warmstart.sweep on three config-1 frames: flow RMS from the plain
    pyramid and time per frame of short refinements from the zero field, the
    network, the true deformation and the plain result; the fastest
    configuration within 0.1 voxel RMS that starts from the zero field or the
    network, and its speed-up over plain."""
    from wholistic_registration_b200.warmstart import WarmStartNet, sweep

    net = WarmStartNet(device)
    meta = net.load(weights)
    rows, plain_ms = sweep((128, 1024, 1024), 3, net=net, device=device)
    # usable starts only: the true deformation and the plain result are diagnostics (upper bounds)
    ok = [r for r in rows if r["rms"] <= 0.1 and r["start"] in ("zero", "network")]
    best = min(ok, key=lambda r: r["ms_per_frame"]) if ok else None
    out = {"plain_ms_per_frame": round(plain_ms, 3), "network_parameters": net.parameter_count(),
           "trained_pairs": int(meta.get("steps", 0)),
           "rows": [{k: (round(v, 4) if isinstance(v, float) else v) for k, v in r.items()} for r in rows]}
    if best:
        out["fastest_within_0.1_vox_rms"] = dict(best, speedup_vs_plain=round(plain_ms / best["ms_per_frame"], 3))
    return out

def cpu_baseline_obj(pool, cores, wl, updates):
    sec_per_vi, times = cpu_rate(pool, cores)
    vi = voxel_iters_per_volume(wl, updates)
    vps = cores / (sec_per_vi * vi)
    return {
        "value": vps, "unit": "volumes/s", "cores": cores, "kind": "port",
        "sample": (f"oracle port with the reference's scipy correlate box sums: one LK iteration (r=16) on a "
                   f"{CPU_SLAB[0]}x{CPU_SLAB[1]}x{CPU_SLAB[2]} slab per core, {len(times)} cores in parallel, "
                   f"median {statistics.median(times):.2f} s; extrapolated to {vi:.3g} voxel-iterations per volume "
                   f"(updates per level {['%.2f' % u for u in (updates or [wl['iter'] - 1] * (wl['layer'] + 1))]})"),
        "seconds_per_volume_per_core": sec_per_vi * vi,
    }


def run_reference(args, wl, rank):
    if rank != 0:
        return None
    cores = cpu_cores()
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores) as pool:
        pool.map(_cpu_sample, [0] * min(cores, 2)) if args.warmup > 0 else None
        vals = []
        t_all = time.perf_counter()
        for k in range(args.steps):
            t = time.perf_counter()
            pool.map(_cpu_sample, [k * cores + i for i in range(cores)])
            vals.append(time.perf_counter() - t)
        wall = time.perf_counter() - t_all
    n = CPU_SLAB[0] * CPU_SLAB[1] * CPU_SLAB[2]
    vi = voxel_iters_per_volume(wl, None)
    step_s = statistics.median(vals)
    vps = cores * n / step_s / vi
    return {
        "metric": METRIC, "value": vps, "unit": "volumes/s", "n_gpus": 0, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": step_s * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic", "impl": "reference",
        "config": {"workload": args.workload, "shape_zyx": list(wl["shape"]), "layer": wl["layer"], "r": wl["r"],
                   "iter": wl["iter"], "path": "CPU oracle port, reference correlate cost"},
        "cpu_baseline": {"value": vps, "unit": "volumes/s", "cores": cores, "kind": "port",
                         "sample": (f"each step: one LK iteration (r=16) on a {CPU_SLAB[0]}x{CPU_SLAB[1]}x{CPU_SLAB[2]} "
                                    f"slab on each of {cores} cores; extrapolated to {vi:.3g} voxel-iterations "
                                    f"per volume (every level at the iteration cap)")},
        "e2e": {"value": vps, "unit": "volumes/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "wall_s": wall,
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=32)
    ap.add_argument("--warmup", type=int, default=4)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="series-128x1024x1024")
    ap.add_argument("--frames", type=int, default=32)
    ap.add_argument("--precision", choices=["f32", "f16", "bf16"], default="f32")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-warmstart", action="store_true")
    ap.add_argument("--no-mixed", action="store_true", help="skip the float16-level measurement")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-xres", action="store_true", help="skip the cross-resolution (getMotion_v2) measurement")
    ap.add_argument("--xres-shape", default="32x1024x1024:128",
                    help="moving stack ZxYxX and reference z extent of the cross-resolution measurement")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    wl = WORKLOADS[args.workload]
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        res = run_reference(args, wl, rank)
        if res is not None:
            print(json.dumps(res), flush=True)
        return

    pool = None
    cores = cpu_cores()
    if rank == 0 and world == 1 and not args.no_cpu:
        pool = mp.get_context("spawn").Pool(cores)

    import torch
    import torch.distributed as dist

    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local_rank))
    res, updates = run_ours(args, wl, rank, world, local_rank)
    if pool is not None:
        res["cpu_baseline"] = cpu_baseline_obj(pool, cores, wl, updates)
        pool.close()
        pool.join()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
