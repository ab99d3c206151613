"""Autotuner for the launch shape of the fused iteration kernel.

Candidates are the tile visiting order of the persistent CTAs (z fastest, so
that concurrent CTAs share moving-volume planes in L2, or x fastest, so that
they share window halos) times the number of persistent CTAs per SM (as many
as fit, or fewer).  Each candidate registers a synthetic pair of the
requested shape with fixed per-level update counts, so every candidate does
the same work, and is timed with CUDA events; results never depend on the
choice.  The fastest is cached per (device, SM count, shape, parameters,
dtype, masks) in a JSON file (``$WR_B200_CACHE`` or
``~/.cache/wholistic_registration_b200/autotune.json``) and returned as
``WrLKParams.flags`` bits.
"""

from __future__ import annotations

import dataclasses
import json
import os
import threading

import torch

from . import _lib

ORDERS = (0, _lib.WR_LK_TILE_ORDER_X)
CTAS_PER_SM = (0, 3, 2)
_lock = threading.Lock()


def cache_path() -> str:
    base = os.environ.get("WR_B200_CACHE") or os.path.join(os.path.expanduser("~"), ".cache",
                                                            "wholistic_registration_b200")
    return os.path.join(base, "autotune.json")


def _key(shape, params, dtype, mask, device) -> str:
    prop = torch.cuda.get_device_properties(device)
    p = dataclasses.asdict(params)
    p.pop("forced_updates", None)
    p.pop("smoothPenalty", None)
    p.pop("tol", None)
    return json.dumps([prop.name, prop.multi_processor_count, list(shape), p, str(dtype), bool(mask)], sort_keys=True)


def _load() -> dict:
    try:
        with open(cache_path()) as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return {}


def _store(d: dict):
    path = cache_path()
    os.makedirs(os.path.dirname(path), exist_ok=True)
    tmp = path + f".{os.getpid()}.tmp"
    with open(tmp, "w") as fh:
        json.dump(d, fh, indent=1, sort_keys=True)
    os.replace(tmp, path)


def candidates():
    return [o | _lib.WR_LK_CTAS_PER_SM(c) for o in ORDERS for c in CTAS_PER_SM]


def tune(shape, params, dtype=torch.uint16, mask=True, device=None, use_cache=True, reps=3, report=None) -> int:
    """Flags of the fastest candidate for this shape and parameter set.

    ``report`` (a dict) receives the per-candidate milliseconds."""
    from . import synthetic
    from .registrar import LKRegistrar, penalty_factor

    device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    shape = tuple(int(v) for v in shape)
    key = _key(shape, params, dtype, mask, device)
    if use_cache:
        with _lock:
            hit = _load().get(key)
        if hit is not None:
            if report is not None:
                report.update(hit.get("ms", {}))
            return int(hit["flags"])
    tmpl, mov, _ = synthetic.make_pair(shape, 12345, n_blobs=max(200, shape[0] * shape[1] * shape[2] // 6700),
                                       max_disp=(4.0, 4.0, 1.5), device=device)
    if dtype == torch.float32:
        tmpl, mov = tmpl.float(), mov.float()
    elif dtype == torch.uint8:
        tmpl = (tmpl.float() / 256).clamp(0, 255).to(torch.uint8)
        mov = (mov.float() / 256).clamp(0, 255).to(torch.uint8)
    tmpl, mov = tmpl.contiguous(), mov.contiguous()
    excl = (~synthetic.ellipsoid_inclusion(shape, 0.7, device=device)).to(torch.uint8) if mask else None
    p = dataclasses.replace(params, forced_updates={l: min(3, params.iter - 1) for l in range(params.layer + 1)},
                            smoothPenalty=0.08 * float(penalty_factor(tmpl.float().contiguous())))
    reg = LKRegistrar(shape, p, device)
    motion = torch.empty(shape + (3,), dtype=torch.float32, device=device)
    times = {}
    for flags in candidates():
        reg.tune_flags = flags
        reg.register(mov, tmpl, excl, excl, out=motion)    # warm-up (and occupancy query)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            reg.register(mov, tmpl, excl, excl, out=motion, reuse_reference=True)
        e1.record()
        torch.cuda.synchronize()
        times[flags] = e0.elapsed_time(e1) / reps
    best = min(times, key=times.get)
    ms = {str(k): round(v, 4) for k, v in times.items()}
    if report is not None:
        report.update(ms)
    if use_cache:
        with _lock:
            d = _load()
            d[key] = {"flags": best, "ms": ms}
            _store(d)
    return best
