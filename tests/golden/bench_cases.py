"""Registration cases at the benchmarked configuration (r = 16, 33 x 33 patches).

Shared by the fixture generator (``make_golden.py --only bench``), which runs
the reference's ``getMotion`` / ``correctMotion`` on them, and by the tests,
which regenerate the same inputs from the seeded generator and check their
SHA-256 against the fixture before comparing.  Only a strided subsample of
the reference's motion and warped volume is committed (``bench_<name>.npz``).

Arrays are in the reference's internal (x, y, z) layout.
"""

from __future__ import annotations

import hashlib

import numpy as np

from wholistic_registration_b200 import synthetic

# name: (z, y, x), seed, blobs, max_disp (x, y, z), layer, mask coverage (None = no exclusion), stride
BENCH_CASES = {
    # config-0 generator (2000 blobs per 64x256x256), an 8-slice slab, 70 % ellipsoid mask
    "c0slab_8x256x256_l2": ((8, 256, 256), 9001, 250, (4.0, 4.0, 1.5), 2, 0.70, 3),
    # config-1 density (20k blobs per 128x1024x1024); level 3 is 64x64: one CP window plus an overhang
    "c1slab_4x512x512_l3": ((4, 512, 512), 9002, 160, (8.0, 8.0, 3.0), 3, 0.70, 5),
    # config 0 itself: 64x256x256, 2000 blobs, max 4/4/1.5, no exclusion, 3 levels
    "c0full_64x256x256_l2": ((64, 256, 256), 9003, 2000, (4.0, 4.0, 1.5), 2, None, 5),
    # a config-1 slab: 8x1024x1024 at config-1 density, max 8/8/3, 70 % ellipsoid, 4 levels
    "c1slab_8x1024x1024_l3": ((8, 1024, 1024), 9004, 1250, (8.0, 8.0, 3.0), 3, 0.70, 9),
}
BENCH_R = 16
BENCH_ITER = 10
BENCH_RAW_PENALTY = 0.08


def bench_inputs(name):
    """(template, moving, exclusion, sha256): uint16 volumes and the boolean
    exclusion mask in (x, y, z) layout, and the SHA-256 of template + moving bytes."""
    import torch

    zyx, seed, nb, md, _, cov, _ = BENCH_CASES[name]
    tmpl, mov, _ = synthetic.make_pair(zyx, seed, n_blobs=nb, max_disp=md)
    t = np.ascontiguousarray(tmpl.to(torch.int32).numpy().astype(np.uint16).transpose(2, 1, 0))
    m = np.ascontiguousarray(mov.to(torch.int32).numpy().astype(np.uint16).transpose(2, 1, 0))
    if cov is None:
        excl = np.zeros(t.shape, bool)
    else:
        excl = np.ascontiguousarray(~synthetic.ellipsoid_inclusion(zyx, cov).numpy().transpose(2, 1, 0))
    return t, m, excl, hashlib.sha256(t.tobytes() + m.tobytes()).hexdigest()


def bench_option(name, smooth_penalty):
    """The reference's option dict for a case (masks as exclusion, both sides)."""
    _, _, _, _, layer, _, _ = BENCH_CASES[name]
    return {"layer": layer, "iter": BENCH_ITER, "r": BENCH_R, "zRatio": 1.0, "movRange": 5.0, "motion": None,
            "smoothPenalty": float(smooth_penalty), "tol": 1e-3, "save_ite": 100}
