"""Shared pytest configuration.

Tests marked ``gpu`` need a CUDA device and the built library; everything else
runs on CPU (``pytest -m "not gpu"``).
"""

from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU and the built sm_100a library")


@pytest.fixture
def rng() -> np.random.Generator:
    return np.random.default_rng(seed=42)


def load_motion_case(name):
    """(arrays, meta) for a golden getMotion case."""
    import json

    with open(os.path.join(GOLDEN, "motion_cases.json")) as fh:
        meta = json.load(fh)[name]
    arrays = dict(np.load(os.path.join(GOLDEN, f"motion_{name}.npz")))
    return arrays, meta


def motion_case_names():
    import json

    with open(os.path.join(GOLDEN, "motion_cases.json")) as fh:
        return sorted(json.load(fh))


def option_from_case(arrays, meta):
    return {
        "mask_ref": arrays["mask_ref"].copy(),
        "mask_mov": arrays["mask_mov"].copy(),
        "layer": meta["layer"],
        "iter": meta["iter"],
        "r": meta["r"],
        "zRatio": meta["zRatio"],
        "movRange": meta["movRange"],
        "motion": arrays.get("motion_init"),
        "smoothPenalty": meta["smoothPenalty"],
        "tol": meta["tol"],
        "save_ite": 100,
    }


def updates_per_layer(arrays, meta):
    """Number of motion updates the reference performed at each layer."""
    return {l: len(arrays[f"layer_{l}/max_diff_motion"]) for l in range(meta["layer"] + 1)}


def xres_case_names():
    import json

    with open(os.path.join(GOLDEN, "xres_cases.json")) as fh:
        return sorted(json.load(fh))


def load_xres_case(name):
    """(arrays, option) for a golden getMotion_v2 case (wrong-region correction off)."""
    import json

    with open(os.path.join(GOLDEN, "xres_cases.json")) as fh:
        meta = json.load(fh)[name]
    arrays = dict(np.load(os.path.join(GOLDEN, f"xres_{name}.npz")))
    option = dict(meta)
    option.update({"mask_ref": arrays["mask_ref"].copy(), "mask_mov": arrays["mask_mov"].copy(),
                   "motion": arrays.get("motion_init"), "wrong_region_enable": False})
    if "phase_init" in arrays:
        option["phase"] = arrays["phase_init"]
    return arrays, option


def xres_wr_case_names():
    import glob

    return sorted(os.path.basename(f)[len("xreswr_"):-4] for f in glob.glob(os.path.join(GOLDEN, "xreswr_*.npz")))


def xres_hr_case_names():
    import glob

    return sorted(os.path.basename(f)[len("xreshr_"):-4] for f in glob.glob(os.path.join(GOLDEN, "xreshr_*.npz")))


def load_xres_hr_case(name):
    """(arrays, option) for a getMotion_v2 case with the wrong-region
    correction in its "highresidual" exclusion mode."""
    arrays, option = load_xres_case(name)
    out = dict(np.load(os.path.join(GOLDEN, f"xreshr_{name}.npz")))
    option.update({"wrong_region_enable": True, "wrong_region_exclude_mode": "highresidual",
                   "quantile_threshold_q": float(out.pop("quantile_q"))})
    arrays.update(out)
    return arrays, option


def xres_opt_case_names():
    import glob

    return sorted(os.path.basename(f)[len("xresopt_"):-4] for f in glob.glob(os.path.join(GOLDEN, "xresopt_*.npz")))


def load_xres_opt_case(name):
    """(arrays, option) for a getMotion_v2 case with the wrong-region
    correction at non-default options (stored with the fixture)."""
    import json

    arrays, option = load_xres_case(name)
    out = dict(np.load(os.path.join(GOLDEN, f"xresopt_{name}.npz")))
    option["wrong_region_enable"] = True
    option.update(json.loads(str(out.pop("options"))))
    arrays.update(out)
    return arrays, option


def load_xres_wr_case(name):
    """(arrays, option) for a getMotion_v2 case with the wrong-region correction
    on: the inputs of the xres case, the outputs of the reference's run with
    the correction."""
    arrays, option = load_xres_case(name)
    out = dict(np.load(os.path.join(GOLDEN, f"xreswr_{name}.npz")))
    arrays.update(out)
    option["wrong_region_enable"] = True
    return arrays, option


def projection_ref_cases():
    """(name, arrays) of the fixtures from the reference's own projection
    kernels (tests/golden/make_projection_golden.py)."""
    d = dict(np.load(os.path.join(GOLDEN, "projection_ref.npz")))
    names = sorted({k[: -len("_params")] for k in d if k.endswith("_params")})
    return [(n, {k[len(n) + 1:]: v for k, v in d.items() if k.startswith(n + "_")}) for n in names]
