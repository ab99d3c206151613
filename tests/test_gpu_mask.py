"""Device outlier masks (getMask, bwareafilt3_wei) against the reference's
own utils/mask.py (fixtures) and the mask oracle: exact masks."""

from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import GOLDEN

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _need():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _dev(a):
    """(x, y, z) numpy -> (z, y, x) CUDA tensor"""
    return torch.from_numpy(np.ascontiguousarray(a.transpose(2, 1, 0))).cuda()


def _host(t):
    return t.cpu().numpy().transpose(2, 1, 0)


@pytest.mark.parametrize("name", ["mask_a", "mask_b", "mask_c"])
def test_masks_match_reference_fixture(name):
    _need()
    from wholistic_registration_b200.mask import bwareafilt3_wei, getMask

    d = np.load(os.path.join(GOLDEN, "masks.npz"))
    vol = d[f"{name}_vol"]
    thres, lo, hi = d[f"{name}_params"]
    stats = torch.zeros(3, dtype=torch.float64, device="cuda")
    m = getMask(_dev(vol), float(thres), stats=stats)
    np.testing.assert_array_equal(_host(m), d[f"{name}_mask"])
    mu, sg = d[f"{name}_musig"]
    np.testing.assert_allclose(stats[:2].cpu().numpy(), [mu, sg], rtol=2e-6)
    assert np.float32(stats[2].item()) == np.percentile(vol.astype(np.float32).ravel(), 95)
    f = bwareafilt3_wei(m, (int(lo), int(hi)))
    np.testing.assert_array_equal(_host(f), d[f"{name}_filtered"])


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_percentile_exact_for_float_data(seed):
    """Negative values, ties, and sizes whose float32 index is inexact."""
    _need()
    from wholistic_registration_b200.mask import getMask

    rng = np.random.default_rng(seed)
    shape = (7, 33, 29 + seed)
    v = (rng.standard_normal(shape) * 50).round(1).astype(np.float32)
    v[rng.random(shape) < 0.1] = 3.5
    stats = torch.zeros(3, dtype=torch.float64, device="cuda")
    getMask(torch.from_numpy(v).cuda(), 2.0, stats=stats)
    assert np.float32(stats[2].item()) == np.percentile(v.ravel(), 95)


def test_bwareafilt_edge_cases():
    _need()
    from oracle import mask_oracle as M
    from wholistic_registration_b200.mask import bwareafilt3_wei

    rng = np.random.default_rng(5)
    cases = [np.zeros((4, 9, 7), bool), np.ones((4, 9, 7), bool)]
    diag = np.zeros((5, 6, 6), bool)
    for k in range(5):
        diag[k, k, k] = True       # one component through corners only (26-connectivity)
    cases.append(diag)
    for p in (0.05, 0.2, 0.35):
        cases.append(rng.random((9, 40, 37)) < p)
    for c in cases:
        n = torch.zeros(1, dtype=torch.int32, device="cuda")
        for rng_ in ((1, 10 ** 9), (2, 30), (5, 5)):
            got = bwareafilt3_wei(torch.from_numpy(c).cuda(), rng_, n_components=n)
            want, kept = M.bwareafilt3(c.transpose(2, 1, 0), rng_)
            np.testing.assert_array_equal(_host(got), want)
            assert int(n.item()) == kept


def test_get_mask_against_oracle_random():
    _need()
    from oracle import mask_oracle as M
    from wholistic_registration_b200.mask import getMask

    rng = np.random.default_rng(9)
    for shape in ((6, 50, 44), (3, 17, 131)):
        v = rng.poisson(200, size=shape).astype(np.uint16)
        v[rng.random(shape) < 0.01] += 400
        m = getMask(torch.from_numpy(v).cuda(), 3.0)
        np.testing.assert_array_equal(_host(m), M.get_mask(v.transpose(2, 1, 0), 3.0))
