"""The iteration kernel's gradient rule near the volume faces, checked on the
CPU against the oracle's restatement of the reference's clipped central
difference (utils/calFlow3d_Wei_v1.py:134-206).

The kernel samples the stored half differences G (central inside, one-sided
on the faces) at c and, along an axis where c lies outside [0, n - 1],
multiplies by min(c + 1, n - c) clamped to [0, 1].  This test states that
rule in float64 and compares it with the oracle for coordinates inside,
between and beyond the faces, for extents 1, 2 and larger.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import lk_oracle


def half_differences(vol):
    """(Gx, Gy, Gz): half the edge-clamped central difference along each axis."""
    out = []
    for k in range(3):
        n = vol.shape[k]
        up = np.take(vol, np.minimum(np.arange(n) + 1, n - 1), axis=k)
        dn = np.take(vol, np.maximum(np.arange(n) - 1, 0), axis=k)
        out.append(0.5 * (up - dn))
    return out


@pytest.mark.parametrize("shape", [(9, 7, 6), (2, 5, 3), (1, 4, 4), (6, 1, 2)])
def test_face_rule_matches_clipped_difference(shape):
    rng = np.random.default_rng(sum(shape))
    vol = rng.normal(100.0, 20.0, size=shape)
    G = half_differences(vol)
    m = 4000
    # multiples of 1/64 keep c +- 1 exact in float32, as the rule assumes
    coords = np.stack([np.round(rng.uniform(-2.5, n + 1.5, size=m) * 64.0) / 64.0 for n in shape], axis=-1)
    coords = coords.astype(np.float32)
    want = lk_oracle.spatial_gradient(vol, coords)
    c = [coords[:, k].astype(np.float64) for k in range(3)]
    for k in range(3):
        n = shape[k]
        got = lk_oracle.trilinear(G[k], *c)
        scale = np.where((c[k] >= 0) & (c[k] <= n - 1), 1.0, np.clip(np.minimum(c[k] + 1.0, n - c[k]), 0.0, 1.0))
        np.testing.assert_allclose(got * scale, want[k], rtol=0, atol=1e-9 * np.abs(vol).max())
