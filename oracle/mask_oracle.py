"""CPU oracle for the outlier masks of the per-batch registration wrapper.

TEST INFRASTRUCTURE ONLY.  Only ``tests/`` may import it; the product path
(``wholistic_registration_b200``) never calls into it.

It restates, in NumPy and ``scipy.ndimage`` (paths relative to the
reference's ``src/wholistic_registration``):

* ``utils/preprocess.py:69-84``  ``robust_mean_std``: mean / std of the values
  at or below the 95th percentile (numpy "linear" percentile), in float32
* ``utils/mask.py:59-111``       ``getMask``: |z| > thresFactor, then
  ``binary_opening`` and ``binary_dilation`` with a (3, 3, 1) footprint
* ``utils/mask.py:8-56``         ``bwareafilt3_wei``: 26-connected components
  whose voxel count lies in [min, max] (inclusive)

The reference calls scikit-image (``>= 0.21``, its ``pyproject.toml:21``),
which is not installed here; its functions are restated from their documented
semantics: ``binary_erosion`` treats the outside as set, ``binary_dilation``
as clear, ``binary_opening`` is the dilation of the erosion, and
``label(connectivity=3)`` is 26-connectivity.  Arrays follow the reference's
(x, y, z) layout.  ``tests/test_oracle_golden.py`` checks this module against
fixtures made by running the reference's own ``utils/mask.py`` with
scikit-image stand-ins (``tests/golden/make_golden.py``): the reference's
logic is pinned by those runs, scikit-image's by its documentation.
"""

from __future__ import annotations

import numpy as np
from scipy import ndimage

FOOTPRINT = np.ones((3, 3, 1), dtype=bool)


def robust_mean_std(data, percentile=95):
    flat = data.flatten()
    thr = np.percentile(flat, percentile)
    sel = flat[flat <= thr]
    return np.mean(sel), np.std(sel)


def get_mask(dat, thres_factor):
    d = dat.astype(np.float32)
    mu, sigma = robust_mean_std(d)
    m = np.abs((d - mu) / sigma) > thres_factor
    m = ndimage.binary_erosion(m, structure=FOOTPRINT, border_value=1)
    m = ndimage.binary_dilation(m, structure=FOOTPRINT, border_value=0)
    return ndimage.binary_dilation(m, structure=FOOTPRINT, border_value=0)


def bwareafilt3(vol, size_range):
    """(filtered mask, number of components kept)"""
    lab, n = ndimage.label(vol.astype(bool), structure=np.ones((3, 3, 3), bool))
    if n == 0:
        return np.zeros(vol.shape, bool), 0
    sizes = np.bincount(lab.ravel())
    keep = (sizes >= size_range[0]) & (sizes <= size_range[1])
    keep[0] = False
    return keep[lab], int(keep.sum())
