"""The pyramid's alternative kernel paths.

The level builder picks between kernels by row length and alignment: rows of
at most 1024 voxels with aligned inputs take the staged x pass
(``k_resample_x_pp``), the vector y pass, the vectorised mask x pass and the
four-voxels-per-lane packing and mask-class kernels; longer rows or inputs
that are not 16-byte aligned take the general kernels.  Every pair computes
the same sums in the same order, so:

* a registration of the same data from unaligned buffers (views one element
  into a larger allocation) gives the same motion and warped volume bit for
  bit as from aligned ones;
* the level images of volumes with rows longer and shorter than 1024 both
  match the oracle's imresize (utils/imresize.py:148-191) to float32 rounding.
"""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _need():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _offset_copy(t):
    """A contiguous copy of ``t`` whose data starts one element into its
    allocation (not 16-byte aligned)."""
    flat = torch.empty(t.numel() + 1, dtype=t.dtype, device=t.device)
    v = flat[1:].view(t.shape)
    v.copy_(t)
    assert v.data_ptr() % 16 != 0
    return v


@pytest.mark.parametrize("shape,layer,r", [((8, 128, 256), 2, 4), ((6, 96, 1040), 2, 3)])
def test_unaligned_inputs_give_identical_results(shape, layer, r):
    _need()
    from wholistic_registration_b200 import synthetic
    from wholistic_registration_b200.registrar import LKParams, LKRegistrar

    dev = torch.device("cuda")
    tmpl, mov, _ = synthetic.make_pair(shape, 5, n_blobs=400, max_disp=(3.0, 3.0, 1.0), device=dev)
    excl = (~synthetic.ellipsoid_inclusion(shape, 0.7, device=dev)).to(torch.uint8).contiguous()
    p = LKParams(layer=layer, iter=4, r=r, zRatio=1.0, movRange=5.0, smoothPenalty=50.0, tol=1e-3)
    reg = LKRegistrar(shape, p, dev)
    outs = []
    for conv in (lambda t: t.contiguous(), _offset_copy):
        m, t, e = conv(mov), conv(tmpl), conv(excl)
        warped = torch.empty(shape, dtype=torch.float32, device=dev)
        motion = reg.register(m, t, e, e, None, warped_out=warped)
        torch.cuda.synchronize()
        outs.append((motion.clone(), warped.clone()))
    assert torch.equal(outs[0][0], outs[1][0])
    assert torch.equal(outs[0][1], outs[1][1])


@pytest.mark.parametrize("shape_xyz", [(1040, 24, 3), (1000, 24, 3), (256, 40, 4)])
def test_level_images_match_oracle_imresize(shape_xyz):
    _need()
    from oracle import lk_oracle as O
    from wholistic_registration_b200 import calFlow3d_Wei_v1 as cf3

    rng = np.random.default_rng(7)
    ref = rng.integers(0, 4000, size=shape_xyz).astype(np.uint16)
    mov = rng.integers(0, 4000, size=shape_xyz).astype(np.uint16)
    option = {"layer": 2, "iter": 1, "r": 2, "zRatio": 1.0, "movRange": 5.0, "motion": None,
              "smoothPenalty": 0.0, "tol": 1e-3, "save_ite": 1, "keep_snapshots": True}
    _, _, _, log = cf3.getMotion(mov, ref, option)
    for layer in (1, 2):
        shape = (int(shape_xyz[0] / 2 ** layer), int(shape_xyz[1] / 2 ** layer), shape_xyz[2])
        for key, vol in (("data_ref", ref), ("data_mov", mov)):
            got = np.asarray(log[f"layer_{layer}"][key], np.float64)
            want = O.imresize(vol, shape)
            assert got.shape == want.shape
            # float32 sums with float32 weights against the float64 resize
            err = np.abs(got - want).max() / np.abs(want).max()
            assert err <= 2e-6, (layer, key, err)
