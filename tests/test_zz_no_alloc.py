"""The allocation-free penalty-factor entry point.

Some callers cannot call cudaMalloc: a host application that owns all device
memory through its own pool, or an acquisition loop that must not enter the
allocator between frames.  ``wr_penalty_factor_noalloc`` serves them by
keeping its partial sums in a static device array.  This file is collected
last so that a failure here leaves every other test already run.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _call_both(lib, _lib, ref, mask):
    vol = _lib.volume(ref.data_ptr(), _lib.WR_F32 if ref.dtype == torch.float32 else _lib.WR_U16, ref.shape)
    mptr = None if mask is None else mask.data_ptr()
    out_a = torch.full((), float("nan"), dtype=torch.float64, device=ref.device)
    out_b = torch.full((), float("nan"), dtype=torch.float64, device=ref.device)
    nbytes = ctypes.c_size_t(0)
    _lib.check("scratch", lib.wr_penalty_factor_scratch(*ref.shape, ctypes.byref(nbytes)))
    scratch = torch.empty(int(nbytes.value), dtype=torch.uint8, device=ref.device)
    stream = torch.cuda.current_stream().cuda_stream
    _lib.check("wr_penalty_factor", lib.wr_penalty_factor(ctypes.byref(vol), mptr, out_a.data_ptr(),
                                                         scratch.data_ptr(), int(nbytes.value), stream))
    _lib.check("wr_penalty_factor_noalloc", lib.wr_penalty_factor_noalloc(ctypes.byref(vol), mptr,
                                                                         out_b.data_ptr(), stream))
    torch.cuda.synchronize()
    return float(out_a), float(out_b)


def test_no_alloc_penalty_factor_matches_allocating_entry_point():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from wholistic_registration_b200 import _lib

    lib = _lib.load()
    gen = torch.Generator(device="cuda")
    gen.manual_seed(5)
    # two calls in a row on different volumes: the second must not see the first's partials
    first = torch.rand((24, 160, 200), generator=gen, device="cuda") * 1000
    mask = (torch.rand((24, 160, 200), generator=gen, device="cuda") > 0.8).to(torch.uint8)
    second = (torch.rand((9, 64, 80), generator=gen, device="cuda") * 60000).to(torch.int32).to(torch.uint16)
    for ref, m in ((first, mask), (second, None)):
        a, b = _call_both(lib, _lib, ref, m)
        assert np.isfinite(a) and a > 0
        np.testing.assert_allclose(b, a, rtol=1e-12)


@pytest.mark.parametrize("shape", [(20, 1024, 1024), (128, 1024, 1024)])
def test_no_alloc_penalty_factor_large_volumes(shape):
    """Volumes whose partial sums fill more than 1024 slots of the static
    array (20 x 1024 x 1024: 1280 slots) and exactly all of it
    (128 x 1024 x 1024 = 134,217,728 voxels: 8192 slots), against the
    allocating entry point, two calls in a row."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from wholistic_registration_b200 import _lib

    lib = _lib.load()
    gen = torch.Generator(device="cuda")
    gen.manual_seed(11)
    ref = (torch.rand(shape, generator=gen, device="cuda") * 60000).to(torch.int32).to(torch.uint16)
    mask = (torch.rand(shape, generator=gen, device="cuda") > 0.7).to(torch.uint8)
    for m in (mask, None):
        a, b = _call_both(lib, _lib, ref, m)
        assert np.isfinite(a) and a > 0
        np.testing.assert_allclose(b, a, rtol=1e-12)
    del ref, mask
    torch.cuda.empty_cache()


def test_no_alloc_rejects_volumes_beyond_its_scratch():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from wholistic_registration_b200 import _lib

    lib = _lib.load()
    vol = _lib.volume(256, _lib.WR_U16, (129, 1024, 1024))
    out = torch.zeros((), dtype=torch.float64, device="cuda")
    rc = lib.wr_penalty_factor_noalloc(ctypes.byref(vol), None, out.data_ptr(), None)
    assert rc == 2
    assert b"134217728" in lib.wr_last_error()
