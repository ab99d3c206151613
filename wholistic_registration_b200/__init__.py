"""B200-native pyramid patch-wise Lucas-Kanade 3-D registration.

A drop-in for the registration path of the reference package
``wholistic_registration``: ``getMotion`` / ``correctMotion``
(``calFlow3d_Wei_v1``) keep the reference's signatures; ``LKRegistrar`` is the
device-level API on (z, y, x) CUDA tensors.  All compute runs in the sm_100a
library ``_wr_b200.so`` (C ABI in ``include/wr_b200.h``).
"""

from . import _lib
from .registrar import LKParams, LKRegistrar, penalty_factor, warp

__all__ = ["LKParams", "LKRegistrar", "warp", "penalty_factor", "getMotion", "correctMotion"]


def __getattr__(name):
    if name in ("getMotion", "correctMotion"):
        from . import calFlow3d_Wei_v1

        return getattr(calFlow3d_Wei_v1, name)
    raise AttributeError(name)
