"""hit3d_b200 -- B200-native pseudospectral timestep of HIT3DP.

The product is the C-ABI library ``libhit3d_gpu.so`` (include/hit3d_gpu.h) built
from ``csrc/`` for sm_100a.  This package binds it (``gpu``), parses the
reference's input file (``params``) and restates the reference's host main loop
over the C-ABI (``driver``).
"""
from .gpu import Context, Hit3dError, Mlp, Params, lib  # noqa: F401

__all__ = ["Context", "Hit3dError", "Mlp", "Params", "lib"]
