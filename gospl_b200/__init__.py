"""gospl_b200: goSPL's per-timestep surface-process path on NVIDIA B200 (sm_100a).

Receivers, depression filling, flow accumulation with the lake cascade,
implicit stream-power erosion and hillslope diffusion run as hand-written CUDA
kernels in ``libgospl_b200.so`` behind a C ABI (``include/gospl_b200.h``);
``gospl_b200.Model`` drives them with the reference's method names.
"""
from . import _lib  # noqa: F401

__version__ = "0.1.0"


def Model(*args, **kwargs):
    from .model import Model as _M
    return _M(*args, **kwargs)
