"""cmfb200: B200-native (sm_100a) CaMa-Flood per-sub-step river routing.

The model object `CaMaFlood` keeps the reference model/module API (tensor
names, `set_inputs`, `step_advance`); all compute runs in libcmfb200.so
(hand-written CUDA kernels behind a C ABI, include/cmfb200.h).
"""
from .model import CaMaFlood, InputProxy, Module  # noqa: F401
from .prefetch import InputPrefetcher  # noqa: F401
from . import synthetic, topology  # noqa: F401

__all__ = ["CaMaFlood", "InputProxy", "InputPrefetcher", "Module", "synthetic", "topology"]
