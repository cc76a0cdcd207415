"""B200-native rigorous EUV mask-3D simulation (drop-in for the abbe/m3d path
of takahashi-edalab/EUVlitho).

The compute runs in ``libeuvl_b200.so`` (hand-written sm_100a CUDA behind the
C ABI of ``include/euvl_b200.h``); this package is the host side.
"""
from .config import SimConfig, Stack, preset  # noqa: F401

__all__ = ["SimConfig", "Stack", "preset", "Plan"]


def __getattr__(name):
    if name == "Plan":
        from .engine import Plan
        return Plan
    raise AttributeError(name)
