"""Shared helpers for the tests: seeded masks and config conversion."""
from __future__ import annotations

import dataclasses

import numpy as np

from euvlitho_b200.config import SimConfig
from oracle import euv_oracle as O


def to_oracle(cfg: SimConfig) -> O.SimConfig:
    """Same configuration for the oracle (independent dataclasses, same fields)."""
    d = dataclasses.asdict(cfg)
    st = O.Stack(**d.pop("stack"))
    z = d.pop("z")
    d["eabs"] = tuple(d["eabs"])
    d["dabs"] = tuple(d["dabs"])
    return O.SimConfig(stack=st, zlist=(z,), **d)


def random_mask(ndivx: int, ndivy: int, seed: int, frac: float = 0.36) -> np.ndarray:
    """Seeded lines-and-contacts layout, 0/1 [ndivy][ndivx] (1 = vacuum)."""
    from euvlitho_b200.masks import synth_mask
    return synth_mask(ndivx, ndivy, seed, frac)


def packed(mask2d: np.ndarray) -> np.ndarray:
    return np.packbits(mask2d.reshape(-1), bitorder="big")


def flat_bits(mask2d: np.ndarray) -> np.ndarray:
    """Oracle mask2d layout (int32 [ndivx*j + i])."""
    return mask2d.reshape(-1).astype(np.int32)


def rel_err(a, b) -> float:
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))
