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
    """Seeded layout of lines and contacts, 0/1 [ndivy][ndivx] (1 = vacuum).

    Axis-aligned lines of width 16..64 nm at pitch 2-4x width plus square
    contacts 16..64 nm, absorber area fraction around `frac`."""
    rng = np.random.Generator(np.random.PCG64(seed))
    m = np.ones((ndivy, ndivx), np.uint8)
    vertical = rng.random() < 0.5
    w = int(rng.integers(max(2, min(16, ndivx // 16)), max(3, min(64, ndivx // 4))))
    pitch = int(w * rng.uniform(2.0, 4.0))
    off = int(rng.integers(0, pitch))
    n = ndivx if vertical else ndivy
    for s in range(off, n, pitch):
        if vertical:
            m[:, s:s + w] = 0
        else:
            m[s:s + w, :] = 0
    while (1.0 - m.mean()) < frac:
        c = int(rng.integers(max(2, min(16, ndivx // 16)), max(3, min(64, ndivx // 4))))
        x = int(rng.integers(0, ndivx - c))
        y = int(rng.integers(0, ndivy - c))
        m[y:y + c, x:x + c] = 0
    return m


def packed(mask2d: np.ndarray) -> np.ndarray:
    return np.packbits(mask2d.reshape(-1), bitorder="big")


def flat_bits(mask2d: np.ndarray) -> np.ndarray:
    """Oracle mask2d layout (int32 [ndivx*j + i])."""
    return mask2d.reshape(-1).astype(np.int32)


def rel_err(a, b) -> float:
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))
