"""Seeded synthetic mask clips (input generator for tests and measurements).

The reference ships one mask and a rand()-driven line generator
(cnn/intensity/mask/mask.cpp, mVBF.h); the measured workloads use seeded
layouts instead: axis-aligned lines 16-64 nm wide at a pitch of 2-4x their
width plus square contacts 16-64 nm, drawn until the absorber covers ~36 % of
the clip (the reference mask has 63.9 % vacuum).  Output arrays are 0/1
[ndivy][ndivx] with 1 = vacuum (row j = y), packed MSB first like mask.bin.
"""
from __future__ import annotations

from typing import List

import numpy as np


def synth_mask(ndivx: int, ndivy: int, seed: int, frac: float = 0.36) -> np.ndarray:
    rng = np.random.Generator(np.random.PCG64(seed))
    m = np.ones((ndivy, ndivx), np.uint8)
    lo = max(2, min(16, ndivx // 16))
    hi = max(lo + 1, min(64, ndivx // 4))
    vertical = rng.random() < 0.5
    w = int(rng.integers(lo, hi))
    pitch = int(w * rng.uniform(2.0, 4.0))
    off = int(rng.integers(0, pitch))
    n = ndivx if vertical else ndivy
    for s in range(off, n, pitch):
        if vertical:
            m[:, s:s + w] = 0
        else:
            m[s:s + w, :] = 0
    while (1.0 - m.mean()) < frac:
        c = int(rng.integers(lo, hi))
        x = int(rng.integers(0, ndivx - c))
        y = int(rng.integers(0, ndivy - c))
        m[y:y + c, x:x + c] = 0
    return m


def sidewall_slices(mask: np.ndarray, n_slices: int, slice_nm: float, angle_deg: float = 84.0,
                    pixel_nm: float = 1.0) -> List[np.ndarray]:
    """Per-slice masks of an absorber with a sloped sidewall (index 0 = top).

    The drawn mask is the bottom slice; every slice above is eroded (absorber
    shrinks) by round(depth * tan(90 deg - angle) / pixel) pixels on each side,
    depth measured from the bottom slice.  Rounded pixel erosion."""
    bias = slice_nm * np.tan(np.deg2rad(90.0 - angle_deg)) / pixel_nm
    out = []
    for n in range(n_slices):
        r = int(round((n_slices - 1 - n) * bias))
        a = (mask == 0)
        for _ in range(r):  # erode the absorber by one pixel in x and y
            a = a & np.roll(a, 1, 0) & np.roll(a, -1, 0) & np.roll(a, 1, 1) & np.roll(a, -1, 1)
        out.append((~a).astype(np.uint8))
    return out


def pack(mask2d: np.ndarray) -> np.ndarray:
    return np.packbits(np.asarray(mask2d, np.uint8).reshape(-1), bitorder="big")


def batch(ndivx: int, ndivy: int, seeds, n_slices: int = 1, slice_nm: float = 0.0,
          angle_deg: float = 84.0) -> np.ndarray:
    """Packed uint8 [clips, slices, bytes] for the given seeds; n_slices > 1
    gives sidewall slices."""
    out = []
    for s in seeds:
        m = synth_mask(ndivx, ndivy, int(s))
        if n_slices > 1:
            out.append(np.stack([pack(x) for x in sidewall_slices(m, n_slices, slice_nm, angle_deg)]))
        else:
            out.append(pack(m)[None])
    return np.stack(out)
