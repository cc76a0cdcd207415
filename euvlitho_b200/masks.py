"""Seeded synthetic mask clips (input generator for tests and measurements).

The reference ships one mask and a rand()-driven line generator
(cnn/intensity/mask/mask.cpp, mVBF.h), reproduced here bit for bit
(``vbf_rectangles`` + the device rasteriser ``rasterize``); the measured
workloads use seeded layouts instead: axis-aligned lines 16-64 nm wide at a pitch of 2-4x their
width plus square contacts 16-64 nm, drawn until the absorber covers ~36 % of
the clip (the reference mask has 63.9 % vacuum).  Output arrays are 0/1
[ndivy][ndivx] with 1 = vacuum (row j = y), packed MSB first like mask.bin.
"""
from __future__ import annotations

import ctypes
import ctypes.util
from typing import List, Optional, Sequence, Tuple

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


def unpack(bits: np.ndarray, ndivx: int, ndivy: int) -> np.ndarray:
    return np.unpackbits(np.asarray(bits, np.uint8), bitorder="big")[: ndivx * ndivy].reshape(ndivy, ndivx)


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


# ------------------------------------------------------------ reference generator
class LibcRand:
    """The C library's rand() stream, which the reference's mask generator
    draws from (mask.cpp never calls srand: seed 1).  ``srand(seed)`` on
    creation.  The stream is the process's single libc generator, so draw
    from one LibcRand at a time."""

    def __init__(self, seed: int = 1):
        self._libc = ctypes.CDLL(ctypes.util.find_library("c"))
        self._libc.srand(int(seed))

    def __call__(self) -> int:
        return int(self._libc.rand())


def vbf_rectangles(ndivx: int, ndivy: int, rand, cd: int = 56,
                   gap: int = 80) -> List[Tuple[int, int, int, int]]:
    """Absorber rectangles (x0, x1, y0, y1), half-open, of one mask of the
    reference generator (mVBF.h:2-70), drawing from ``rand``: columns of width
    cd alternate between vacuum stripes and absorber lines broken along y into
    runs of gap * (rand() % 5) (+ 3 gap for absorber runs).  The tail rules are
    kept: past the last full run, a column tail is absorber when the next run
    would have been a gap; past the last full stripe, the tail is absorber when
    the next stripe would have been a line, else a copy of the last line's y
    pattern (vacuum if no line was drawn: the reference leaves that array
    uninitialised)."""
    def line_runs() -> List[Tuple[int, int]]:  # mVBF.h:41-70
        runs = []
        line = rand() % 2
        s = 0
        while s < ndivy - gap:
            a = gap * (rand() % 5)
            if line == 1:
                a += 3 * gap
                runs.append((s, min(s + a, ndivy)))
            line = 1 - line
            s += a
        if line == 0 and s < ndivy:
            runs.append((s, ndivy))
        return runs

    rects: List[Tuple[int, int, int, int]] = []
    last: List[Tuple[int, int]] = []
    space = rand() % 2
    s = 0
    while s < ndivx - cd:  # mVBF.h:11-29
        x1 = min(s + cd, ndivx)
        if space == 1:
            space = 0
        else:
            last = line_runs()
            rects.extend((s, x1, y0, y1) for y0, y1 in last)
            space = 1
        s += cd
    if s < ndivx:  # mVBF.h:30-38
        if space == 0:
            rects.append((s, ndivx, 0, ndivy))
        else:
            rects.extend((s, ndivx, y0, y1) for y0, y1 in last)
    return rects


def paint(rects, ndivx: int, ndivy: int) -> np.ndarray:
    """Host raster of absorber rectangles on vacuum: 0/1 [ndivy][ndivx]."""
    m = np.ones((ndivy, ndivx), np.uint8)
    for x0, x1, y0, y1 in rects:
        # clip both ends to the grid (a negative end must not wrap)
        xa, xb = min(max(x0, 0), ndivx), min(max(x1, 0), ndivx)
        ya, yb = min(max(y0, 0), ndivy), min(max(y1, 0), ndivy)
        m[ya:yb, xa:xb] = 0
    return m


def sidewall_erosion(n_slices: int, slice_nm: float, angle_deg: float = 84.0,
                     pixel_nm: float = 1.0) -> List[int]:
    """Erosion radius (pixels) of each slice, index 0 = top: the rule of
    ``sidewall_slices``."""
    bias = slice_nm * np.tan(np.deg2rad(90.0 - angle_deg)) / pixel_nm
    return [int(round((n_slices - 1 - n) * bias)) for n in range(n_slices)]


def rasterize(rects_per_mask: Sequence[Sequence[Tuple[int, int, int, int]]], ndivx: int,
              ndivy: int, erosion: Sequence[int] = (0,), device=None, out=None):
    """Packed masks [n_masks, n_slices, ndivx*ndivy/8] on the device from
    absorber rectangles (euv_mask_raster): slice s eroded by erosion[s]
    cross steps (``sidewall_erosion``).  ``out``: an existing uint8 tensor of
    that shape to fill."""
    import torch
    from . import _lib as L
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    n = len(rects_per_mask)
    flat = [(m, *r) for m, rs in enumerate(rects_per_mask) for r in rs]
    d_rects = (torch.tensor(flat, dtype=torch.int32).to(dev) if flat
               else torch.zeros((1, 5), dtype=torch.int32, device=dev))
    er = (ctypes.c_int * len(erosion))(*[int(e) for e in erosion])
    nb = ndivx * ndivy // 8
    if out is None:
        out = torch.empty((n, len(erosion), nb), dtype=torch.uint8, device=dev)
    wb = L.lib().euv_mask_raster_workspace_bytes(n, ndivx, ndivy)
    ws = torch.empty(wb, dtype=torch.uint8, device=dev)
    L.call("euv_mask_raster", n, ndivx, ndivy, len(flat), d_rects.data_ptr(), len(erosion), er,
           out.data_ptr(), ws.data_ptr(), wb, torch.cuda.current_stream(dev).cuda_stream)
    return out


def vbf_batch(n: int, ndivx: int = 2048, ndivy: int = 2048, seed: int = 1,
              erosion: Sequence[int] = (0,), device=None, rand: Optional[LibcRand] = None):
    """n consecutive masks of the reference generator (mask.cpp's ndata loop),
    rasterised on the device: [n, slices, bytes]."""
    rand = rand if rand is not None else LibcRand(seed)
    rects = [vbf_rectangles(ndivx, ndivy, rand) for _ in range(n)]
    return rasterize(rects, ndivx, ndivy, erosion, device)
