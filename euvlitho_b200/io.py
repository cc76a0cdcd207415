"""File formats of the reference drivers.

* mask.bin: ndivx*ndivy bits, MSB first, bit index ndivx*j + i, 1 = vacuum
  (intensity.cpp:20-29, 110-116, 197-207); several masks are concatenated
  (m3d.cpp:87-88, 199-203).
* emint.csv: rows j = YDIV-1 .. 0, each value printed with 6 significant
  digits and followed by ',' (intensity.cpp:390-408).
* inputxx.csv: six rows Re a0, Im a0 (all pupil orders), Re ax, Im ax, Re ay,
  Im ay (orders with xinput = 1) (m3d.cpp:468-558).
* inputlm.csv: one row "l,m,xinput" per pupil order (m3d.cpp:159-195).
"""
from __future__ import annotations

import numpy as np


def read_mask_bin(path: str, ndivx: int, ndivy: int, count: int = 1) -> np.ndarray:
    """Packed masks as uint8 [count, ndivx*ndivy/8]."""
    nb = ndivx * ndivy // 8
    data = np.fromfile(path, dtype=np.uint8, count=nb * count)
    if data.size != nb * count:
        raise ValueError("%s holds %d bytes, expected %d" % (path, data.size, nb * count))
    return data.reshape(count, nb)


def write_mask_bin(path: str, packed: np.ndarray) -> None:
    np.asarray(packed, np.uint8).tofile(path)


def pack_mask(mask2d: np.ndarray) -> np.ndarray:
    """0/1 array [ndivy, ndivx] (row j = y) -> packed MSB-first bytes."""
    return np.packbits(np.asarray(mask2d, np.uint8).reshape(-1), bitorder="big")


def unpack_mask(packed: np.ndarray, ndivx: int, ndivy: int) -> np.ndarray:
    return np.unpackbits(np.asarray(packed, np.uint8), bitorder="big")[: ndivx * ndivy].reshape(ndivy, ndivx)


def _fmt(v: float) -> str:
    return "%.6g," % v


def write_emint(path: str, image: np.ndarray) -> None:
    """image[x][y] -> emint.csv."""
    I = np.asarray(image)
    with open(path, "w") as fh:
        for j in range(I.shape[1] - 1, -1, -1):
            fh.write("".join(_fmt(I[i, j]) for i in range(I.shape[0])))
            fh.write("\n")


def read_emint(path_or_file) -> np.ndarray:
    fh = open(path_or_file) if isinstance(path_or_file, str) else path_or_file
    rows = [[float(v) for v in line.strip().split(",") if v] for line in fh]
    rows = [r for r in rows if r]
    return np.array(rows)[::-1, :].T.copy()


def write_inputxx(path: str, a0, ax, ay, xinput) -> None:
    sel = np.asarray(xinput) == 1
    a0, ax, ay = np.asarray(a0), np.asarray(ax)[sel], np.asarray(ay)[sel]
    with open(path, "w") as fh:
        for row in (a0.real, a0.imag, ax.real, ax.imag, ay.real, ay.imag):
            fh.write("".join(_fmt(v) for v in row))
            fh.write("\n")


def read_inputxx(path_or_file):
    fh = open(path_or_file) if isinstance(path_or_file, str) else path_or_file
    rows = [np.array([float(v) for v in line.strip().split(",") if v]) for line in fh]
    return {"a0": rows[0] + 1j * rows[1], "ax": rows[2] + 1j * rows[3], "ay": rows[4] + 1j * rows[5]}


def expand_xinput(values, xinput) -> np.ndarray:
    """Slopes stored for the xinput points only (inputxx.csv rows 3-6) -> one
    value per pupil point, zero elsewhere."""
    out = np.zeros(len(xinput), np.complex128)
    out[np.asarray(xinput) == 1] = values
    return out


def write_image_full(path: str, image: np.ndarray) -> None:
    """linear.py's intlinear.csv / intft.csv layout (linear.py:245-258): row j
    holds I[i][XDIV-1-j] for i < XDIV, each value at full precision followed by
    a comma."""
    n = image.shape[0]
    with open(path, "w") as fh:
        for j in range(n):
            fh.write("".join("%r," % float(image[i, n - 1 - j]) for i in range(n)))
            fh.write("\n")


def write_inputlm(path: str, linput, minput, xinput) -> None:
    with open(path, "w") as fh:
        for l, m, x in zip(linput, minput, xinput):
            fh.write("%d,%d,%d\n" % (l, m, x))
