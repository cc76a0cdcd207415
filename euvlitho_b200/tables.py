"""Config-only index and coefficient tables (host side, built once per plan).

These follow the set-up loops of the reference drivers: order sets
(intensity.cpp:148-164, m3d.cpp:113-157), the pupil set with the xinput flag
(intensity.cpp:166-195, m3d.cpp:160-195), the Bloch-family source lists
(source(), intensity.cpp:467-502), and the per-(source, pupil order) E-field
factors of the Abbe loop (rotate(), intensity.cpp:276-353, 423-465).  They
depend on the configuration only, never on a mask, so a plan keeps them
resident on the device.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Dict, List, Tuple

import numpy as np

from .config import PI, SimConfig


def order_set(kind: str, LMAX: int, MMAX: int) -> Tuple[np.ndarray, np.ndarray]:
    """Orders (l, m) in the reference enumeration (l outer, m inner)."""
    l = np.repeat(np.arange(-LMAX, LMAX + 1), 2 * MMAX + 1)
    m = np.tile(np.arange(-MMAX, MMAX + 1), 2 * LMAX + 1)
    if kind == "diamond":  # intensity.cpp:156
        keep = (np.abs(l) / float(LMAX + 0.01) + 1.0) * (np.abs(m) / float(MMAX + 0.01) + 1.0) <= 2.0
    elif kind == "ellipse":  # m3d.cpp:123
        keep = (l / float(LMAX + 0.01)) ** 2 + (m / float(MMAX + 0.01)) ** 2 <= 1.0
    elif kind == "box":
        keep = np.ones(l.shape, bool)
    else:
        raise ValueError("unknown order set %r" % kind)
    return l[keep].astype(np.int32), m[keep].astype(np.int32)


def in_na(cfg: SimConfig, l, m):
    """(l MX/dx)^2 + (m MY/dy)^2 <= (NA/lambda)^2 (intensity.cpp:177-179)."""
    l = np.asarray(l)
    m = np.asarray(m)
    return ((l * cfg.mx) / cfg.dx) ** 2 + ((m * cfg.my) / cfg.dy) ** 2 <= (cfg.na / cfg.wavelength) ** 2


def na_sources(cfg: SimConfig) -> List[Tuple[int, int]]:
    """Source orders inside the NA circle, ls outer / ms inner (header.h:1394-1397)."""
    out = []
    for ls in range(-cfg.lsmaxX, cfg.lsmaxX + 1):
        for ms in range(-cfg.lsmaxY, cfg.lsmaxY + 1):
            if in_na(cfg, ls, ms):
                out.append((ls, ms))
    return out


def pupil_set(cfg: SimConfig):
    """(linput, minput, xinput, snum): pupil orders seen by at least one NA
    source, l-major; xinput = snum >= 8 (m3d.cpp:181-186)."""
    lsx, lsy, lpx, lpy = cfg.lsmaxX, cfg.lsmaxY, cfg.lpmaxX, cfg.lpmaxY
    ls = np.arange(-lsx, lsx + 1)[:, None]
    ms = np.arange(-lsy, lsy + 1)[None, :]
    src_ok = in_na(cfg, ls, ms)  # [nsX, nsY]
    lp = np.arange(-lpx, lpx + 1)[:, None, None, None]
    mp = np.arange(-lpy, lpy + 1)[None, :, None, None]
    both = src_ok[None, None] & in_na(cfg, lp + ls[None, None], mp + ms[None, None])
    snum = both.sum(axis=(2, 3))  # [noutX, noutY]
    ip, jp = np.nonzero(snum > 0)  # row-major = ip outer, jp inner
    lin = (ip - lpx).astype(np.int32)
    min_ = (jp - lpy).astype(np.int32)
    sn = snum[ip, jp]
    return lin, min_, (sn >= 8).astype(np.int32), sn.astype(np.int32)


@dataclass
class Family:
    nsx: int
    nsy: int
    pts: List[Tuple[int, int]]


def sources(cfg: SimConfig) -> Tuple[int, List[Family]]:
    """Bloch families and their source orders (intensity.cpp:467-502); empty
    families are dropped, ``max_sources`` keeps the first points of the
    family-major enumeration."""
    ndivs = cfg.ndivs_eff()
    k, NA, MX, MY = cfg.k, cfg.na, cfg.mx, cfg.my
    dkx, dky = 2.0 * PI / cfg.dx, 2.0 * PI / cfg.dy
    l0max = int(k * NA / MX * cfg.sigma1 / dkx + 1)
    m0max = int(k * NA / MY * cfg.sigma1 / dky + 1)
    tan_half = np.tan(PI * cfg.openangle / 180.0 / 2.0)
    s1, s2, t = cfg.sigma1, cfg.sigma2, cfg.illum_type
    fams: List[Family] = []
    total = 0
    for nsx in range(ndivs):
        for nsy in range(ndivs):
            pts = []
            for l in range(-l0max, l0max + 1):
                for m in range(-m0max, m0max + 1):
                    skx = l * dkx + 2.0 * PI / cfg.dx * nsx / float(ndivs)
                    sky = m * dky + 2.0 * PI / cfg.dy * nsy / float(ndivs)
                    skxo, skyo = skx * MX, sky * MY
                    r2 = skxo * skxo + skyo * skyo
                    r = np.sqrt(r2)
                    ok = ((t == 0 and r2 <= (k * NA * s1) ** 2)
                          or (t == 1 and r <= k * NA * s1 and r >= k * NA * s2)
                          or (t == 2 and r <= k * NA * s1 and r >= k * NA * s2
                              and abs(skyo) <= abs(skxo) * tan_half)
                          or (t == 3 and r <= k * NA * s1 and r >= k * NA * s2
                              and abs(skxo) <= abs(skyo) * tan_half))
                    if ok and (cfg.max_sources is None or total < cfg.max_sources):
                        pts.append((l, m))
                        total += 1
            if pts:
                fams.append(Family(nsx, nsy, pts))
    return ndivs, fams


def rotate(k, MX, MY, px, py, sx0, sy0) -> np.ndarray:
    """Polarisation rotation R (3x2) of intensity.cpp:423-465, vectorised over
    (px, py); returns [..., 3, 2]."""
    px = np.asarray(px, np.float64)
    py = np.asarray(py, np.float64)
    shp = np.broadcast(px, py).shape
    px = np.broadcast_to(px, shp)
    py = np.broadcast_to(py, shp)
    s0 = np.array([sx0, sy0, -np.sqrt(k * k - sx0 * sx0 - sy0 * sy0)])
    s0b = np.broadcast_to(s0, shp + (3,))
    zero = np.zeros(shp)
    p = np.stack([px, py, zero], -1)
    with np.errstate(invalid="ignore"):  # points outside the pupil are filtered by the caller
        pp = np.stack([MX * px, MY * py, -np.sqrt(k * k - MX * px * MX * px - MY * py * MY * py)], -1)
    ez = np.broadcast_to(np.array([0.0, 0.0, 1.0]), shp + (3,))
    unit = lambda v: v / np.linalg.norm(v, axis=-1, keepdims=True)
    with np.errstate(invalid="ignore", divide="ignore"):
        es_a = unit(np.cross(p, s0b))
        esp_a = unit(np.cross(pp, ez))
        em_a = np.cross(es_a, unit(p + s0b))
        emp_a = np.cross(esp_a, pp) / k
        es_b = unit(np.cross(ez, s0b))
        esp_b = -es_b
        em_b = np.cross(es_b, s0b) / k
        emp_b = np.cross(esp_b, -ez)
    a = ((px * px + py * py) > 0.00001)[..., None]
    es = np.where(a, es_a, es_b)
    esp = np.where(a, esp_a, esp_b)
    em = np.where(a, em_a, em_b)
    emp = np.where(a, emp_a, emp_b)
    return esp[..., :, None] * es[..., None, :2] + emp[..., :, None] * em[..., None, :2]


def order_positions(lidx, midx) -> Dict[Tuple[int, int], int]:
    return {(int(a), int(b)): i for i, (a, b) in enumerate(zip(lidx, midx))}


def family_offsets(cfg: SimConfig, ndivs: int, fam: Family) -> Tuple[float, float]:
    """sx0, sy0 of a family (intensity.cpp:234-238)."""
    sx0 = 2.0 * PI / cfg.dx * fam.nsx / float(ndivs) + cfg.kx0
    sy0 = 2.0 * PI / cfg.dy * fam.nsy / float(ndivs) + cfg.ky0
    return sx0, sy0


def abbe_table(cfg: SimConfig, pol: str, ndivs: int, fam: Family, pos, linput, minput, n_src: int):
    """E-field factors of one (polarisation, family): coef[s][i][3] and the order
    index nidx[s][i] of pupil point i seen from source s (-1 = outside the
    pupil NA), following intensity.cpp:276-366."""
    k, dx, dy, MX, MY, NA = cfg.k, cfg.dx, cfg.dy, cfg.mx, cfg.my, cfg.na
    kx0, ky0, z0, z = cfg.kx0, cfg.ky0, cfg.z0, float(cfg.z)
    sx0, sy0 = family_offsets(cfg, ndivs, fam)
    ncut = len(linput)
    coef = np.zeros((n_src, ncut, 3), np.complex128)
    nidx = np.full((n_src, ncut), -1, np.int32)
    for s, (l0, m0) in enumerate(fam.pts):
        kx = sx0 + 2.0 * PI / dx * l0
        ky = sy0 + 2.0 * PI / dy * m0
        kxn = 2.0 * PI / dx * fam.nsx / float(ndivs) + 2.0 * PI / dx * l0 + 2.0 * PI * linput / dx
        kyn = 2.0 * PI / dy * fam.nsy / float(ndivs) + 2.0 * PI / dy * m0 + 2.0 * PI * minput / dy
        ok = (MX * MX * kxn * kxn + MY * MY * kyn * kyn) <= (NA * k) ** 2
        R = rotate(k, MX, MY, kxn, kyn, kx0, ky0)  # [ncut, 3, 2]
        phase = np.exp(1j * ((kxn + kx0) * (kxn + kx0) + (kyn + ky0) * (kyn + ky0)) / 2.0 / k * z0
                       + 1j * (MX * MX * kxn * kxn + MY * MY * kyn * kyn) / 2.0 / k * z)
        if pol == "X":
            f = 1j * k * R[:, :, 0] / np.sqrt(k * k - kx * kx)
        else:
            f = 1j * k * R[:, :, 1] / np.sqrt(k * k - ky * ky)
        for i in np.nonzero(ok)[0]:
            key = (int(l0 + linput[i]), int(m0 + minput[i]))
            n = pos.get(key)
            if n is None:
                raise ValueError("order set misses pupil order %s of source %s; widen the "
                                 "order set" % (key, (l0, m0)))
            nidx[s, i] = n
            coef[s, i] = f[i] * phase[i]
    return coef, nidx


def required_orders(cfg: SimConfig) -> Tuple[int, int]:
    """Largest |l|, |m| of the diffracted orders the Abbe loop reads: source
    order + pupil order inside the pupil NA (intensity.cpp:320-321, 356).  An
    order set must contain them (the reference reads its -1000 sentinel
    otherwise, intensity.cpp:297-299)."""
    k, dx, dy, MX, MY, NA = cfg.k, cfg.dx, cfg.dy, cfg.mx, cfg.my, cfg.na
    ndivs, fams = sources(cfg)
    lin, mn, _, _ = pupil_set(cfg)
    lmax = mmax = 0
    for f in fams:
        pts = np.array(f.pts)
        l0 = pts[:, 0][:, None]
        m0 = pts[:, 1][:, None]
        kxn = 2.0 * PI / dx * f.nsx / float(ndivs) + 2.0 * PI / dx * l0 + 2.0 * PI * lin[None, :] / dx
        kyn = 2.0 * PI / dy * f.nsy / float(ndivs) + 2.0 * PI / dy * m0 + 2.0 * PI * mn[None, :] / dy
        ok = (MX * MX * kxn * kxn + MY * MY * kyn * kyn) <= (NA * k) ** 2
        if ok.any():
            lmax = max(lmax, int(np.abs(l0 + lin[None, :])[ok].max()))
            mmax = max(mmax, int(np.abs(m0 + mn[None, :])[ok].max()))
    return lmax, mmax


def row_starts(linput: np.ndarray, lpx: int) -> np.ndarray:
    """row_start[l] = first pupil point with linput = l - lpx (points are l-major)."""
    if np.any(np.diff(linput) < 0):
        raise ValueError("pupil points must be l-major")
    return np.searchsorted(linput, np.arange(-lpx, lpx + 2), side="left").astype(np.int32)


# ----------------------------------------------------------- linear model
def linear_sources(cfg: SimConfig, mesh_deg: float = 0.2) -> Tuple[np.ndarray, np.ndarray]:
    """Source shifts (dsx, dsy) of the linear model (linear.py:47-96): a square
    grid of step k * mesh (radians) in the mask-side source plane, l outer and
    m inner, kept where the illumination holds at (MX dsx, MY dsy)."""
    k, NA = cfg.k, cfg.na
    kmesh = k * mesh_deg * (PI / 180.0)
    l0max = int(k * NA / cfg.mx * cfg.sigma1 / kmesh) + 1
    m0max = int(k * NA / cfg.my * cfg.sigma1 / kmesh) + 1
    l, m = np.meshgrid(np.arange(-l0max, l0max + 1), np.arange(-m0max, m0max + 1), indexing="ij")
    skx, sky = (l * kmesh).ravel(), (m * kmesh).ravel()
    xo, yo = skx * cfg.mx, sky * cfg.my
    r = np.sqrt(xo * xo + yo * yo)
    r1, r2 = k * NA * cfg.sigma1, k * NA * cfg.sigma2
    t = np.tan(PI * cfg.openangle / 180.0 / 2.0)
    ring = (r2 <= r) & (r <= r1)
    ok = {0: xo * xo + yo * yo <= r1 * r1, 1: ring,
          2: ring & (np.abs(yo) <= np.abs(xo) * t),
          3: ring & (np.abs(xo) <= np.abs(yo) * t)}[int(cfg.illum_type)]
    return skx[ok], sky[ok]


def linear_abbe_table(cfg: SimConfig, dsx, dsy, linput, minput):
    """E-field factors of the linear model for the fused Abbe kernel:
    coef[s][i][3] = i k R(:, 0) phase / sqrt(k^2 - (kx0 + dsx_s)^2) and the
    identity index nidx[s][i] = i (-1 where the pupil point is outside
    obscuration <= |p| / (NA k) <= 1), X polarisation, following
    elitho/electro_field.py:45-76 and linear.py:11-43 (phase with z0 and the
    defocus cfg.z)."""
    k, dx, dy, MX, MY, NA = cfg.k, cfg.dx, cfg.dy, cfg.mx, cfg.my, cfg.na
    kx0, ky0, z0, z = cfg.kx0, cfg.ky0, cfg.z0, float(cfg.z)
    dsx = np.asarray(dsx, np.float64)[:, None]
    dsy = np.asarray(dsy, np.float64)[:, None]
    kxn = dsx + 2.0 * PI * np.asarray(linput, np.float64)[None, :] / dx
    kyn = dsy + 2.0 * PI * np.asarray(minput, np.float64)[None, :] / dy
    p2 = MX * MX * kxn * kxn + MY * MY * kyn * kyn
    ok = (p2 <= (NA * k) ** 2) & (p2 >= (NA * k * cfg.obscuration) ** 2)
    R = rotate(k, MX, MY, kxn, kyn, kx0, ky0)[..., 0]  # [S, ncut, 3]
    phase = np.exp(1j * ((kxn + kx0) ** 2 + (kyn + ky0) ** 2) / (2.0 * k) * z0
                   + 1j * p2 / (2.0 * k) * z)
    f = 1j * k / np.sqrt(k * k - (kx0 + dsx) ** 2)
    coef = np.where(ok[..., None], (f * phase)[..., None] * R, 0.0).astype(np.complex128)
    nidx = np.where(ok, np.arange(len(linput), dtype=np.int32)[None, :], -1).astype(np.int32)
    return coef, nidx


# ----------------------------------------------------------- STCC-SOCS
def socs_phase(cfg: SimConfig, z: float, dsx, dsy, linput, minput):
    """Pupil-source phase matrices of the TCC (eigenfunction.py:84-111):
    P[c][i][s] = phase(i, s) R(c, 0) for pupil point i and source s (zero
    outside the pupil NA), and the source weight w0[s] = k^2 / (k^2 - (kx0 +
    dsx_s)^2).  TCC_w = sum_c P_c diag(w w0) P_c^H / S for w = 1, dsx, dsy."""
    k, dx, dy, MX, MY, NA = cfg.k, cfg.dx, cfg.dy, cfg.mx, cfg.my, cfg.na
    kx0, ky0, z0 = cfg.kx0, cfg.ky0, cfg.z0
    dsx = np.asarray(dsx, np.float64)
    dsy = np.asarray(dsy, np.float64)
    ksx = (2 * PI / dx * np.asarray(linput, np.float64))[:, None] + dsx[None, :]
    ksy = (2 * PI / dy * np.asarray(minput, np.float64))[:, None] + dsy[None, :]
    p2 = MX * MX * ksx * ksx + MY * MY * ksy * ksy
    phase = np.exp(1j * ((ksx + kx0) ** 2 + (ksy + ky0) ** 2) / 2.0 / k * z0
                   + 1j * p2 / 2.0 / k * z) * (p2 <= (k * NA) ** 2)
    R = rotate(k, MX, MY, ksx, ksy, kx0, ky0)[..., 0]  # [n, S, 3]
    P = np.moveaxis(phase[..., None] * R, -1, 0)       # [3, n, S]
    w0 = k * k / (k * k - (kx0 + dsx) ** 2)
    return np.nan_to_num(P), w0


def socs_interp_tables(nout: int, xdiv: int, ydiv: int):
    """DFT matrix E[a][b] = e^{2 pi i a b / nout} and the Fourier-interpolation
    kernels K[x][u] = (1/nout) sum_{i=-nout/2}^{nout/2-1} e^{2 pi i i (x/xdiv - u/nout)}
    (socs.py:137-150) for x and y."""
    a = np.arange(nout)
    E = np.exp(2j * PI * np.outer(a, a) / nout)
    i = np.arange(-(nout // 2), nout // 2)

    def kern(xd):
        x = np.arange(xd)
        ph = x[:, None, None] / xd - a[None, :, None] / nout  # [x, u, 1]
        return np.exp(2j * PI * i[None, None, :] * ph).sum(-1) / nout

    return E, kern(xdiv), kern(ydiv)
