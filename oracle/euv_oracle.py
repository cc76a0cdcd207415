"""CPU FP64 oracle for the rigorous EUV mask-3D solve, Abbe imaging and M3D fit.

TEST INFRASTRUCTURE ONLY.  This module is the checker: only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may import
it.  The product (``euvlitho_b200``) never imports, links or calls it; the
product fails loudly when its CUDA library is missing.

It restates, in NumPy/SciPy double precision, the algorithm of the reference
(takahashi-edalab/EUVlitho, paths relative to the reference repository):

* ``cnn/include/header.h``      -- ``multilayerS`` (5-363), ``absorberS``
  (365-752), ``absorberS0`` (754-1145), ``maskamp`` (1147-1206), ``ampS``
  (1208-1466), ``matinv``/``matproduct`` (1468-1619), ``fourier``/``exponential``
  (1621-1648);
* ``cnn/intensity/abbe/intensity.cpp`` -- order/pupil sets (139-195), the Abbe
  loop (219-408), ``rotate`` (423-465), ``source`` (467-502),
  ``decompressBits`` (20-29);
* ``cnn/intensity/m3d/m3d.cpp`` -- narrow/wide order sets (97-157), pupil set
  with the ``xinput`` flag (159-195), the M3D-parameter extraction (212-558).

The eigen-decomposition is LAPACK ``zgeev`` (``numpy.linalg.eig``) where the
reference calls cuSOLVER ``Xgeev``; inverses are LU (``numpy.linalg.inv``) where
the reference uses Eigen ``colPivHouseholderQr`` (N<=5000) or cuSOLVER
``getrf/getrs``.  These give the same invariant outputs (Ax, intensity, M3D
parameters) to rounding; eigenvector scaling/order does not reach the outputs.

Reference quirks are kept, behind flags where the build generalises:

1. ``sigma1`` is not refreshed in the slice loop (header.h:1327-1353):
   ``refresh_sigma=False`` reproduces it.
2. Every slice uses the same mask (header.h:1243-1251): pass one mask per
   slice to generalise (sidewall slices); a single mask reproduces it.
3. kx0 = k sin(theta0) cos(90 deg) is tiny but non-zero (intensity.cpp:235).
4. ``klm = sqrt(k^2 - kxy2)`` is a REAL square root (header.h:1283): an
   evanescent order gives NaN, as in the reference.
5. Square-grid Abbe (intensity.cpp:222,359-360) is generalised to
   XDIV x YDIV with XDIV = NDIVX/MX, YDIV = NDIVY/MY; square configurations
   are unchanged.

Parity of this module is pinned against the reference's golden outputs
``cnn/intensity/abbe/emint.csv`` and ``cnn/intensity/m3d/inputxx.csv`` by
``oracle/pin_golden.py`` (the fixture summary lives in ``tests/golden``).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

PI = float(np.arctan(1.0) * 4.0)  # intensity.cpp:55 ``pi=atan(1.)*4.``


# --------------------------------------------------------------------------
# Configuration (the constants of intensity.cpp:44-146 / m3d.cpp:34-157)
# --------------------------------------------------------------------------
@dataclass
class Stack:
    """Multilayer materials and thicknesses (header.h:1217-1223)."""

    n_mo: complex = 0.9238 + 0.006435j
    n_si: complex = 0.999 + 0.001826j
    n_ru: complex = 0.8863 + 0.01706j
    n_mosi2: complex = 0.9693 + 0.004333j
    n_rusi: complex = 0.9099 + 0.01547j
    n_sio2: complex = 0.978 + 0.01083j
    d_mo: float = 2.052
    d_mosi: float = 1.661
    d_si: float = 2.283
    d_simo: float = 1.045
    d_siru: float = 0.8
    d_ru: float = 2.5
    nml: int = 40


@dataclass
class SimConfig:
    """Geometry, optics, illumination and absorber of one simulation."""

    ndivx: int = 2048          # mask pixels in x (intensity.cpp:48)
    ndivy: int = 2048
    delta: float = 1.0         # Fourier grid step (intensity.cpp:106)
    wavelength: float = 13.5
    theta0: float = -6.0       # degrees (intensity.cpp:59)
    azimuth: float = 0.0
    na: float = 0.33
    mx: int = 4
    my: int = 4
    # illumination (intensity.cpp:67-71, source() 467-502)
    illum_type: int = 1        # 0 conventional, 1 annular, 2 X dipole, 3 Y dipole
    sigma1: float = 0.9        # outer
    sigma2: float = 0.55       # inner
    openangle: float = 90.0
    sigmadiv: float = 0.5
    ndivs: Optional[int] = None      # None: reference rule intensity.cpp:90
    max_sources: Optional[int] = None  # keep only the first points (enumeration order)
    # absorber slices, index 0 = top slice (header.h:1331 uses NABS-1 = bottom)
    eabs: Sequence[complex] = (complex(0.9567, 0.0343) ** 2,)
    dabs: Sequence[float] = (60.0,)
    z0_offset: float = 42.0    # z0 = total absorber thickness + 42 (intensity.cpp:80)
    stack: Stack = field(default_factory=Stack)
    refresh_sigma: bool = False  # quirk 1
    # order sets
    order_kind: str = "diamond"  # "diamond" (cut), "ellipse" (cut), "box" (lbox, mbox)
    cut: float = 6.0
    lbox: int = 0
    mbox: int = 0
    zlist: Sequence[int] = (0,)  # defocus (intensity.cpp:73-78)
    # pattern row j reads mask row NDIVY-1-j + yflip_offset (header.h:1159 has
    # 0; rows outside the mask are absorber).  1 reproduces the revision that
    # wrote the golden emint.csv / inputxx.csv.
    yflip_offset: int = 0
    # central obscuration of the pupil as a fraction of NA, used by the linear
    # model's E-field (elitho/const.py co: 0.2 at NA 0.55, 0 at NA 0.33)
    obscuration: float = 0.0

    @property
    def dx(self) -> float:
        return float(self.ndivx)

    @property
    def dy(self) -> float:
        return float(self.ndivy)

    @property
    def k(self) -> float:
        return 2.0 * PI / self.wavelength

    @property
    def fdivx(self) -> int:
        return int(self.dx / self.delta + 0.000001)

    @property
    def fdivy(self) -> int:
        return int(self.dy / self.delta + 0.000001)

    @property
    def kx0(self) -> float:
        phi0 = 90.0 - self.azimuth
        return self.k * np.sin(PI / 180.0 * self.theta0) * np.cos(PI / 180.0 * phi0)

    @property
    def ky0(self) -> float:
        phi0 = 90.0 - self.azimuth
        return self.k * np.sin(PI / 180.0 * self.theta0) * np.sin(PI / 180.0 * phi0)

    @property
    def z0(self) -> float:
        return float(sum(self.dabs)) + self.z0_offset

    @property
    def nabs(self) -> int:
        return len(self.eabs)

    # intensity.cpp:117-129
    @property
    def lsmaxX(self) -> int:
        return int(self.na * self.dx / float(self.mx) / self.wavelength + 1)

    @property
    def lsmaxY(self) -> int:
        return int(self.na * self.dy / float(self.my) / self.wavelength + 1)

    @property
    def lpmaxX(self) -> int:
        return int(self.na * self.dx / float(self.mx) * 2 / self.wavelength + 0.0001)

    @property
    def lpmaxY(self) -> int:
        return int(self.na * self.dy / float(self.my) * 2 / self.wavelength + 0.0001)

    @property
    def xdiv(self) -> int:
        return self.ndivx // self.mx

    @property
    def ydiv(self) -> int:
        return self.ndivy // self.my

    def ndivs_eff(self) -> int:
        if self.ndivs is not None:
            return int(self.ndivs)
        return max(1, int(180.0 / PI * self.wavelength / self.dx / self.sigmadiv))


# --------------------------------------------------------------------------
# Mask input
# --------------------------------------------------------------------------
def decompress_bits(data: bytes, nbits: int) -> np.ndarray:
    """MSB-first unpack (intensity.cpp:20-29); returns int32 mask2d[NDIVX*j+i]."""
    raw = np.frombuffer(data, dtype=np.uint8)
    bits = np.unpackbits(raw, bitorder="big")[:nbits]
    return bits.astype(np.int32)


def read_mask_bin(path: str, ndivx: int, ndivy: int, index: int = 0) -> np.ndarray:
    n = ndivx * ndivy
    with open(path, "rb") as fh:
        fh.seek(index * (n // 8))
        data = fh.read(n // 8)
    return decompress_bits(data, n)


# --------------------------------------------------------------------------
# Mask generator (cnn/intensity/mask/mVBF.h, mask.cpp)
# --------------------------------------------------------------------------
def vbf_mask(ndivx: int, ndivy: int, rand, cd: int = 56, gap: int = 80) -> np.ndarray:
    """One mask of the reference generator, mask2d[ndivx*j + i] (1 = vacuum),
    drawing from ``rand`` (a callable returning the C library's rand() values):
    columns of width cd alternate between all-vacuum stripes and absorber lines
    broken along y into runs of gap * (rand() % 5) (+ 3 gap for absorber runs)
    (mVBF.h:2-70, including its tail rules)."""
    m = np.zeros((ndivy, ndivx), np.int32)          # m[j][i]
    col = np.zeros(ndivy, np.int32)                  # mask1dY, kept across stripes

    def randmask():                                  # mVBF.h:41-70
        line = rand() % 2
        s = 0
        while s < ndivy - gap:
            a = gap * (rand() % 5)
            if line == 1:
                a += 3 * gap
            col[s:min(s + a, ndivy)] = 0 if line == 1 else 1
            line = 0 if line == 1 else 1
            s += a
        col[s:] = 0 if line == 0 else 1

    space = rand() % 2                               # mVBF.h:9-29
    s = 0
    while s < ndivx - cd:
        if space == 1:
            m[:, s:min(s + cd, ndivx)] = 1
            space = 0
        else:
            randmask()
            m[:, s:min(s + cd, ndivx)] = col[:, None]
            space = 1
        s += cd
    if space == 0:                                   # mVBF.h:30-38
        m[:, s:] = 0
    else:
        m[:, s:] = col[:, None]
    return m.reshape(-1)


# --------------------------------------------------------------------------
# Order sets, pupil set, sources
# --------------------------------------------------------------------------
def order_set(kind: str, LMAX: int, MMAX: int) -> Tuple[np.ndarray, np.ndarray]:
    """Orders (l,m) in the reference enumeration order (intensity.cpp:148-164).

    ``diamond``: (|l|/(L+.01)+1)(|m|/(M+.01)+1) <= 2 (intensity.cpp:156);
    ``ellipse``: (l/(L+.01))^2+(m/(M+.01))^2 <= 1 (m3d.cpp:123);
    ``box``: every (l,m) with |l|<=L, |m|<=M.
    """
    li, mi = [], []
    for i in range(2 * LMAX + 1):
        ii = i - LMAX
        for j in range(2 * MMAX + 1):
            jj = j - MMAX
            if kind == "diamond":
                ok = (abs(ii) / float(LMAX + 0.01) + 1.0) * (abs(jj) / float(MMAX + 0.01) + 1.0) <= 2.0
            elif kind == "ellipse":
                ok = (ii / float(LMAX + 0.01)) ** 2 + (jj / float(MMAX + 0.01)) ** 2 <= 1.0
            elif kind == "box":
                ok = True
            else:
                raise ValueError(kind)
            if ok:
                li.append(ii)
                mi.append(jj)
    return np.array(li, dtype=np.int64), np.array(mi, dtype=np.int64)


def order_limits(cfg: SimConfig, kind: str, cut: float) -> Tuple[int, int]:
    """LMAX, MMAX for a cut factor (intensity.cpp:139-146) or the box half sizes."""
    if kind == "box":
        return cfg.lbox, cfg.mbox
    cutx = cfg.na / cfg.mx * cut
    cuty = cfg.na / cfg.my * cut
    return int(cutx * cfg.dx / cfg.wavelength), int(cuty * cfg.dy / cfg.wavelength)


def _in_na(cfg: SimConfig, l, m) -> bool:
    return (l * cfg.mx / cfg.dx) ** 2 + (m * cfg.my / cfg.dy) ** 2 <= (cfg.na / cfg.wavelength) ** 2


def pupil_set(cfg: SimConfig):
    """Pupil orders with at least one overlapping source order (intensity.cpp:166-195,
    m3d.cpp:160-195).  Returns (linput, minput, xinput, snum)."""
    lsx, lsy, lpx, lpy = cfg.lsmaxX, cfg.lsmaxY, cfg.lpmaxX, cfg.lpmaxY
    lin, min_, xin, sn = [], [], [], []
    for ip in range(2 * lpx + 1):
        for jp in range(2 * lpy + 1):
            snum = 0
            for is_ in range(2 * lsx + 1):
                for js in range(2 * lsy + 1):
                    if _in_na(cfg, is_ - lsx, js - lsy) and _in_na(
                        cfg, ip - lpx + is_ - lsx, jp - lpy + js - lsy
                    ):
                        snum += 1
            if snum > 0:
                lin.append(ip - lpx)
                min_.append(jp - lpy)
                xin.append(1 if snum >= 8 else 0)
                sn.append(snum)
    return (np.array(lin, np.int64), np.array(min_, np.int64), np.array(xin, np.int64), np.array(sn, np.int64))


def source(cfg: SimConfig):
    """Source orders per Bloch family (intensity.cpp:467-502).

    Returns ``(ndivs, fams)`` with ``fams[(nsx,nsy)] = [(l, m), ...]`` in the
    reference enumeration order.  ``max_sources`` truncates the global
    enumeration (family-major) to its first points.
    """
    ndivs = cfg.ndivs_eff()
    k, NA, MX, MY = cfg.k, cfg.na, cfg.mx, cfg.my
    dkx, dky = 2.0 * PI / cfg.dx, 2.0 * PI / cfg.dy
    skangx = k * NA / MX * cfg.sigma1
    skangy = k * NA / MY * cfg.sigma1
    l0max = int(skangx / dkx + 1)
    m0max = int(skangy / dky + 1)
    s1, s2 = cfg.sigma1, cfg.sigma2
    tan_half = np.tan(PI * cfg.openangle / 180.0 / 2.0)
    fams: Dict[Tuple[int, int], List[Tuple[int, int]]] = {}
    total = 0
    for nsx in range(ndivs):
        for nsy in range(ndivs):
            pts = []
            for l in range(-l0max, l0max + 1):
                for m in range(-m0max, m0max + 1):
                    skx = l * dkx + 2.0 * PI / cfg.dx * nsx / float(ndivs)
                    sky = m * dky + 2.0 * PI / cfg.dy * nsy / float(ndivs)
                    skxo, skyo = skx * MX, sky * MY
                    r = np.sqrt(skxo * skxo + skyo * skyo)
                    t = cfg.illum_type
                    ok = (
                        (t == 0 and (skxo * skxo + skyo * skyo) <= (k * NA * s1) ** 2)
                        or (t == 1 and r <= k * NA * s1 and r >= k * NA * s2)
                        or (t == 2 and r <= k * NA * s1 and r >= k * NA * s2 and abs(skyo) <= abs(skxo) * tan_half)
                        or (t == 3 and r <= k * NA * s1 and r >= k * NA * s2 and abs(skxo) <= abs(skyo) * tan_half)
                    )
                    if ok:
                        if cfg.max_sources is not None and total >= cfg.max_sources:
                            continue
                        pts.append((l, m))
                        total += 1
            fams[(nsx, nsy)] = pts
    return ndivs, fams


# --------------------------------------------------------------------------
# Fourier coefficients of the mask pattern
# --------------------------------------------------------------------------
def exponential(fdiv: int) -> np.ndarray:
    """cexp[i] = exp(-2 pi i i/FDIV), i in [0, FDIV] (header.h:1637-1648)."""
    i = np.arange(fdiv + 1, dtype=np.float64)
    return np.exp(-2.0 * PI * 1j * i / float(fdiv))


def fourier(l: int, f: np.ndarray, cexp: np.ndarray, fdiv: int) -> complex:
    """Direct DFT coefficient (header.h:1621-1635)."""
    i = np.arange(fdiv, dtype=np.int64)
    if l >= 0:
        j = (i * l) % fdiv
    else:
        j = fdiv - ((-i * l) % fdiv)
    return complex(np.sum(f * cexp[j]) / float(fdiv))


def mask_pattern(mask2d: np.ndarray, cfg: SimConfig, ampta, ampvc) -> np.ndarray:
    """pattern(i,j), i = x in [0,FDIVX), j = y in [0,FDIVY) (header.h:1153-1166).
    Pixel y is flipped: jj = NDIVY-1-j/meshY."""
    FX, FY = cfg.fdivx, cfg.fdivy
    meshX, meshY = FX // cfg.ndivx, FY // cfg.ndivy
    ii = np.arange(FX) // meshX
    jj = cfg.ndivy - 1 - np.arange(FY) // meshY + cfg.yflip_offset
    m = mask2d.reshape(cfg.ndivy, cfg.ndivx)  # m[j][i] = mask2d[NDIVX*j+i]
    inside = (jj >= 0) & (jj < cfg.ndivy)
    bits = np.where(inside[:, None], m[np.clip(jj, 0, cfg.ndivy - 1)][:, ii], 0).T  # [x][y]
    return np.where(bits == 0, ampta, ampvc).astype(np.complex128)


def maskamp(mask2d, cfg: SimConfig, ampta, ampvc, LMAX, MMAX, direct=False) -> np.ndarray:
    """famp[(4L+1) x (4M+1)] at orders -2L..2L, -2M..2M (header.h:1147-1206).

    ``direct=True`` runs the reference's direct per-coefficient DFT
    (``fourier``); the default uses the FFT of the same pattern, which gives the
    same coefficients to rounding (checked in tests on small grids)."""
    FX, FY = cfg.fdivx, cfg.fdivy
    pattern = mask_pattern(mask2d, cfg, ampta, ampvc)
    ls = np.arange(-2 * LMAX, 2 * LMAX + 1)
    ms = np.arange(-2 * MMAX, 2 * MMAX + 1)
    if direct:
        cx, cy = exponential(FX), exponential(FY)
        ftmp = np.empty((FX, len(ms)), np.complex128)
        for i in range(FX):
            for j, m in enumerate(ms):
                ftmp[i, j] = fourier(int(m), pattern[i, :], cy, FY)
        famp = np.empty((len(ls), len(ms)), np.complex128)
        for j in range(len(ms)):
            for i, l in enumerate(ls):
                famp[i, j] = fourier(int(l), ftmp[:, j], cx, FX)
        return famp
    F = np.fft.fft2(pattern) / (float(FX) * float(FY))
    return F[np.ix_(ls % FX, ms % FY)]


# --------------------------------------------------------------------------
# Multilayer cascade (diagonal per order)
# --------------------------------------------------------------------------
def multilayer_s(polar: str, k: float, kxplus, kyplus, kxy2, st: Stack):
    """Diagonals of URUU, URUB (header.h:5-363)."""
    esio2, emo, esi = st.n_sio2 ** 2, st.n_mo ** 2, st.n_si ** 2
    emosi2, eru, erusi = st.n_mosi2 ** 2, st.n_ru ** 2, st.n_rusi ** 2
    al = lambda e: np.sqrt(k * k * e - kxy2 + 0j)
    alsio2, almo, alsi, almosi2, alru, alrusi = al(esio2), al(emo), al(esi), al(emosi2), al(eru), al(erusi)
    kp = kxplus if polar == "X" else kyplus

    def ratio(e_num, e_den):
        return (k - kp * kp / k / e_num) / (k - kp * kp / k / e_den)

    def blocks(cj, al_out, al_in, thick):
        # (UL, UR, BL, BR) of one interface + layer (header.h:68-92 pattern)
        expz = np.exp(1j * al_in * thick)
        a = al_out / al_in
        return (0.5 * (cj + a) / expz, 0.5 * (cj - a) / expz, 0.5 * (cj - a) * expz, 0.5 * (cj + a) * expz)

    TMO = blocks(ratio(emosi2, emo), almosi2, almo, st.d_mo)        # header.h:47-92
    TMOSI = blocks(ratio(emo, emosi2), almo, almosi2, st.d_mosi)    # header.h:94-139
    TSI = blocks(ratio(emosi2, esi), almosi2, alsi, st.d_si)        # header.h:141-186
    TSIMO = blocks(ratio(esi, emosi2), alsi, almosi2, st.d_simo)    # header.h:188-233
    TSIRU = blocks(ratio(esi, erusi), alsi, alrusi, st.d_siru)      # header.h:235-280
    TRU = blocks(ratio(erusi, eru), alrusi, alru, st.d_ru)          # header.h:282-327
    # substrate interface (header.h:294-321): only the UL/BL blocks are used
    cj = ratio(esio2, emo)
    expz = np.exp(1j * almo * st.d_mo)
    a = alsio2 / almo
    UU = 0.5 * (cj + a) / expz
    UB = 0.5 * (cj - a) * expz

    def apply(T, UU, UB):
        UL, UR, BL, BR = T
        return UL * UU + UR * UB, BL * UU + BR * UB

    for i in range(st.nml - 1, -1, -1):  # header.h:326-359
        if i < st.nml - 1:
            UU, UB = apply(TMO, UU, UB)
        UU, UB = apply(TMOSI, UU, UB)
        UU, UB = apply(TSI, UU, UB)
        if i > 0:
            UU, UB = apply(TSIMO, UU, UB)
        else:
            UU, UB = apply(TSIRU, UU, UB)
    URUU, URUB = apply(TRU, UU, UB)  # header.h:361-362
    return URUU, URUB


# --------------------------------------------------------------------------
# Absorber slices
# --------------------------------------------------------------------------
def _toeplitz_index(lidx, midx, LMAX, MMAX):
    LL = lidx[:, None] - lidx[None, :] + 2 * LMAX
    MM = midx[:, None] - midx[None, :] + 2 * MMAX
    return LL, MM


def _build_D(polar, LL, MM, k, kxp, kyp, kxy2, eps1, eta1, zeta1):
    """D(i,j) = k^2 eps - i eta kx+_j (X) / - i zeta ky+_j (Y), minus kxy2 on the
    diagonal (header.h:416-431 / 806-821)."""
    if polar == "X":
        D = k * k * eps1[LL, MM] - 1j * eta1[LL, MM] * kxp[None, :]
    else:
        D = k * k * eps1[LL, MM] - 1j * zeta1[LL, MM] * kyp[None, :]
    D[np.diag_indices_from(D)] -= kxy2
    return D


def _b1(polar, LL, MM, k, kxp, kyp, sigma1, br1):
    """B1 = i (k br1 - kp/k * Sigma br1), Sigma(i,ip) = sigma[..] kp_ip
    (header.h:596-623 / 989-1017)."""
    kp = kxp if polar == "X" else kyp
    Sigma = sigma1[LL, MM] * kp[None, :]
    SUM = Sigma @ br1
    del Sigma
    return 1j * (k * br1 - (kp[:, None] / k) * SUM)


def _t_blocks(Cj, Cjp, al1, al2, dabs1):
    gamma = np.exp(1j * al1 * dabs1)
    A = (al2[None, :] / al1[:, None]) * Cjp
    P = 0.5 * (Cj + A)
    M = 0.5 * (Cj - A)
    return P, M, gamma


def absorber_s0(polar, LL, MM, k, kxp, kyp, kxy2, eps1, eta1, zeta1, sigma1, dabs1,
                al2, B2diag, U2Udiag, U2Bdiag):
    """Bottom slice against the Ru cap (header.h:754-1145)."""
    D = _build_D(polar, LL, MM, k, kxp, kyp, kxy2, eps1, eta1, zeta1)
    w, br1 = np.linalg.eig(D)  # cusolverDnXgeev, right vectors (header.h:837-882)
    del D
    al1 = np.sqrt(w)  # header.h:918-921
    Cjp = np.linalg.inv(br1)  # matinv(FG) with br2 = I (header.h:933-976)
    B1 = _b1(polar, LL, MM, k, kxp, kyp, sigma1, br1)
    Cj = np.linalg.inv(B1) * B2diag[None, :]  # Cj = B1^-1 Bru (header.h:1053-1055)
    P, M, gamma = _t_blocks(Cj, Cjp, al1, al2, dabs1)
    del Cj, Cjp
    g = gamma[:, None]
    # U1U = T1UL U2U + T1UR U2B, U1B = T1BL U2U + T1BR U2B (U2* diagonal; header.h:1085-1144)
    U1U = (P / g) * U2Udiag[None, :] + (M / g) * U2Bdiag[None, :]
    U1B = (M * g) * U2Udiag[None, :] + (P * g) * U2Bdiag[None, :]
    return al1, br1, B1, U1U, U1B


def absorber_s(polar, LL, MM, k, kxp, kyp, kxy2, eps1, eta1, zeta1, sigma1, dabs1,
               al2, br2, B2, U2U, U2B):
    """Upper slice against the previous slice (header.h:365-752)."""
    D = _build_D(polar, LL, MM, k, kxp, kyp, kxy2, eps1, eta1, zeta1)
    w, br1 = np.linalg.eig(D)  # header.h:447-498
    del D
    al1 = np.sqrt(w)
    Cjp = np.linalg.inv(br1) @ br2  # header.h:551-583
    B1 = _b1(polar, LL, MM, k, kxp, kyp, sigma1, br1)
    Cj = np.linalg.inv(B1) @ B2  # header.h:660-663
    P, M, gamma = _t_blocks(Cj, Cjp, al1, al2, dabs1)
    del Cj, Cjp
    g = gamma[:, None]
    U1U = (P / g) @ U2U + (M / g) @ U2B  # header.h:692-720
    U1B = (M * g) @ U2U + (P * g) @ U2B  # header.h:721-751
    return al1, br1, B1, U1U, U1B


def mask_coefficients(masks, cfg: SimConfig, LMAX, MMAX):
    """Per slice eps, sigma (=F[1/eps pattern]), eta, zeta (header.h:1232-1268).

    ``masks``: one mask2d per slice (index 0 = top) or a single mask for all."""
    nabs = cfg.nabs
    if isinstance(masks, np.ndarray):
        masks = [masks] * nabs
    out = []
    i = np.arange(4 * LMAX + 1)
    j = np.arange(4 * MMAX + 1)
    zetal = 1j * 2.0 * PI * (i - 2 * LMAX).astype(np.float64) / cfg.dx
    zetam = 1j * 2.0 * PI * (j - 2 * MMAX).astype(np.float64) / cfg.dy
    for n in range(nabs):
        e = complex(cfg.eabs[n])
        eps = maskamp(masks[n], cfg, e, 1.0, LMAX, MMAX)
        sigma = maskamp(masks[n], cfg, 1.0 / e, 1.0, LMAX, MMAX)
        leps = maskamp(masks[n], cfg, np.log(e), 0.0, LMAX, MMAX)
        eta = zetal[:, None] * leps
        zeta = zetam[None, :] * leps
        out.append((eps, sigma, eta, zeta))
    return out


def amp_s(polar: str, masks, cfg: SimConfig, lidx, midx, LMAX, MMAX, kx0, ky0,
          coefs=None, source_orders=None):
    """The reference operator ``ampS`` (header.h:1208-1466) for one Bloch family.

    Returns ``{(ls, ms): Ax}`` with Ax a length-N complex vector, for every
    source order inside the NA circle (header.h:1394-1397), plus any extra
    ``source_orders`` requested (used by the Abbe loop when a family-shifted
    source order falls outside that circle)."""
    k = cfg.k
    dx, dy = cfg.dx, cfg.dy
    lidx = np.asarray(lidx, np.int64)
    midx = np.asarray(midx, np.int64)
    N = len(lidx)
    if coefs is None:
        coefs = mask_coefficients(masks, cfg, LMAX, MMAX)
    LL, MM = _toeplitz_index(lidx, midx, LMAX, MMAX)
    kxp = kx0 + 2 * PI * lidx / dx  # header.h:1277-1284
    kyp = ky0 + 2 * PI * midx / dy
    kxy2 = kxp ** 2 + kyp ** 2
    with np.errstate(invalid="ignore"):
        klm = np.sqrt(k * k - kxy2).astype(np.complex128)  # real sqrt (quirk 4)
    st = cfg.stack
    URUU, URUB = multilayer_s(polar, k, kxp, kyp, kxy2, st)
    eru = st.n_ru ** 2
    alru = np.sqrt(k * k * eru - kxy2 + 0j)  # header.h:1292-1303
    kp = kxp if polar == "X" else kyp
    Bru = 1j * k - 1j / k / eru * kp ** 2
    nabs = cfg.nabs
    n = nabs - 1
    eps1, sigma1, eta1, zeta1 = coefs[n]
    sigma_bottom = sigma1
    al1, br1, B1, U1U, U1B = absorber_s0(
        polar, LL, MM, k, kxp, kyp, kxy2, eps1, eta1, zeta1, sigma1, float(cfg.dabs[n]),
        alru, Bru, URUU, URUB)
    for n in range(nabs - 2, -1, -1):  # header.h:1337-1353
        eps1, sig_n, eta1, zeta1 = coefs[n]
        sig = sig_n if cfg.refresh_sigma else sigma_bottom
        al1, br1, B1, U1U, U1B = absorber_s(
            polar, LL, MM, k, kxp, kyp, kxy2, eps1, eta1, zeta1, sig, float(cfg.dabs[n]),
            al1, br1, B1, U1U, U1B)
    del B1
    # U0 = T0L U1U + T0R U1B (header.h:1355-1371)
    T0L = klm[:, None] * br1 + br1 * al1[None, :]
    T0R = klm[:, None] * br1 - br1 * al1[None, :]
    U0 = T0L @ U1U + T0R @ U1B
    del T0L, T0R
    U0I = np.linalg.inv(U0)  # header.h:1372-1379
    del U0
    U = (U1U - U1B) @ U0I
    del U0I, U1U, U1B
    FG = ((1.0 / klm)[:, None] * br1 * al1[None, :]) @ U  # header.h:1380-1391
    del U
    lsmaxX, lsmaxY = cfg.lsmaxX, cfg.lsmaxY
    wanted = []
    for ls in range(-lsmaxX, lsmaxX + 1):
        for ms in range(-lsmaxY, lsmaxY + 1):
            if (ls * cfg.mx / dx) ** 2 + (ms * cfg.my / dy) ** 2 <= (cfg.na / cfg.wavelength) ** 2:
                wanted.append((ls, ms))
    if source_orders is not None:
        for o in source_orders:
            if o not in wanted:
                wanted.append(o)
    pos = {(int(a), int(b)): i for i, (a, b) in enumerate(zip(lidx, midx))}
    Ax = {}
    for (ls, ms) in wanted:  # header.h:1394-1465
        kx = kx0 + ls * 2.0 * PI / dx
        ky = ky0 + ms * 2.0 * PI / dy
        kz = np.sqrt(k * k - kx * kx - ky * ky)
        idx = pos.get((ls, ms))
        if idx is None:
            v = np.zeros(N, np.complex128)
        else:
            v = -(FG[:, idx] * (2.0 * kz))
            v[idx] += 1.0
        Ax[(ls, ms)] = v
    return Ax


# --------------------------------------------------------------------------
# Abbe imaging (intensity.cpp)
# --------------------------------------------------------------------------
def rotate(k, MX, MY, px, py, sx0, sy0) -> np.ndarray:
    """3x2 polarisation rotation (intensity.cpp:423-465)."""
    s0 = np.array([sx0, sy0, -np.sqrt(k * k - sx0 * sx0 - sy0 * sy0)])
    p = np.array([px, py, 0.0])
    pp = np.array([MX * px, MY * py, -np.sqrt(k * k - MX * px * MX * px - MY * py * MY * py)])
    ez = np.array([0.0, 0.0, 1.0])
    ezp = ez
    if (px * px + py * py) > 0.00001:
        es = np.cross(p, s0)
        es = es / np.linalg.norm(es)
        esp = np.cross(pp, ezp)
        esp = esp / np.linalg.norm(esp)
        ps0 = p + s0
        ps0 = ps0 / np.linalg.norm(ps0)
        em = np.cross(es, ps0)
        emp = np.cross(esp, pp) / k
    else:
        es = np.cross(ez, s0)
        es = es / np.linalg.norm(es)
        esp = -es
        em = np.cross(es, s0) / k
        emp = np.cross(esp, -ezp)
    return np.outer(esp, es[:2]) + np.outer(emp, em[:2])


def rotate_many(k, MX, MY, px, py, sx0, sy0) -> np.ndarray:
    """``rotate`` for arrays of pupil coordinates px, py: returns [n, 3, 2]."""
    px = np.asarray(px, np.float64)
    py = np.asarray(py, np.float64)
    n = px.shape[0]
    s0 = np.broadcast_to(np.array([sx0, sy0, -np.sqrt(k * k - sx0 * sx0 - sy0 * sy0)]), (n, 3))
    p = np.stack([px, py, np.zeros(n)], -1)
    with np.errstate(invalid="ignore"):
        pp = np.stack([MX * px, MY * py, -np.sqrt(k * k - (MX * px) ** 2 - (MY * py) ** 2)], -1)
    ez = np.broadcast_to(np.array([0.0, 0.0, 1.0]), (n, 3))
    nrm = lambda v: v / np.linalg.norm(v, axis=-1, keepdims=True)
    with np.errstate(invalid="ignore", divide="ignore"):
        es1 = nrm(np.cross(p, s0))
        esp1 = nrm(np.cross(pp, ez))
        em1 = np.cross(es1, nrm(p + s0))
        emp1 = np.cross(esp1, pp) / k
        es2 = nrm(np.cross(ez, s0))
        esp2 = -es2
        em2 = np.cross(es2, s0) / k
        emp2 = np.cross(esp2, -ez)
    big = ((px * px + py * py) > 0.00001)[:, None]
    es, esp = np.where(big, es1, es2), np.where(big, esp1, esp2)
    em, emp = np.where(big, em1, em2), np.where(big, emp1, emp2)
    return esp[:, :, None] * es[:, None, :2] + emp[:, :, None] * em[:, None, :2]


def abbe_family_fields(cfg: SimConfig, polar, Ax, lidx, midx, nsx, nsy, ndivs, pts,
                       linput, minput, z):
    """Pupil-grid fields of one family's source points (intensity.cpp:248-366).
    Returns a list of (Fx, Fy, Fz) XDIV x YDIV spectra, one per source point.

    The reference loops over source points and, inside, over pupil points
    (intensity.cpp:276-331, 333-366); the pupil loop is written here as array
    operations on all pupil points of a source at once (same arithmetic per
    point: the NA test, the order lookup, rotate(), E = ik R A and the phase)."""
    k, dx, dy = cfg.k, cfg.dx, cfg.dy
    MX, MY, NA = cfg.mx, cfg.my, cfg.na
    kx0, ky0 = cfg.kx0, cfg.ky0
    sx0 = 2.0 * PI / dx * nsx / float(ndivs) + kx0
    sy0 = 2.0 * PI / dy * nsy / float(ndivs) + ky0
    XD, YD = cfg.xdiv, cfg.ydiv
    pos = {(int(a), int(b)): i for i, (a, b) in enumerate(zip(lidx, midx))}
    z0 = cfg.z0
    lin = np.asarray(linput, np.int64)
    mn = np.asarray(minput, np.int64)
    px_all = (lin + XD) % XD
    py_all = (mn + YD) % YD
    out = []
    for (l0, m0) in pts:
        kx = sx0 + 2.0 * PI / dx * l0
        ky = sy0 + 2.0 * PI / dy * m0
        F = np.zeros((3, XD, YD), np.complex128)
        kxn = 2.0 * PI / dx * nsx / float(ndivs) + 2.0 * PI / dx * l0 + 2.0 * PI * lin / dx
        kyn = 2.0 * PI / dy * nsy / float(ndivs) + 2.0 * PI / dy * m0 + 2.0 * PI * mn / dy
        inside = (MX * MX * kxn * kxn + MY * MY * kyn * kyn) <= (NA * k) ** 2
        sel = np.nonzero(inside)[0]
        if sel.size:
            try:
                n = np.array([pos[(int(l0 + lin[i]), int(m0 + mn[i]))] for i in sel])
            except KeyError:
                raise ValueError("pupil order outside the order set")
            a = Ax[(l0, m0)][n]
            R = rotate_many(k, MX, MY, kxn[sel], kyn[sel], kx0, ky0)      # [n, 3, 2]
            if polar == "X":
                E = 1j * k * (R[:, :, 0] * (a / np.sqrt(k * k - kx * kx))[:, None])
            else:
                E = 1j * k * (R[:, :, 1] * (a / np.sqrt(k * k - ky * ky))[:, None])
            phase = np.exp(1j * ((kxn[sel] + kx0) ** 2 + (kyn[sel] + ky0) ** 2) / 2.0 / k * z0
                           + 1j * (MX * MX * kxn[sel] ** 2 + MY * MY * kyn[sel] ** 2) / 2.0 / k
                           * float(z))
            F[:, px_all[sel], py_all[sel]] = (E * phase[:, None]).T
        out.append(F)
    return out


def _abbe_family_fields_loop(cfg: SimConfig, polar, Ax, lidx, midx, nsx, nsy, ndivs, pts,
                             linput, minput, z):
    """The same fields with the reference's pupil loop written out point by
    point (intensity.cpp:276-366): the check of the array form."""
    k, dx, dy = cfg.k, cfg.dx, cfg.dy
    MX, MY, NA = cfg.mx, cfg.my, cfg.na
    kx0, ky0 = cfg.kx0, cfg.ky0
    sx0 = 2.0 * PI / dx * nsx / float(ndivs) + kx0
    sy0 = 2.0 * PI / dy * nsy / float(ndivs) + ky0
    XD, YD = cfg.xdiv, cfg.ydiv
    pos = {(int(a), int(b)): i for i, (a, b) in enumerate(zip(lidx, midx))}
    z0 = cfg.z0
    out = []
    for (l0, m0) in pts:
        kx = sx0 + 2.0 * PI / dx * l0
        ky = sy0 + 2.0 * PI / dy * m0
        F = np.zeros((3, XD, YD), np.complex128)
        for i in range(len(linput)):
            kxn = 2.0 * PI / dx * nsx / float(ndivs) + 2.0 * PI / dx * l0 + 2.0 * PI * linput[i] / dx
            kyn = 2.0 * PI / dy * nsy / float(ndivs) + 2.0 * PI / dy * m0 + 2.0 * PI * minput[i] / dy
            if (MX * MX * kxn * kxn + MY * MY * kyn * kyn) <= (NA * k) ** 2:
                n = pos.get((int(l0 + linput[i]), int(m0 + minput[i])))
                if n is None:
                    raise ValueError("pupil order outside the order set")
                a = Ax[(l0, m0)][n]
                if polar == "X":
                    Axv, Ayv = a / np.sqrt(k * k - kx * kx), 0.0
                else:
                    Axv, Ayv = 0.0, a / np.sqrt(k * k - ky * ky)
                R = rotate(k, MX, MY, kxn, kyn, kx0, ky0)
                E = 1j * k * (R[:, 0] * Axv + R[:, 1] * Ayv)
                phase = np.exp(1j * ((kxn + kx0) ** 2 + (kyn + ky0) ** 2) / 2.0 / k * z0
                               + 1j * (MX * MX * kxn * kxn + MY * MY * kyn * kyn) / 2.0 / k * float(z))
                px = (int(linput[i]) + XD) % XD
                py = (int(minput[i]) + YD) % YD
                F[:, px, py] = E * phase
        out.append(F)
    return out


def intensity(cfg: SimConfig, masks, polars=("X",), z=None, return_ax=False, ax_cache=None):
    """Abbe image(s), one XDIV x YDIV array per polarisation (intensity.cpp:35-421).

    ``I[pol][i][j]`` with i = x, j = y, normalised by the total source count."""
    LMAX, MMAX = order_limits(cfg, cfg.order_kind, cfg.cut)
    lidx, midx = order_set(cfg.order_kind, LMAX, MMAX)
    linput, minput, _, _ = pupil_set(cfg)
    ndivs, fams = source(cfg)
    sdivsum = sum(len(v) for v in fams.values())
    coefs = mask_coefficients(masks, cfg, LMAX, MMAX)
    zz = cfg.zlist[0] if z is None else z
    XD, YD = cfg.xdiv, cfg.ydiv
    images = {}
    axs = {}
    for polar in polars:
        isum = np.zeros((XD, YD))
        for (nsx, nsy), pts in fams.items():
            if not pts:
                continue
            sx0 = 2.0 * PI / cfg.dx * nsx / float(ndivs) + cfg.kx0
            sy0 = 2.0 * PI / cfg.dy * nsy / float(ndivs) + cfg.ky0
            key = (polar, nsx, nsy)
            if ax_cache is not None and key in ax_cache:
                Ax = ax_cache[key]
            else:
                Ax = amp_s(polar, masks, cfg, lidx, midx, LMAX, MMAX, sx0, sy0, coefs=coefs,
                           source_orders=pts)
            if return_ax:
                axs[(polar, nsx, nsy)] = Ax
            for F in abbe_family_fields(cfg, polar, Ax, lidx, midx, nsx, nsy, ndivs, pts,
                                        linput, minput, zz):
                f = np.fft.ifft2(F, axes=(1, 2)) * (XD * YD)  # cufft INVERSE, unnormalised
                isum += np.sum(f.real ** 2 + f.imag ** 2, axis=0)
        images[polar] = isum / sdivsum
    if return_ax:
        return images, axs
    return images


def write_emint(path: str, I: np.ndarray) -> None:
    """emint.csv: rows j = YDIV-1..0, each value followed by ',' (intensity.cpp:390-408)."""
    with open(path, "w") as fh:
        for j in range(I.shape[1] - 1, -1, -1):
            fh.write("".join("%.6g," % I[i, j] for i in range(I.shape[0])))
            fh.write("\n")


def read_emint(path) -> np.ndarray:
    rows = []
    fh = open(path) if isinstance(path, str) else path
    for line in fh:
        vals = [float(v) for v in line.strip().split(",") if v != ""]
        if vals:
            rows.append(vals)
    A = np.array(rows)  # A[r][i] = I[i][YDIV-1-r]
    return A[::-1, :].T.copy()


# --------------------------------------------------------------------------
# M3D parameters (m3d.cpp)
# --------------------------------------------------------------------------
def thin_mask_spectrum(mask2d, cfg: SimConfig) -> np.ndarray:
    """fmask[noutX x noutY]: DFT of the 0/1 mask, y flipped (m3d.cpp:287-327)."""
    lpx, lpy = cfg.lpmaxX, cfg.lpmaxY
    m = mask2d.reshape(cfg.ndivy, cfg.ndivx)
    idiv = int(1.0 / cfg.delta + 0.000001)
    jj = cfg.ndivy - 1 - np.arange(cfg.ndivy) + cfg.yflip_offset
    inside = (jj >= 0) & (jj < cfg.ndivy)
    # mask(i,j) = mask2d[NDIVX*(NDIVY-1-j)+i] (with the same optional offset)
    mask = np.where(inside[:, None], m[np.clip(jj, 0, cfg.ndivy - 1)], 0).T.astype(np.float64)
    pattern = np.repeat(np.repeat(mask, idiv, axis=0), idiv, axis=1)
    FX, FY = pattern.shape
    F = np.fft.fft2(pattern) / (float(FX) * float(FY))
    ls = np.arange(-lpx, lpx + 1)
    ms = np.arange(-lpy, lpy + 1)
    return F[np.ix_(ls % FX, ms % FY)]


def m3d(cfg: SimConfig, mask2d, polar="X", Ax_wide=None):
    """M3D parameters a0, ax, ay per pupil order (m3d.cpp:197-558).

    Returns dict with 'a0' (ninput), 'ax', 'ay' (xinput subset), 'linput',
    'minput', 'xinput'."""
    k, dx, dy = cfg.k, cfg.dx, cfg.dy
    MX, MY, NA, lam = cfg.mx, cfg.my, cfg.na, cfg.wavelength
    kx0, ky0 = cfg.kx0, cfg.ky0
    lsx, lsy, lpx, lpy = cfg.lsmaxX, cfg.lsmaxY, cfg.lpmaxX, cfg.lpmaxY
    # narrow (ellipse, cut 1.5) and wide (diamond, cut 6) sets (m3d.cpp:97-157);
    # the ampS calls use the wide LMAX/MMAX for both (m3d.cpp:131-139,221)
    Ln, Mn = order_limits(cfg, "ellipse", 1.5)
    lidxp, midxp = order_set("ellipse", Ln, Mn)
    if cfg.order_kind == "box":
        LMAX, MMAX = cfg.lbox, cfg.mbox
    else:
        LMAX, MMAX = order_limits(cfg, cfg.order_kind, cfg.cut)
    lidx, midx = order_set(cfg.order_kind, LMAX, MMAX)
    linput, minput, xinput, _ = pupil_set(cfg)
    ones = np.ones_like(mask2d)
    zeros = np.zeros_like(mask2d)
    Axvc = amp_s(polar, ones, cfg, lidxp, midxp, LMAX, MMAX, kx0, ky0)   # m3d.cpp:214-225
    Axab = amp_s(polar, zeros, cfg, lidxp, midxp, LMAX, MMAX, kx0, ky0)  # m3d.cpp:227-238
    posp = {(int(a), int(b)): i for i, (a, b) in enumerate(zip(lidxp, midxp))}
    insrc = lambda is_, js: _in_na(cfg, is_ - lsx, js - lsy)
    vcxx = np.full((2 * lsx + 1, 2 * lsy + 1), np.nan + 0j)
    abxx = np.full((2 * lsx + 1, 2 * lsy + 1), np.nan + 0j)
    for (ls, ms), v in Axvc.items():  # m3d.cpp:240-258
        i = posp.get((ls, ms))
        if i is not None:
            vcxx[ls + lsx, ms + lsy] = v[i]
            abxx[ls + lsx, ms + lsy] = Axab[(ls, ms)][i]
    Ax = Ax_wide if Ax_wide is not None else amp_s(
        polar, mask2d, cfg, lidx, midx, LMAX, MMAX, kx0, ky0)  # m3d.cpp:279-285
    fmask = thin_mask_spectrum(mask2d, cfg)
    noutX, noutY = 2 * lpx + 1, 2 * lpy + 1
    # thin-mask amplitudes of the centre source (m3d.cpp:329-356); kxs=kx0, kys=ky0
    kxp = 2.0 * PI * (np.arange(noutX) - lpx) / dx
    kyp = 2.0 * PI * (np.arange(noutY) - lpy) / dy
    phasesp = np.exp(-1j * (kx0 * kxp[:, None] + kxp[:, None] ** 2 / 2.0
                            + ky0 * kyp[None, :] + kyp[None, :] ** 2 / 2.0) / k * cfg.z0)
    vc_c, ab_c = vcxx[lsx, lsy], abxx[lsx, lsy]
    famp_c = fmask * phasesp * (vc_c - ab_c)
    famp_c[lpx, lpy] += ab_c
    phase_c = vc_c / abs(vc_c)
    famp_c = famp_c / phase_c  # fampxx[lsmaxX][lsmaxY] / phasexx (m3d.cpp:384-394)
    pos = {(int(a), int(b)): i for i, (a, b) in enumerate(zip(lidx, midx))}
    ninput = len(linput)
    a0 = np.zeros(ninput, np.complex128)
    ax = np.zeros(ninput, np.complex128)
    ay = np.zeros(ninput, np.complex128)
    for n in range(ninput):  # m3d.cpp:426-467
        ip, jp = linput[n] + lpx, minput[n] + lpy
        lp, mp = float(ip - lpx), float(jp - lpy)
        xxf1 = xxfx = xxfy = 0j
        c1 = cx = cy = cx2 = cy2 = cxy = 0.0
        for is_ in range(2 * lsx + 1):
            for js in range(2 * lsy + 1):
                if insrc(is_, js) and _in_na(cfg, ip - lpx + is_ - lsx, jp - lpy + js - lsy):
                    l_abs = int(ip - lpx + is_ - lsx)
                    m_abs = int(jp - lpy + js - lsy)
                    amp = Ax[(is_ - lsx, js - lsy)][pos[(l_abs, m_abs)]]
                    phase = vcxx[is_, js] / abs(vcxx[is_, js])
                    f = amp / phase - famp_c[ip, jp]  # dampxx (m3d.cpp:406-424)
                    ls_ = is_ - lsx + lp / 2.0
                    ms_ = js - lsy + mp / 2.0
                    xxf1 += f
                    xxfx += ls_ * f
                    xxfy += ms_ * f
                    c1 += 1
                    cx += ls_
                    cy += ms_
                    cx2 += ls_ * ls_
                    cy2 += ms_ * ms_
                    cxy += ls_ * ms_
        if xinput[n] == 1:
            cd = c1 * cx2 * cy2 + 2.0 * cx * cxy * cy - c1 * cxy * cxy - cx2 * cy * cy - cy2 * cx * cx
            a0[n] = 1.0 / cd * ((cx2 * cy2 - cxy * cxy) * xxf1 + (-cx * cy2 + cy * cxy) * xxfx + (cx * cxy - cy * cx2) * xxfy)
            ax[n] = 1.0 / cd * ((-cx * cy2 + cy * cxy) * xxf1 + (c1 * cy2 - cy * cy) * xxfx + (-c1 * cxy + cx * cy) * xxfy)
            ay[n] = 1.0 / cd * ((cx * cxy - cy * cx2) * xxf1 + (-c1 * cxy + cx * cy) * xxfx + (c1 * cx2 - cx * cx) * xxfy)
        else:
            a0[n] = xxf1 / c1
    sel = xinput == 1
    return {"a0": a0, "ax": ax[sel], "ay": ay[sel], "linput": linput, "minput": minput,
            "xinput": xinput, "Ax": Ax, "vcxx": vcxx, "abxx": abxx}


# --------------------------------------------------------------------------
# Linear Abbe model from the M3D parameters (cnn/intensity/linear/linear.py)
# --------------------------------------------------------------------------
def linear_sources(cfg: SimConfig, mesh_deg: float = 0.2):
    """Source points of the linear model (linear.py:47-96): a square grid of
    step kmesh = k * mesh (radians) in the mask-side source plane, l outer and
    m inner, kept where the illumination holds at (MX skx, MY sky).  Returns
    the shifts dsx, dsy (rad/nm) in that order."""
    k, NA = cfg.k, cfg.na
    kmesh = k * mesh_deg * (PI / 180.0)
    l0max = int(k * NA / cfg.mx * cfg.sigma1 / kmesh) + 1
    m0max = int(k * NA / cfg.my * cfg.sigma1 / kmesh) + 1
    r1, r2 = k * NA * cfg.sigma1, k * NA * cfg.sigma2
    t = np.tan(PI * cfg.openangle / 180.0 / 2.0)
    dsx, dsy = [], []
    for l in range(-l0max, l0max + 1):
        for m in range(-m0max, m0max + 1):
            skx, sky = l * kmesh, m * kmesh
            xo, yo = skx * cfg.mx, sky * cfg.my
            r = np.sqrt(xo * xo + yo * yo)
            if cfg.illum_type == 0:
                ok = xo * xo + yo * yo <= r1 * r1
            elif cfg.illum_type == 1:
                ok = r2 <= r <= r1
            elif cfg.illum_type == 2:
                ok = r2 <= r <= r1 and abs(yo) <= abs(xo) * t
            else:
                ok = r2 <= r <= r1 and abs(xo) <= abs(yo) * t
            if ok:
                dsx.append(skx)
                dsy.append(sky)
    return np.array(dsx), np.array(dsy)


def linear_amplitudes(cfg: SimConfig, mask2d, a0, ax, ay, ampvc, ampab, dsx, dsy,
                      linput, minput):
    """Per source s and pupil point i, without the 1/sqrt(k^2 - kx^2) factor
    (linear.py:120-172): the thin-mask amplitude
        famp = (ab delta + (vc - ab) F_vac) phaseX phaseY / phase0
    and the linear one  famp + a0 + ax (ls + lp/2) + ay (ms + mp/2)  with
    ls = dsx / (2 pi / dx).  a0, ax, ay: one value per pupil point (ax, ay zero
    where the fit has no slope).  Returns (A_linear, A_thin), [S][ncut]."""
    k, dx, dy, z0 = cfg.k, cfg.dx, cfg.dy, cfg.z0
    lpx, lpy = cfg.lpmaxX, cfg.lpmaxY
    fvac = thin_mask_spectrum(mask2d, cfg)
    lp = np.asarray(linput, np.float64)
    mp = np.asarray(minput, np.float64)
    f = (ampvc - ampab) * fvac[np.asarray(linput) + lpx, np.asarray(minput) + lpy]
    f = f + np.where((lp == 0) & (mp == 0), ampab, 0.0)
    kxp = 2.0 * PI * lp / dx
    kyp = 2.0 * PI * mp / dy
    ph = np.exp(-1j * (cfg.kx0 * kxp + kxp * kxp / 2.0) / k * z0) * \
        np.exp(-1j * (cfg.ky0 * kyp + kyp * kyp / 2.0) / k * z0)
    famp = f * ph / (ampvc / abs(ampvc))
    ls = np.asarray(dsx)[:, None] / (2.0 * PI / dx)
    ms = np.asarray(dsy)[:, None] / (2.0 * PI / dy)
    alin = famp[None, :] + np.asarray(a0)[None, :] + np.asarray(ax)[None, :] * (ls + lp / 2.0) + \
        np.asarray(ay)[None, :] * (ms + mp / 2.0)
    return alin, np.broadcast_to(famp, alin.shape)


def linear_image(cfg: SimConfig, amp, dsx, dsy, linput, minput, z: float = 0.0,
                 obscuration: float = 0.0) -> np.ndarray:
    """Abbe image of per-(source, pupil point) amplitudes on the linear model's
    source grid (linear.py:11-43 with the high-NA E-field of
    elitho/electro_field.py:45-76, X polarisation): E = i k R(:, 0) A /
    sqrt(k^2 - kx^2) with kx = kx0 + dsx, zero outside obscuration <= |p|/(NA k)
    <= 1; phase, scatter, unnormalised inverse DFT, |E|^2 summed over sources
    and divided by their count.  Returns I[x][y]."""
    k, dx, dy = cfg.k, cfg.dx, cfg.dy
    MX, MY, NA = cfg.mx, cfg.my, cfg.na
    kx0, ky0, z0 = cfg.kx0, cfg.ky0, cfg.z0
    XD, YD = cfg.xdiv, cfg.ydiv
    S = len(dsx)
    lin = np.asarray(linput, np.int64)
    mn = np.asarray(minput, np.int64)
    isum = np.zeros((XD, YD))
    for s in range(S):
        kx = kx0 + dsx[s]
        kxn = dsx[s] + 2.0 * PI * lin / dx
        kyn = dsy[s] + 2.0 * PI * mn / dy
        p2 = MX * MX * kxn * kxn + MY * MY * kyn * kyn
        ok = np.nonzero((p2 <= (NA * k) ** 2) & (p2 >= (NA * k * obscuration) ** 2))[0]
        F = np.zeros((3, XD, YD), np.complex128)
        R = rotate_many(k, MX, MY, kxn[ok], kyn[ok], kx0, ky0)[:, :, 0]  # [n_ok, 3]
        phase = np.exp(1j * ((kxn[ok] + kx0) ** 2 + (kyn[ok] + ky0) ** 2) / (2.0 * k) * z0
                       + 1j * p2[ok] / (2.0 * k) * z)
        E = 1j * k * R * (amp[s, ok] * phase / np.sqrt(k * k - kx * kx))[:, None]
        F[:, lin[ok] % XD, mn[ok] % YD] = E.T
        f = np.fft.ifft2(F, axes=(1, 2)) * (XD * YD)
        isum += np.sum(f.real ** 2 + f.imag ** 2, axis=0) / S
    return isum


# --------------------------------------------------------------------------
# STCC-SOCS imaging (cnn/intensity/stccsocs/eigenfunction.py, socs.py)
# --------------------------------------------------------------------------
def socs_tcc(cfg: SimConfig, z: float = 0.0, mesh_deg: float = 0.2):
    """The three transmission cross-coefficient matrices (eigenfunction.py:5-124)
    on the pupil points: TCC_w = sum_c P_c diag(w k^2/(k^2 - (kx0+dsx)^2)) P_c^H / S
    for w = 1, dsx, dsy, with P_c[i, s] = phase(i, s) R(c, 0) (zero outside the
    pupil NA) over the linear model's source grid.  Returns (s0, sx, sy)."""
    k, dx, dy, MX, MY, NA = cfg.k, cfg.dx, cfg.dy, cfg.mx, cfg.my, cfg.na
    kx0, ky0, z0 = cfg.kx0, cfg.ky0, cfg.z0
    dsx, dsy = linear_sources(cfg, mesh_deg)
    lin, mn, _, _ = pupil_set(cfg)
    S, n = len(dsx), len(lin)
    ksx = (2 * PI / dx * lin)[:, None] + dsx[None, :]
    ksy = (2 * PI / dy * mn)[:, None] + dsy[None, :]
    p2 = MX * MX * ksx * ksx + MY * MY * ksy * ksy
    phase = np.exp(1j * ((ksx + kx0) ** 2 + (ksy + ky0) ** 2) / 2.0 / k * z0
                   + 1j * p2 / 2.0 / k * z) * (p2 <= (k * NA) ** 2)
    R = rotate_many(k, MX, MY, ksx.ravel(), ksy.ravel(), kx0, ky0)[:, :, 0].reshape(n, S, 3)
    w0 = k * k / (k * k - (kx0 + dsx) ** 2)
    out = []
    for wt in (w0, dsx * w0, dsy * w0):
        t = np.zeros((n, n), np.complex128)
        for c in range(3):
            P = phase * R[:, :, c]
            t += P @ (np.conj(P).T * wt[:, None])
        out.append(t / S)
    return tuple(out)


def socs_padding(cfg: SimConfig):
    """(index of the (0,0) pupil point, its extra copies) of the reference's TCC:
    eigenfunction.py:60-66 takes ncut = len(linput) from find_valid_pupil_points,
    whose arrays have the wide order count (rounded diamond, cut 6) with the
    unused tail left at (0,0) -- so the TCC runs over the pupil points plus
    Nrange - ncut copies of the (0,0) point."""
    lin, mn, _, _ = pupil_set(cfg)
    L_, M_ = order_limits(cfg, "diamond", 6.0)
    nrange = len(order_set("diamond", L_, M_)[0])
    z = int(np.nonzero((lin == 0) & (mn == 0))[0][0])
    return z, nrange - len(lin)


def socs_eigen(tcc, z=None, copies=0):
    """Eigenpairs of one TCC sorted by |alpha|, largest first, ties in
    ascending-eigenvalue order (eigenfunction.py:125-163).  Returns (alpha,
    phi) with phi[m] the m-th eigenvector on the pupil points.

    With ``copies`` > 0, the eigenpairs of the padded TCC M T M^H (point z
    repeated ``copies`` more times) restricted to the pupil points: its nonzero
    spectrum is that of D^1/2 T D^1/2 with D = I + copies e_z e_z^T, and the
    eigenvector on the pupil points is y with y_z / sqrt(1 + copies)."""
    t = np.array(tcc, copy=True)
    if copies:
        sc = np.sqrt(1.0 + copies)
        t[z, :] *= sc
        t[:, z] *= sc
    w, v = np.linalg.eigh(t)
    if copies:
        v[z, :] /= sc
    order = np.argsort(-np.abs(w), kind="stable")
    return w[order], v[:, order].T.copy()


def socs_image(cfg: SimConfig, mask2d, a0, ax, ay, ampvc, ampab, eig, nsocs: int = 100,
               nsocsxy: int = 20, nout: int = 64) -> np.ndarray:
    """SOCS image from the M3D parameters (socs.py:12-151): the kernels of the
    three TCCs weighted by the pupil amplitudes on an nout x nout grid, the
    |.|^2 sum (plus the first-order cross terms of ax, ay), and Fourier
    interpolation to XDIV x YDIV.  a0, ax, ay: one value per pupil point.
    ``eig`` = (alpha_s0, phi_s0, alpha_sx, phi_sx, alpha_sy, phi_sy).
    Returns the real part (what socs.py writes)."""
    a_s0, p_s0, a_sx, p_sx, a_sy, p_sy = eig
    dx, dy = cfg.dx, cfg.dy
    lin, mn, _, _ = pupil_set(cfg)
    famp = linear_amplitudes(cfg, mask2d, np.zeros(len(lin)), np.zeros(len(lin)),
                             np.zeros(len(lin)), ampvc, ampab, [0.0], [0.0], lin, mn)[1][0]
    a0, ax, ay = np.asarray(a0), np.asarray(ax), np.asarray(ay)
    A0 = famp + a0
    Ax = ax * dx / (2 * PI)
    Ay = ay * dy / (2 * PI)
    Axy = ax * lin / 2.0 + ay * mn / 2.0
    px, py = lin % nout, mn % nout

    def field(v):
        g = np.zeros((nout, nout), np.complex128)
        g[px, py] = v
        return np.fft.ifft2(g) * nout * nout

    small = np.zeros((nout, nout))
    for m in range(nsocs):
        f0 = field(A0 * p_s0[m])
        small += a_s0[m] * np.abs(f0) ** 2
        if m < nsocsxy:
            f0x, fx = field(A0 * p_sx[m]), field(Ax * p_sx[m])
            f0y, fy = field(A0 * p_sy[m]), field(Ay * p_sy[m])
            fxy = field(Axy * p_s0[m])
            small += 2 * a_sx[m] * (f0x * np.conj(fx)).real + 2 * a_sy[m] * (f0y * np.conj(fy)).real \
                + 2 * a_s0[m] * (f0 * np.conj(fxy)).real
    spec = np.fft.fft2(small) / nout / nout
    XD, YD = cfg.xdiv, cfg.ydiv
    big = np.zeros((XD, YD), np.complex128)
    h = nout // 2
    for i in range(-h, h):
        for j in range(-h, h):
            big[i, j] = spec[i, j]
    return (np.fft.ifft2(big) * XD * YD).real


def expand_xinput(values, xinput):
    """Slopes stored for the xinput points only (inputxx.csv rows 3-6) -> one
    value per pupil point, zero elsewhere."""
    out = np.zeros(len(xinput), np.complex128)
    out[np.asarray(xinput) == 1] = values
    return out


def write_inputxx(path: str, res) -> None:
    """Six rows: Re a0, Im a0, Re ax, Im ax, Re ay, Im ay (m3d.cpp:468-558)."""
    rows = [res["a0"].real, res["a0"].imag, res["ax"].real, res["ax"].imag,
            res["ay"].real, res["ay"].imag]
    with open(path, "w") as fh:
        for r in rows:
            fh.write("".join("%.6g," % v for v in r))
            fh.write("\n")


def read_inputxx(path):
    rows = []
    fh = open(path) if isinstance(path, str) else path
    for line in fh:
        rows.append(np.array([float(v) for v in line.strip().split(",") if v != ""]))
    return {"a0": rows[0] + 1j * rows[1], "ax": rows[2] + 1j * rows[3], "ay": rows[4] + 1j * rows[5]}


def write_inputlm(path: str, res) -> None:
    with open(path, "w") as fh:
        for l, m, x in zip(res["linput"], res["minput"], res["xinput"]):
            fh.write("%d,%d,%d\n" % (l, m, x))
