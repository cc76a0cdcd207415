"""Simulation configuration: the constants of the reference drivers, made parameters.

``SimConfig()`` with no arguments is the reference configuration of
``cnn/intensity/abbe/intensity.cpp:44-146`` and ``cnn/intensity/m3d/m3d.cpp:34-157``
(NA 0.33, 4x, 2048 nm clip on a 2048^2 grid, annular 0.55-0.9, Ta absorber
60 nm, 40 Mo/Si periods with interlayers, Ru cap).  ``presets`` holds the
workloads the library is measured on.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field, replace
from typing import Optional, Sequence, Tuple

PI = math.atan(1.0) * 4.0


@dataclass(frozen=True)
class Stack:
    """Multilayer refractive indices and thicknesses (header.h:1217-1230)."""

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


@dataclass(frozen=True)
class SimConfig:
    ndivx: int = 2048
    ndivy: int = 2048
    delta: float = 1.0
    wavelength: float = 13.5
    theta0: float = -6.0
    azimuth: float = 0.0
    na: float = 0.33
    mx: int = 4
    my: int = 4
    illum_type: int = 1          # 0 conventional, 1 annular, 2 X dipole, 3 Y dipole
    sigma1: float = 0.9
    sigma2: float = 0.55
    openangle: float = 90.0
    sigmadiv: float = 0.5
    ndivs: Optional[int] = None  # Bloch families per axis; None = reference rule
    max_sources: Optional[int] = None
    eabs: Tuple[complex, ...] = (complex(0.9567, 0.0343) ** 2,)
    dabs: Tuple[float, ...] = (60.0,)
    z0_offset: float = 42.0
    stack: Stack = field(default_factory=Stack)
    refresh_sigma: bool = False
    order_kind: str = "diamond"  # "diamond" | "ellipse" | "box"
    cut: float = 6.0
    lbox: int = 0
    mbox: int = 0
    z: int = 0                   # defocus (nm)
    # y flip of the mask onto the Fourier grid: pattern row j reads mask row
    # ndivy-1-j + yflip_offset (header.h:1159 has 0); rows outside the mask are
    # absorber.  1 reproduces the revision that wrote the reference's golden
    # emint.csv / inputxx.csv, whose flip is one row off.
    yflip_offset: int = 0
    # central obscuration of the pupil as a fraction of NA, used by the linear
    # model's E-field (elitho/const.py co: 0.2 at NA 0.55, 0 at NA 0.33)
    obscuration: float = 0.0

    # --- derived quantities (intensity.cpp:52-146) ---
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
        return self.k * math.sin(PI / 180.0 * self.theta0) * math.cos(PI / 180.0 * phi0)

    @property
    def ky0(self) -> float:
        phi0 = 90.0 - self.azimuth
        return self.k * math.sin(PI / 180.0 * self.theta0) * math.sin(PI / 180.0 * phi0)

    @property
    def z0(self) -> float:
        return float(sum(self.dabs)) + self.z0_offset

    @property
    def nabs(self) -> int:
        return len(self.eabs)

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

    def order_limits(self, kind: Optional[str] = None, cut: Optional[float] = None) -> Tuple[int, int]:
        kind = self.order_kind if kind is None else kind
        cut = self.cut if cut is None else cut
        if kind == "box":
            return self.lbox, self.mbox
        cutx = self.na / self.mx * cut
        cuty = self.na / self.my * cut
        return int(cutx * self.dx / self.wavelength), int(cuty * self.dy / self.wavelength)

    def with_(self, **kw) -> "SimConfig":
        return replace(self, **kw)


# Materials of the measured workloads (n + ik of the workload definitions).
_BASE_STACK = Stack(n_mo=0.924 + 0.0064j, n_si=0.999 + 0.0018j, n_ru=0.886 + 0.017j,
                    d_mo=2.8, d_si=4.2, d_mosi=0.0, d_simo=0.0, d_siru=0.0, d_ru=2.5)
_ABS = complex(0.95, 0.031) ** 2


def sidewall_slices(total: float = 60.0, n: int = 8) -> Tuple[Tuple[complex, ...], Tuple[float, ...]]:
    return tuple([_ABS] * n), tuple([total / n] * n)


def preset(name: str) -> SimConfig:
    """Named workloads.

    reference: the golden configuration of the reference drivers.
    small:     256 nm clip, NA 0.55 anamorphic 4x/8x, 11x11 orders, 1 slice,
               annular 0.5-0.9 with 2x2 Bloch families (26 source points).
    batched:   1024 nm clip, 31x31 orders, 200-point annular source (2x2
               families, first 200 points), both polarisations.
    mixed:     'small' with the absorber as 8 slices of 7.5 nm.
    large:     2048 nm clip, 41x41 orders, 8 slices.
    """
    high = dict(na=0.55, mx=4, my=8, theta0=-6.0, stack=_BASE_STACK, eabs=(_ABS,), dabs=(60.0,),
                sigma1=0.9, sigma2=0.5, illum_type=1, order_kind="box")
    if name == "reference":
        return SimConfig()
    if name == "small":
        return SimConfig(ndivx=256, ndivy=256, lbox=5, mbox=5, ndivs=2, **high)
    if name == "batched":
        return SimConfig(ndivx=1024, ndivy=1024, lbox=15, mbox=15, ndivs=2, max_sources=200, **high)
    if name == "mixed":
        e, d = sidewall_slices()
        h = dict(high, eabs=e, dabs=d)
        return SimConfig(ndivx=256, ndivy=256, lbox=5, mbox=5, ndivs=2, **h)
    if name == "large":
        e, d = sidewall_slices()
        h = dict(high, eabs=e, dabs=d)
        return SimConfig(ndivx=2048, ndivy=2048, lbox=20, mbox=20, ndivs=1, **h)
    raise KeyError(name)
