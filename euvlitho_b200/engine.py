"""Host driver: the loops of intensity.cpp / m3d.cpp over the batched C ABI.

A :class:`Plan` owns, per configuration, the resident device tables (order set,
pupil set, per-family source lists and Abbe E-field factors, the mask-independent
vacuum/absorber solves of m3d) and a workspace.  Its methods enqueue work on the
current torch CUDA stream through ``libeuvl_b200.so``; device buffers are torch
tensors.  Nothing here computes physics on the host.

Entry points mirror the reference:
  * :meth:`Plan.amp`        -- ampS (header.h:1208-1466), batched over units;
  * :meth:`Plan.intensity`  -- the Abbe image of intensity.cpp (emint.csv);
  * :meth:`Plan.m3d`        -- the M3D parameters of m3d.cpp (inputxx.csv).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np
import torch

from . import _lib as L
from .config import PI, SimConfig
from . import tables as T

_POL = {"X": 0, "Y": 1}


def _ptr(t: Optional[torch.Tensor]) -> Optional[int]:
    return None if t is None else t.data_ptr()


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


def stack_struct(cfg: SimConfig) -> L.Stack:
    s = cfg.stack
    return L.Stack(L.c64.of(s.n_mo ** 2), L.c64.of(s.n_si ** 2), L.c64.of(s.n_ru ** 2),
                   L.c64.of(s.n_mosi2 ** 2), L.c64.of(s.n_rusi ** 2), L.c64.of(s.n_sio2 ** 2),
                   s.d_mo, s.d_mosi, s.d_si, s.d_simo, s.d_siru, s.d_ru, s.nml)


@dataclass
class OrderSet:
    kind: str
    lmax: int
    mmax: int
    lidx: np.ndarray
    midx: np.ndarray

    @property
    def n(self) -> int:
        return len(self.lidx)


class Workspace:
    """Grow-only device scratch buffer."""

    def __init__(self, device):
        self.device = device
        self.buf: Optional[torch.Tensor] = None

    def get(self, nbytes: int) -> torch.Tensor:
        nbytes = max(int(nbytes), 256)
        if self.buf is None or self.buf.numel() < nbytes:
            self.buf = None
            self.buf = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
        return self.buf


class Plan:
    """Resident tables and workspace for one configuration."""

    def __init__(self, cfg: SimConfig, device: Optional[torch.device] = None,
                 precision: str = "fp64", pols: Sequence[str] = ("X",)):
        L.lib()  # fail loudly if the library is missing
        if not torch.cuda.is_available():
            raise RuntimeError("euvlitho_b200 needs a CUDA device")
        self.cfg = cfg
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.precision = {"fp64": L.EUV_PREC_FP64, "mixed": L.EUV_PREC_MIXED}[precision]
        self.pols = tuple(pols)
        for p in self.pols:
            if p not in _POL:
                raise ValueError("polarisation must be 'X' or 'Y'")
        if cfg.nabs > L.EUV_MAX_SLICES:
            raise ValueError("at most %d absorber slices" % L.EUV_MAX_SLICES)
        if cfg.fdivx % cfg.ndivx or cfg.fdivy % cfg.ndivy:
            raise ValueError("the Fourier grid must refine the mask grid by an integer factor")
        lmax, mmax = cfg.order_limits()
        li, mi = T.order_set(cfg.order_kind, lmax, mmax)
        self.orders = OrderSet(cfg.order_kind, lmax, mmax, li, mi)
        self.pos = T.order_positions(li, mi)
        kxy_max = (abs(cfg.kx0) + 2 * PI * (lmax + 1) / cfg.dx) ** 2 + \
                  (abs(cfg.ky0) + 2 * PI * (mmax + 1) / cfg.dy) ** 2
        if kxy_max >= cfg.k ** 2:
            # header.h:1283 takes a real square root: the reference gives NaN there
            raise ValueError("order set reaches evanescent orders (|k_xy| >= k); the reference "
                             "computes NaN for them; reduce the order cut")
        self.linput, self.minput, self.xinput, _ = T.pupil_set(cfg)
        self.ncut = len(self.linput)
        self.ndivs, self.fams = T.sources(cfg)
        self.sdivsum = sum(len(f.pts) for f in self.fams)
        if self.sdivsum == 0:
            raise ValueError("the illumination has no source point")
        self.work = Workspace(self.device)
        dev = self.device
        self._t_l = torch.tensor(li, dtype=torch.int32, device=dev)
        self._t_m = torch.tensor(mi, dtype=torch.int32, device=dev)
        self._abbe_tables = None
        self._m3d_tables = None
        self._linear_tables = None
        self._uniform = None
        self._batches: Dict[Tuple[int, int], "IntensityBatch"] = {}
        # device status word of the plan's own ampS calls (EUV_STATUS_* bits)
        self.status = torch.zeros(1, dtype=torch.int32, device=dev)

    # ------------------------------------------------------------ helpers
    def _i32(self, a) -> torch.Tensor:
        return torch.tensor(np.asarray(a, np.int32), dtype=torch.int32, device=self.device)

    def _f64(self, a) -> torch.Tensor:
        return torch.tensor(np.asarray(a, np.float64), dtype=torch.float64, device=self.device)

    def _c128(self, a) -> torch.Tensor:
        return torch.tensor(np.asarray(a, np.complex128), dtype=torch.complex128, device=self.device)

    def mask_bytes(self) -> int:
        return self.cfg.ndivx * self.cfg.ndivy // 8

    def as_mask_tensor(self, masks) -> torch.Tensor:
        """uint8 device tensor [clips, slices_or_1, nbytes] of packed mask.bin bits."""
        nb = self.mask_bytes()
        if isinstance(masks, (bytes, bytearray)):
            masks = np.frombuffer(masks, np.uint8)
        t = torch.as_tensor(masks) if not isinstance(masks, torch.Tensor) else masks
        if t.dtype != torch.uint8:
            raise TypeError("masks must be packed uint8 (mask.bin layout)")
        if t.dim() == 1:
            t = t.view(1, 1, -1)
        elif t.dim() == 2:
            t = t.view(t.shape[0], 1, -1)
        if t.shape[-1] != nb:
            raise ValueError("each mask must be %d bytes (ndivx*ndivy/8)" % nb)
        if t.shape[1] not in (1, self.cfg.nabs):
            raise ValueError("give one mask per clip or one per absorber slice")
        return t.to(self.device, non_blocking=True).contiguous()

    # ------------------------------------------------------------ spectra
    def spectra(self, masks: torch.Tensor, lh: int, mh: int, select_vacuum: int = 0,
                per_slice: bool = True) -> torch.Tensor:
        """Indicator spectra [clips, slices, (2lh+1)(2mh+1)] (maskamp, header.h:1147-1206)."""
        cfg = self.cfg
        n_clips, n_m, nb = masks.shape
        flat = masks.reshape(n_clips * n_m, nb)
        out = torch.empty((n_clips * n_m, (2 * lh + 1) * (2 * mh + 1)), dtype=torch.complex128,
                          device=self.device)
        wb = L.lib().euv_mask_spectrum_workspace_bytes(n_clips * n_m, cfg.ndivx, cfg.ndivy,
                                                      cfg.fdivx, cfg.fdivy, lh, mh)
        ws = self.work.get(wb)
        L.call("euv_mask_spectrum", flat.data_ptr(), n_clips * n_m, cfg.ndivx, cfg.ndivy,
               cfg.fdivx, cfg.fdivy, lh, mh, select_vacuum, cfg.yflip_offset, out.data_ptr(), ws.data_ptr(),
               ws.numel(), _stream())
        out = out.view(n_clips, n_m, -1)
        if per_slice and n_m == 1 and cfg.nabs > 1:
            out = out.expand(n_clips, cfg.nabs, out.shape[-1]).contiguous()
        return out

    # ------------------------------------------------------------ ampS
    def amp_desc(self, orders: OrderSet, t_l, t_m, kx0, ky0, polar, spec_of_unit,
                 src_order, src_2kz, keep, status: Optional[torch.Tensor] = None) -> L.AmpDesc:
        cfg = self.cfg
        d = L.AmpDesc()
        d.n_orders = orders.n
        d.lmax, d.mmax = orders.lmax, orders.mmax
        d.d_lindex, d.d_mindex = _ptr(t_l), _ptr(t_m)
        d.dx, d.dy, d.k = cfg.dx, cfg.dy, cfg.k
        d.n_slices = cfg.nabs
        for n in range(cfg.nabs):
            d.eabs[n] = L.c64.of(cfg.eabs[n])
            d.dabs[n] = float(cfg.dabs[n])
        d.refresh_sigma = 1 if cfg.refresh_sigma else 0
        d.stack = stack_struct(cfg)
        d.n_units = int(kx0.numel())
        d.d_kx0, d.d_ky0, d.d_polar, d.d_spec = _ptr(kx0), _ptr(ky0), _ptr(polar), _ptr(spec_of_unit)
        d.n_src = int(src_order.shape[1])
        d.d_src_order, d.d_src_2kz = _ptr(src_order), _ptr(src_2kz)
        d.precision = self.precision
        d.m_max = 0
        d.k0_max = float(max(kx0.abs().max().item(), ky0.abs().max().item()))
        d.d_status = _ptr(self.status if status is None else status)
        keep.extend([t_l, t_m, kx0, ky0, polar, spec_of_unit, src_order, src_2kz])
        return d

    def check(self) -> None:
        """Raise EuvError if a device wait of the plan's own calls gave up, an LU
        met a zero pivot or the double-angle steps were clamped (synchronises
        the current stream; clears the word)."""
        _check_word(self.status, "Plan")

    def run_amp(self, desc: L.AmpDesc, spectra: torch.Tensor, ax: torch.Tensor) -> None:
        wb = L.lib().euv_amp_workspace_bytes(C.byref(desc))
        if wb == 0:
            raise ValueError("invalid ampS descriptor")
        ws = self.work.get(wb)
        L.call("euv_amp", C.byref(desc), spectra.data_ptr(), ax.data_ptr(), ws.data_ptr(),
               ws.numel(), _stream())

    def src_columns(self, kx0: float, ky0: float, srcs: Sequence[Tuple[int, int]], n_src: int):
        """Order index and 2 kz of each source column (header.h:1396-1409)."""
        cfg = self.cfg
        order = np.full(n_src, -1, np.int32)
        kz2 = np.zeros(n_src, np.float64)
        for s, (ls, ms) in enumerate(srcs):
            kx = kx0 + ls * 2.0 * PI / cfg.dx
            ky = ky0 + ms * 2.0 * PI / cfg.dy
            kz2[s] = 2.0 * math.sqrt(cfg.k * cfg.k - kx * kx - ky * ky)
            order[s] = self.pos.get((ls, ms), -1)
        return order, kz2

    def amp(self, masks, polar: str = "X", kx0: Optional[float] = None,
            ky0: Optional[float] = None) -> Tuple[torch.Tensor, List[Tuple[int, int]]]:
        """ampS for every clip at one incidence: Ax[clip][s][N] for the NA-circle
        source orders (header.h:1394-1465); returns (Ax, source order list)."""
        cfg = self.cfg
        m = self.as_mask_tensor(masks)
        nc = m.shape[0]
        kx0 = cfg.kx0 if kx0 is None else kx0
        ky0 = cfg.ky0 if ky0 is None else ky0
        srcs = T.na_sources(cfg)
        o, kz2 = self.src_columns(kx0, ky0, srcs, len(srcs))
        spec = self.spectra(m, 2 * self.orders.lmax, 2 * self.orders.mmax)
        keep: list = []
        desc = self.amp_desc(self.orders, self._t_l, self._t_m, self._f64([kx0] * nc),
                             self._f64([ky0] * nc), self._i32([_POL[polar]] * nc),
                             self._i32(range(nc)), self._i32(np.tile(o, (nc, 1))),
                             self._f64(np.tile(kz2, (nc, 1))), keep)
        ax = torch.empty((nc, len(srcs), self.orders.n), dtype=torch.complex128, device=self.device)
        self.run_amp(desc, spec, ax)
        self.check()
        return ax, srcs

    # ------------------------------------------------------------ Abbe
    def abbe_tables(self, n_src: Optional[int] = None):
        """Resident Abbe tables of every (polarisation, family), with ``n_src``
        source slots per table (default: the largest family; more pads with
        empty slots, so that batches of different configurations share one
        source stride)."""
        need = max(len(f.pts) for f in self.fams)
        n_src = need if n_src is None else int(n_src)
        if n_src < need:
            raise ValueError("n_src %d is below the largest family (%d)" % (n_src, need))
        if self._abbe_tables is None:
            self._abbe_tables = {}
        if n_src in self._abbe_tables:
            return self._abbe_tables[n_src]
        cfg = self.cfg
        coefs, nidxs, kx0s, ky0s, orders, kz2s, pols, nsrcs = [], [], [], [], [], [], [], []
        for p in self.pols:
            for f in self.fams:
                c, n = T.abbe_table(cfg, p, self.ndivs, f, self.pos, self.linput, self.minput, n_src)
                coefs.append(c)
                nidxs.append(n)
                sx0, sy0 = T.family_offsets(cfg, self.ndivs, f)
                o, kz2 = self.src_columns(sx0, sy0, f.pts, n_src)
                if np.any(o[: len(f.pts)] < 0):
                    raise ValueError("a source order of family %s is outside the order set" %
                                     ((f.nsx, f.nsy),))
                kx0s.append(sx0)
                ky0s.append(sy0)
                orders.append(o)
                kz2s.append(kz2)
                pols.append(_POL[p])
                nsrcs.append(len(f.pts))
        tb = dict(
            n_src=n_src,
            coef=self._c128(np.stack(coefs)),
            nidx=self._i32(np.stack(nidxs)),
            px=self._i32(self.linput), py=self._i32(self.minput),
            row_start=self._i32(T.row_starts(self.linput, cfg.lpmaxX)),
            kx0=np.array(kx0s), ky0=np.array(ky0s), order=np.stack(orders), kz2=np.stack(kz2s),
            pol=np.array(pols, np.int32), nsrc=np.array(nsrcs, np.int32),
        )
        self._abbe_tables[n_src] = tb
        return tb

    def intensity_batch(self, n_clips: int, n_mask_slices: int = 1) -> "IntensityBatch":
        """Prepared launch for n_clips clips (cached per shape)."""
        key = (n_clips, n_mask_slices)
        b = self._batches.get(key)
        if b is None:
            b = IntensityBatch(self, n_clips, n_mask_slices)
            self._batches[key] = b
        return b

    def intensity(self, masks, plain: bool = False) -> torch.Tensor:
        """Abbe images [clips, pols, XDIV, YDIV] (intensity.cpp:219-408), I[x][y].

        ``masks``: packed uint8 [clips, bytes] or [clips, slices, bytes], on the
        host or the device.  ``plain=True`` runs one (clip, family,
        polarisation) unit at a time (the unbatched FP64 form).  The result is
        a new tensor."""
        m = self.as_mask_tensor(masks)
        b = self.intensity_batch(m.shape[0], m.shape[1])
        b.masks.copy_(m)
        if plain:
            b.run_plain()
        else:
            b.run()
        b.check()
        return b.image.clone()

    # ------------------------------------------------------------ M3D
    def uniform_solves(self):
        """Mask-independent narrow solves (m3d.cpp:214-238): Ax of the all-vacuum
        and all-absorber masks on the narrow order set (ellipse, cut 1.5,
        m3d.cpp:107-129) for the NA-circle source orders (cached)."""
        if self._uniform is not None:
            return self._uniform
        cfg = self.cfg
        ln, mn = cfg.order_limits("ellipse", 1.5)
        nli, nmi = T.order_set("ellipse", ln, mn)
        narrow = OrderSet("ellipse", ln, mn, nli, nmi)
        npos = T.order_positions(nli, nmi)
        srcs = T.na_sources(cfg)
        ns = len(srcs)
        src_nn = np.array([npos.get(s, -1) for s in srcs], np.int32)
        if np.any(src_nn < 0):
            raise ValueError("narrow order set misses a source order")
        nb = self.mask_bytes()
        uni = torch.stack([torch.full((nb,), 255, dtype=torch.uint8),
                           torch.zeros(nb, dtype=torch.uint8)]).to(self.device)
        spec = self.spectra(uni.view(2, 1, nb), 2 * ln, 2 * mn)
        kz2 = []
        for (ls, ms) in srcs:
            kx = cfg.kx0 + ls * 2.0 * PI / cfg.dx
            ky = cfg.ky0 + ms * 2.0 * PI / cfg.dy
            kz2.append(2.0 * math.sqrt(cfg.k ** 2 - kx * kx - ky * ky))
        t_nl, t_nm = self._i32(nli), self._i32(nmi)
        keep: list = []
        desc = self.amp_desc(narrow, t_nl, t_nm, self._f64([cfg.kx0] * 2), self._f64([cfg.ky0] * 2),
                             self._i32([_POL[self.pols[0]]] * 2), self._i32([0, 1]),
                             self._i32(np.tile(src_nn, (2, 1))), self._f64(np.tile(kz2, (2, 1))), keep)
        axn = torch.empty((2, ns, narrow.n), dtype=torch.complex128, device=self.device)
        self.run_amp(desc, spec, axn)
        self.check()
        self._uniform = dict(narrow=narrow, srcs=srcs, ns=ns, src_nn=src_nn,
                             s_center=srcs.index((0, 0)), n00=npos[(0, 0)],
                             ax_vc=axn[0].contiguous(), ax_ab=axn[1].contiguous(), keep=keep)
        return self._uniform

    def m3d_tables(self):
        if self._m3d_tables is not None:
            return self._m3d_tables
        u = self.uniform_solves()
        srcs = u["srcs"]
        ns = u["ns"]
        pair = np.full((self.ncut, ns), -1, np.int32)
        for n in range(self.ncut):
            lp, mp = int(self.linput[n]), int(self.minput[n])
            for s, (ls, ms) in enumerate(srcs):
                if T.in_na(self.cfg, ls + lp, ms + mp):
                    o = self.pos.get((ls + lp, ms + mp))
                    if o is None:
                        raise ValueError("order set misses pupil order %s" % ((ls + lp, ms + mp),))
                    pair[n, s] = o
        tb = dict(
            narrow=u["narrow"], srcs=srcs, ns=ns,
            src_l=self._i32([s[0] for s in srcs]), src_m=self._i32([s[1] for s in srcs]),
            src_nn=self._i32(u["src_nn"]), s_center=u["s_center"],
            ax_vc=u["ax_vc"], ax_ab=u["ax_ab"],
            lin=self._i32(self.linput), min=self._i32(self.minput), xin=self._i32(self.xinput),
            pair=self._i32(pair), keep=u["keep"],
        )
        self._m3d_tables = tb
        return tb

    def m3d(self, masks) -> Dict[str, torch.Tensor]:
        """M3D parameters per clip (m3d.cpp:197-558): 'a0' [clips, ninput] and
        'ax', 'ay' [clips, ninput] (zero where xinput == 0)."""
        cfg = self.cfg
        tb = self.m3d_tables()
        m = self.as_mask_tensor(masks)
        ax_wide, srcs = self.amp(m, polar=self.pols[0])
        fmask = self.spectra(m[:, :1], cfg.lpmaxX, cfg.lpmaxY, select_vacuum=1, per_slice=False)
        nc = m.shape[0]
        a0 = torch.empty((nc, self.ncut), dtype=torch.complex128, device=self.device)
        axp = torch.empty_like(a0)
        ayp = torch.empty_like(a0)
        d = L.M3dDesc()
        d.n_clips, d.n_src, d.ninput, d.n_order = nc, tb["ns"], self.ncut, self.orders.n
        d.n_order_narrow = tb["narrow"].n
        d.lpx, d.lpy = cfg.lpmaxX, cfg.lpmaxY
        d.k, d.dx, d.dy, d.z0, d.kx0, d.ky0 = cfg.k, cfg.dx, cfg.dy, cfg.z0, cfg.kx0, cfg.ky0
        d.s_center = tb["s_center"]
        d.d_src_l, d.d_src_m, d.d_src_nidx_narrow = _ptr(tb["src_l"]), _ptr(tb["src_m"]), _ptr(tb["src_nn"])
        d.d_ax_vc, d.d_ax_ab = _ptr(tb["ax_vc"]), _ptr(tb["ax_ab"])
        d.d_lin, d.d_min, d.d_xin, d.d_pair_order = _ptr(tb["lin"]), _ptr(tb["min"]), _ptr(tb["xin"]), _ptr(tb["pair"])
        L.call("euv_m3d_fit", C.byref(d), ax_wide.data_ptr(), fmask.data_ptr(), a0.data_ptr(),
               axp.data_ptr(), ayp.data_ptr(), _stream())
        self._last_keep = (ax_wide, fmask)
        return {"a0": a0, "ax": axp, "ay": ayp, "Ax": ax_wide, "srcs": srcs}


    # ------------------------------------------------------------ linear model
    def linear_tables(self, mesh_deg: float = 0.2):
        """Resident tables of the linear model (linear.py:47-172): source grid,
        E-field factors and identity pupil indices for the fused Abbe kernel,
        and the specular amplitudes of the all-vacuum / all-absorber masks
        (the narrow solves of the M3D tables)."""
        tb = self._linear_tables
        if tb is not None and tb["mesh"] == mesh_deg:
            return tb
        cfg = self.cfg
        dsx, dsy = T.linear_sources(cfg, mesh_deg)
        if len(dsx) == 0:
            raise ValueError("the linear model's source grid is empty (mesh %g deg)" % mesh_deg)
        coef, nidx = T.linear_abbe_table(cfg, dsx, dsy, self.linput, self.minput)
        u = self.uniform_solves()
        sc, n00 = u["s_center"], u["n00"]
        vc = complex(u["ax_vc"][sc, n00].item())
        ab = complex(u["ax_ab"][sc, n00].item())
        tb = dict(mesh=mesh_deg, n_src=len(dsx), dsx=dsx, dsy=dsy,
                  coef=self._c128(coef[None]), nidx=self._i32(nidx[None]),
                  ls=self._f64(dsx * cfg.dx / (2.0 * PI)), ms=self._f64(dsy * cfg.dy / (2.0 * PI)),
                  lp=self._i32(self.linput), mp=self._i32(self.minput),
                  row_start=self._i32(T.row_starts(self.linput, cfg.lpmaxX)),
                  amp_vc=vc, amp_ab=ab)
        self._linear_tables = tb
        return tb

    def linear(self, masks, a0, ax, ay, mesh_deg: float = 0.2, thin: bool = True):
        """Linear Abbe images from the M3D parameters (linear.py:45-188).

        ``a0``, ``ax``, ``ay``: [clips, ncut] complex, one value per pupil point
        (``Plan.m3d`` returns them so; ``io.read_inputxx`` + ``expand_xinput``
        for a file).  Returns (intlinear [clips, XDIV, YDIV], intft or None):
        the M3D-corrected image and, with ``thin``, the thin-mask one."""
        cfg = self.cfg
        tb = self.linear_tables(mesh_deg)
        m = self.as_mask_tensor(masks)
        nc, S, ncut = m.shape[0], tb["n_src"], self.ncut
        par = []
        for v in (a0, ax, ay):
            t = torch.as_tensor(v).to(self.device, torch.complex128).reshape(nc, ncut).contiguous()
            par.append(t)
        fvac = self.spectra(m[:, :1], cfg.lpmaxX, cfg.lpmaxY, select_vacuum=1, per_slice=False)
        d = L.LinearDesc()
        d.n_clips, d.n_src, d.ncut, d.lpx, d.lpy = nc, S, ncut, cfg.lpmaxX, cfg.lpmaxY
        d.d_lp, d.d_mp, d.d_ls, d.d_ms = _ptr(tb["lp"]), _ptr(tb["mp"]), _ptr(tb["ls"]), _ptr(tb["ms"])
        d.k, d.dx, d.dy, d.kx0, d.ky0, d.z0 = cfg.k, cfg.dx, cfg.dy, cfg.kx0, cfg.ky0, cfg.z0
        d.amp_vc, d.amp_ab = L.c64.of(tb["amp_vc"]), L.c64.of(tb["amp_ab"])
        amp = torch.empty((nc, S, ncut), dtype=torch.complex128, device=self.device)
        t_tab = self._i32([0] * nc)
        t_img = self._i32(range(nc))
        t_ns = self._i32([S] * nc)
        inv_w = self._f64([1.0 / S] * nc)
        ad = L.AbbeDesc()
        ad.xdiv, ad.ydiv, ad.lpx, ad.lpy = cfg.xdiv, cfg.ydiv, cfg.lpmaxX, cfg.lpmaxY
        ad.ncut, ad.n_units, ad.n_src, ad.n_order = ncut, nc, S, ncut
        ad.d_coef, ad.d_nidx = _ptr(tb["coef"]), _ptr(tb["nidx"])
        ad.d_px, ad.d_py, ad.d_row_start = _ptr(tb["lp"]), _ptr(tb["mp"]), _ptr(tb["row_start"])
        ad.d_tab_of_unit, ad.d_img_of_unit, ad.d_nsrc_of_unit = _ptr(t_tab), _ptr(t_img), _ptr(t_ns)
        ad.n_images, ad.d_inv_weight = nc, _ptr(inv_w)
        out = []
        for with_m3d in ((True, False) if thin else (True,)):
            ptrs = [t.data_ptr() for t in par] if with_m3d else [None, None, None]
            L.call("euv_linear_amp", C.byref(d), fvac.data_ptr(), *ptrs, amp.data_ptr(), _stream())
            img = torch.zeros((nc, cfg.xdiv, cfg.ydiv), dtype=torch.float64, device=self.device)
            L.call("euv_abbe", C.byref(ad), amp.data_ptr(), img.data_ptr(), _stream())
            out.append(img)
        self._last_keep = (fvac, amp, t_tab, t_img, t_ns, inv_w, par)
        return out[0], (out[1] if thin else None)


    # ------------------------------------------------------------ STCC-SOCS
    def socs_padding(self) -> Tuple[int, int]:
        """(index of the (0,0) pupil point, its extra copies) in the reference's
        TCC: eigenfunction.py:60-66 takes ncut = len(linput) from
        find_valid_pupil_points, whose arrays have the wide order count (rounded
        diamond, cut 6) with the unused tail at (0,0)."""
        L_, M_ = self.cfg.order_limits("diamond", 6.0)
        nrange = len(T.order_set("diamond", L_, M_)[0])
        z = int(np.nonzero((self.linput == 0) & (self.minput == 0))[0][0])
        return z, max(0, nrange - self.ncut)

    def socs_tables(self, z: Optional[float] = None, nsocs: int = 100, nsocsxy: int = 20,
                    nout: int = 64, mesh_deg: float = 0.2, max_sweeps: int = 30,
                    reference_padding: bool = True):
        """Resident SOCS kernels (eigenfunction.py:5-163): the three TCC
        matrices over the linear model's source grid as device GEMMs, their
        eigenpairs by the device Jacobi solver (euv_heev), the nsocs / nsocsxy
        kernels of largest |alpha|, and the DFT / interpolation tables.

        ``reference_padding``: reproduce the reference's TCC, which repeats the
        (0,0) pupil point d more times (``socs_padding``).  Its nonzero spectrum
        is that of D^1/2 T D^1/2, D = I + d e_z e_z^T, and its eigenvectors on the
        pupil points are those of D^1/2 T D^1/2 with component z divided by
        sqrt(1 + d): the same result from an ncut-size problem."""
        cfg = self.cfg
        z = float(cfg.z if z is None else z)
        key = (z, nsocs, nsocsxy, nout, mesh_deg, reference_padding)
        tb = getattr(self, "_socs_tables", None)
        if tb is not None and tb["key"] == key:
            return tb
        n = self.ncut
        if nsocs > n or nsocsxy > nsocs:
            raise ValueError("need nsocsxy <= nsocs <= %d pupil points" % n)
        dsx, dsy = T.linear_sources(cfg, mesh_deg)
        S = len(dsx)
        P, w0 = T.socs_phase(cfg, z, dsx, dsy, self.linput, self.minput)
        pall = np.concatenate([P[0], P[1], P[2]], axis=1)                 # [n, 3S]
        dev = self.device
        a_cm = torch.from_numpy(np.ascontiguousarray(pall.T)).to(dev)      # column-major n x 3S
        lib = L.lib()
        wb = lib.euv_heev_workspace_bytes(n)
        hw = torch.empty(wb, dtype=torch.uint8, device=dev)
        iz, pad_copies = self.socs_padding() if reference_padding else (0, 0)
        pad_scale = math.sqrt(1.0 + pad_copies)
        out = {}
        for name, wt in (("s0", np.ones(S)), ("sx", dsx), ("sy", dsy)):
            q = torch.from_numpy(np.conj(pall) * np.tile(wt * w0, 3)[None, :]).to(dev)  # col-major 3S x n
            tcc = torch.empty((n, n), dtype=torch.complex128, device=dev)
            L.call("euv_zgemm", n, n, 3 * S, L.c64.of(1.0 / S), None, a_cm.data_ptr(), n, 0,
                   q.data_ptr(), 3 * S, 0, L.c64.of(0), tcc.data_ptr(), n, 0, L.c64.of(0), 1,
                   None, 0, _stream())
            del q
            if pad_copies:  # column-major: tcc[j][i] = TCC(i, j)
                tcc[iz, :] *= pad_scale
                tcc[:, iz] *= pad_scale
            w = torch.empty(n, dtype=torch.float64, device=dev)
            v = torch.empty((n, n), dtype=torch.complex128, device=dev)
            L.call("euv_heev", n, tcc.data_ptr(), n, w.data_ptr(), v.data_ptr(), n, max_sweeps,
                   1e-14, hw.data_ptr(), wb, self.status.data_ptr(), _stream())
            self.check()
            if pad_copies:  # v[j][i] = component i of eigenvector j
                v[:, iz] /= pad_scale
            wh = w.cpu().numpy()
            order = np.lexsort((wh, -np.abs(wh)))   # |alpha| descending, ties ascending
            keep = nsocs if name == "s0" else nsocsxy
            idx = torch.from_numpy(order[:max(keep, 1)].astype(np.int64)).to(dev)
            out["alpha_" + name] = self._f64(wh[order[:max(keep, 1)]])
            out["phi_" + name] = v.index_select(0, idx).contiguous()  # row m = eigenvector m
            out["eig_" + name] = wh[order]
        E, Kx, Ky = T.socs_interp_tables(nout, cfg.xdiv, cfg.ydiv)
        u = self.uniform_solves()
        tb = dict(key=key, nsocs=nsocs, nsocsxy=nsocsxy, nout=nout, n_src=S,
                  e=self._c128(E), kxT=self._c128(Kx), ky=self._c128(np.ascontiguousarray(Ky.T)),
                  lp=self._i32(self.linput), mp=self._i32(self.minput),
                  amp_vc=complex(u["ax_vc"][u["s_center"], u["n00"]].item()),
                  amp_ab=complex(u["ax_ab"][u["s_center"], u["n00"]].item()), **out)
        self._socs_tables = tb
        return tb

    def socs(self, masks, a0, ax, ay, z: Optional[float] = None, **kw) -> torch.Tensor:
        """STCC-SOCS images [clips, XDIV, YDIV] from the M3D parameters
        (socs.py:12-151; a0, ax, ay as for ``linear``)."""
        cfg = self.cfg
        tb = self.socs_tables(z, **kw)
        m = self.as_mask_tensor(masks)
        nc, ncut = m.shape[0], self.ncut
        par = [torch.as_tensor(v).to(self.device, torch.complex128).reshape(nc, ncut).contiguous()
               for v in (a0, ax, ay)]
        fvac = self.spectra(m[:, :1], cfg.lpmaxX, cfg.lpmaxY, select_vacuum=1, per_slice=False)
        d = L.SocsDesc()
        d.n_clips, d.ncut, d.lpx, d.lpy = nc, ncut, cfg.lpmaxX, cfg.lpmaxY
        d.nsocs, d.nsocsxy, d.nout, d.xdiv, d.ydiv = tb["nsocs"], tb["nsocsxy"], tb["nout"], cfg.xdiv, cfg.ydiv
        d.d_lp, d.d_mp = _ptr(tb["lp"]), _ptr(tb["mp"])
        d.k, d.dx, d.dy, d.kx0, d.ky0, d.z0 = cfg.k, cfg.dx, cfg.dy, cfg.kx0, cfg.ky0, cfg.z0
        d.amp_vc, d.amp_ab = L.c64.of(tb["amp_vc"]), L.c64.of(tb["amp_ab"])
        d.d_phi_s0, d.d_phi_sx, d.d_phi_sy = _ptr(tb["phi_s0"]), _ptr(tb["phi_sx"]), _ptr(tb["phi_sy"])
        d.d_alpha_s0, d.d_alpha_sx, d.d_alpha_sy = (_ptr(tb["alpha_s0"]), _ptr(tb["alpha_sx"]),
                                                    _ptr(tb["alpha_sy"]))
        d.d_e, d.d_kxT, d.d_ky = _ptr(tb["e"]), _ptr(tb["kxT"]), _ptr(tb["ky"])
        wb = L.lib().euv_socs_workspace_bytes(C.byref(d))
        ws = self.work.get(wb)
        img = torch.empty((nc, cfg.xdiv, cfg.ydiv), dtype=torch.complex128, device=self.device)
        L.call("euv_socs_image", C.byref(d), fvac.data_ptr(), par[0].data_ptr(), par[1].data_ptr(),
               par[2].data_ptr(), img.data_ptr(), ws.data_ptr(), ws.numel(), _stream())
        return img.real


def unit_range(n_units: int, world: int, rank: int) -> Tuple[int, int]:
    """Units [u0, u1) of ``rank`` when a step's (clip, polarisation, family)
    units are split over ``world`` GPUs: contiguous ranges whose sizes differ
    by at most one.  The units are independent until the image sum, so each
    rank solves and images its range and one all-reduce (sum) of the images
    finishes the step."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank %d of world %d" % (rank, world))
    base, extra = divmod(n_units, world)
    u0 = rank * base + min(rank, extra)
    return u0, u0 + base + (1 if rank < extra else 0)


def _check_word(word: torch.Tensor, where: str) -> None:
    bits = int(word.item())
    if bits:
        word.zero_()
        L.check_status(where, bits)


class IntensityBatch:
    """Static buffers and descriptors for the Abbe images of ``n_clips`` clips.

    ``run()`` enqueues, on the current stream, the mask spectra, the batched
    ampS of every (clip, polarisation, family) unit and the fused Abbe kernel;
    it allocates nothing and never synchronises, so it can be captured in a
    CUDA graph (``capture()`` / ``replay()``).  ``run_plain()`` is the
    unbatched FP64 form: one unit per ampS call."""

    def __init__(self, plan: Plan, n_clips: int, n_mask_slices: int = 1,
                 max_units: Optional[int] = None, own_work: bool = True):
        cfg = plan.cfg
        self.plan = plan
        self.n_clips = nc = n_clips
        dev = plan.device
        tb = plan.abbe_tables()
        self.tb = tb
        ntab = len(tb["pol"])
        self.U = U = nc * ntab
        tab = np.tile(np.arange(ntab, dtype=np.int32), nc)
        clip = np.repeat(np.arange(nc, dtype=np.int32), ntab)
        npol = len(plan.pols)
        nf = len(plan.fams)
        img = clip * npol + (tab // nf)
        self.masks = torch.zeros((nc, n_mask_slices, plan.mask_bytes()), dtype=torch.uint8, device=dev)
        L_, M_ = plan.orders.lmax, plan.orders.mmax
        self.lh, self.mh = 2 * L_, 2 * M_
        self.spec_raw = torch.empty((nc * n_mask_slices, (2 * self.lh + 1) * (2 * self.mh + 1)),
                                    dtype=torch.complex128, device=dev)
        self.spec = self.spec_raw.view(nc, n_mask_slices, -1) if (n_mask_slices == cfg.nabs or cfg.nabs == 1) \
            else torch.empty((nc, cfg.nabs, self.spec_raw.shape[1]), dtype=torch.complex128, device=dev)
        self.ax = torch.empty((U, tb["n_src"], plan.orders.n), dtype=torch.complex128, device=dev)
        self.image = torch.zeros((nc, npol, cfg.xdiv, cfg.ydiv), dtype=torch.float64, device=dev)
        self.keep: list = []
        self.t_kx0 = plan._f64(tb["kx0"][tab])
        self.t_ky0 = plan._f64(tb["ky0"][tab])
        self.t_pol = plan._i32(tb["pol"][tab])
        self.t_clip = plan._i32(clip)
        self.t_order = plan._i32(tb["order"][tab])
        self.t_kz2 = plan._f64(tb["kz2"][tab])
        # device status word of this batch's ampS calls (EUV_STATUS_* bits)
        self.status = torch.zeros(1, dtype=torch.int32, device=dev)
        self.desc = plan.amp_desc(plan.orders, plan._t_l, plan._t_m, self.t_kx0, self.t_ky0,
                                  self.t_pol, self.t_clip, self.t_order, self.t_kz2, self.keep,
                                  status=self.status)
        self.t_tab, self.t_img, self.t_ns = plan._i32(tab), plan._i32(img), plan._i32(tb["nsrc"][tab])
        self.inv_w = plan._f64([1.0 / plan.sdivsum] * (nc * npol))
        ad = L.AbbeDesc()
        ad.xdiv, ad.ydiv = cfg.xdiv, cfg.ydiv
        ad.lpx, ad.lpy = cfg.lpmaxX, cfg.lpmaxY
        ad.ncut, ad.n_units, ad.n_src, ad.n_order = plan.ncut, U, tb["n_src"], plan.orders.n
        ad.d_coef, ad.d_nidx = _ptr(tb["coef"]), _ptr(tb["nidx"])
        ad.d_px, ad.d_py, ad.d_row_start = _ptr(tb["px"]), _ptr(tb["py"]), _ptr(tb["row_start"])
        ad.d_tab_of_unit, ad.d_img_of_unit = _ptr(self.t_tab), _ptr(self.t_img)
        ad.d_nsrc_of_unit = _ptr(self.t_ns)
        ad.n_images = nc * npol
        ad.d_inv_weight = _ptr(self.inv_w)
        ad.precision = plan.precision  # mixed: the Abbe DFT sums in FP32
        self.adesc = ad
        lib = L.lib()
        self.spec_bytes = lib.euv_mask_spectrum_workspace_bytes(nc * n_mask_slices, cfg.ndivx, cfg.ndivy,
                                                               cfg.fdivx, cfg.fdivy, self.lh, self.mh)
        self.max_units = U if max_units is None else max(1, min(int(max_units), U))
        self.chunks = self._unit_descs(self.max_units)
        self.amp_bytes = max(wb for _, _, _, wb in self.chunks)
        if self.amp_bytes == 0:
            raise ValueError("invalid ampS descriptor")
        self.work_bytes = max(self.spec_bytes, self.amp_bytes)
        self.work = (torch.empty(self.work_bytes, dtype=torch.uint8, device=dev) if own_work
                     else None)
        self.graph: Optional[torch.cuda.CUDAGraph] = None
        self._plain = None
        self._ranges: Dict[Tuple[int, int], tuple] = {}

    def _unit_descs(self, size: int, first: int = 0):
        """ampS / Abbe descriptors for units [u0, u0+size), u0 = first, first +
        size, ...: pointer offsets into the batch's per-unit tables (the C ABI
        takes plain pointers)."""
        out = []
        ns = self.ax.shape[1] * self.ax.shape[2]
        nsrc = self.desc.n_src
        for u0 in range(first, self.U, size):
            n = min(size, self.U - u0)
            d = L.AmpDesc.from_buffer_copy(self.desc)
            d.n_units = n
            d.d_kx0 = self.t_kx0.data_ptr() + 8 * u0
            d.d_ky0 = self.t_ky0.data_ptr() + 8 * u0
            d.d_polar = self.t_pol.data_ptr() + 4 * u0
            d.d_spec = self.t_clip.data_ptr() + 4 * u0
            d.d_src_order = self.t_order.data_ptr() + 4 * u0 * nsrc
            d.d_src_2kz = self.t_kz2.data_ptr() + 8 * u0 * nsrc
            a = L.AbbeDesc.from_buffer_copy(self.adesc)
            a.n_units = n
            a.d_tab_of_unit = self.t_tab.data_ptr() + 4 * u0
            a.d_img_of_unit = self.t_img.data_ptr() + 4 * u0
            a.d_nsrc_of_unit = self.t_ns.data_ptr() + 4 * u0
            wb = L.lib().euv_amp_workspace_bytes(C.byref(d))
            out.append((d, a, self.ax.data_ptr() + 16 * ns * u0, wb))
        return out

    def _spectra(self, work: torch.Tensor) -> None:
        cfg = self.plan.cfg
        n = self.masks.shape[0] * self.masks.shape[1]
        L.call("euv_mask_spectrum", self.masks.data_ptr(), n, cfg.ndivx, cfg.ndivy, cfg.fdivx,
               cfg.fdivy, self.lh, self.mh, 0, cfg.yflip_offset, self.spec_raw.data_ptr(),
               work.data_ptr(), work.numel(), _stream())
        if self.spec.data_ptr() != self.spec_raw.data_ptr():
            self.spec.copy_(self.spec_raw.view(self.n_clips, 1, -1).expand_as(self.spec))

    def run(self, work: Optional[torch.Tensor] = None) -> None:
        """Enqueue spectra, batched ampS (in chunks of max_units units sharing
        one workspace) and the fused Abbe kernel on the current stream.
        ``work``: a workspace of at least ``work_bytes`` (default: the batch's own)."""
        w = self.work if work is None else work
        self._spectra(w)
        for d, _, axp, _ in self.chunks:
            L.call("euv_amp", C.byref(d), self.spec.data_ptr(), axp, w.data_ptr(), w.numel(),
                   _stream())
        self.image.zero_()
        L.call("euv_abbe", C.byref(self.adesc), self.ax.data_ptr(), self.image.data_ptr(), _stream())

    def run_units(self, u0: int, u1: int, work: Optional[torch.Tensor] = None) -> None:
        """Spectra, ampS and Abbe of the units [u0, u1) only: the image holds
        their partial sum (a rank's share of a step split over GPUs; the
        all-reduce of the partial images is the caller's)."""
        if not 0 <= u0 <= u1 <= self.U:
            raise ValueError("unit range [%d, %d) outside [0, %d)" % (u0, u1, self.U))
        w = self.work if work is None else work
        self._spectra(w)
        self.image.zero_()
        if u1 == u0:
            return
        key = (u0, u1)
        if key not in self._ranges:
            self._ranges[key] = self._unit_descs(u1 - u0, first=u0)[0]
        d, a, axp, wb = self._ranges[key]
        L.call("euv_amp", C.byref(d), self.spec.data_ptr(), axp, w.data_ptr(), w.numel(), _stream())
        L.call("euv_abbe", C.byref(a), axp, self.image.data_ptr(), _stream())

    def run_plain(self, work: Optional[torch.Tensor] = None) -> None:
        """The unbatched FP64 form: every unit solved and imaged on its own."""
        if self._plain is None:
            self._plain = self._unit_descs(1)
        w = self.work if work is None else work
        self._spectra(w)
        self.image.zero_()
        for d, a, axp, wb in self._plain:
            L.call("euv_amp", C.byref(d), self.spec.data_ptr(), axp, w.data_ptr(), wb, _stream())
            L.call("euv_abbe", C.byref(a), axp, self.image.data_ptr(), _stream())

    def check(self) -> None:
        """Raise EuvError if the device status word of the batch's runs since
        the last check has a bit set (synchronises the current stream)."""
        _check_word(self.status, "IntensityBatch")

    def capture(self) -> None:
        """Capture run() into a CUDA graph (call run() once before, outside capture)."""
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            with torch.cuda.graph(g, stream=s):
                self.run()
        torch.cuda.current_stream().wait_stream(s)
        self.graph = g

    def replay(self) -> None:
        if self.graph is None:
            self.run()
        else:
            self.graph.replay()
