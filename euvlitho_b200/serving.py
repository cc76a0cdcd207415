"""Continuous-batching server for Abbe images of mask clips.

Requests are single clips with their own optical configuration (period, order
box, source points, polarisations).  The server keeps, per configuration, a
resident :class:`~euvlitho_b200.engine.Plan` (order/pupil/source tables and the
Abbe E-field factors).  One host loop:

* admits the requests that have arrived into per-group queues: a group is an
  order box with its polarisations, so requests of different periods and
  source counts share a queue (``GroupKey``);
* whenever one of ``n_streams`` stream slots is idle, launches the group of
  the oldest waiting request with up to ``max_batch`` of its requests: one
  batched ampS of all their (clip, family, polarisation) units, each unit with
  its own clip period, then one fused Abbe launch per configuration.  Requests
  that arrived while other launches were running join the next launch
  (continuous batching), and launches on different streams overlap on the
  device;
* admits a launch only when its device block fits in the free part of the
  HBM arena (``hbm_budget`` bytes, first fit) and uses at most half of it, so
  the launches in flight never exceed the budget;
* polls CUDA events to complete requests and records their latency from
  arrival to the image being in host memory.

A clip's result does not depend on the other clips of its launch: every
group has one fixed Euler factor count (``Server.group_euler``) and the
double-angle steps are per unit.  ``plain=True`` is the unbatched FP64 form
(one request per launch, one unit per ampS call).

The reference has no serving layer (its drivers read one ``mask.bin`` and write
one file); this is the north-star serving form of the same computation.
"""
from __future__ import annotations

import collections
import ctypes as C
import dataclasses
import math
import time
from typing import Deque, Dict, List, Optional, Sequence, Tuple

import numpy as np
import torch

from . import _lib as L
from . import masks as MK
from . import tables as T
from .config import PI, SimConfig, preset
from .engine import IntensityBatch, Plan


@dataclasses.dataclass(frozen=True)
class ClipKey:
    """Configuration of a request: period (nm), order box half-size, source points."""

    period: int
    box: int
    n_src: int
    pols: Tuple[str, ...] = ("X", "Y")


def config_for(key: ClipKey) -> SimConfig:
    """The high-NA workload optics for a request configuration: NA 0.55, 4x/8x,
    annular 0.5-0.9 with enough Bloch families for ``n_src`` points (the first
    ``n_src`` of the enumeration)."""
    base = preset("small")
    cfg = base.with_(ndivx=key.period, ndivy=key.period, lbox=key.box, mbox=key.box,
                     max_sources=key.n_src, ndivs=1)
    nd = 1
    while sum(len(f.pts) for f in T.sources(cfg.with_(ndivs=nd, max_sources=None))[1]) < key.n_src:
        nd += 1
        if nd > 16:
            break
    return cfg.with_(ndivs=nd)


def propagating(period: int, box: int, cfg: Optional[SimConfig] = None) -> bool:
    """True when every order of the box stays propagating in vacuum (the
    reference takes a real square root there, header.h:1283)."""
    c = preset("small") if cfg is None else cfg
    k = 2 * PI / c.wavelength
    kx = abs(c.kx0) + 2 * PI * (box + 1) / period
    ky = abs(c.ky0) + 2 * PI * (box + 1) / period
    return kx * kx + ky * ky < k * k


@dataclasses.dataclass
class Request:
    rid: int
    key: ClipKey
    mask: np.ndarray          # packed uint8 [bytes]
    arrival: float            # seconds on the server clock
    image: Optional[np.ndarray] = None
    done: Optional[float] = None
    error: Optional[str] = None   # set (and image None) when the device reported a failure

    @property
    def latency(self) -> Optional[float]:
        return None if self.done is None else self.done - self.arrival


class Arena:
    """One device buffer (the serving HBM budget) handed out as first-fit
    regions: a batch is admitted only when its workspace fits."""

    def __init__(self, nbytes: int, device):
        self.buf = torch.empty(int(nbytes), dtype=torch.uint8, device=device)
        self.used: List[Tuple[int, int]] = []  # sorted (offset, size)

    @property
    def size(self) -> int:
        return self.buf.numel()

    def alloc(self, nbytes: int) -> Optional[int]:
        nbytes = (int(nbytes) + 255) & ~255
        off = 0
        for o, sz in self.used:
            if o - off >= nbytes:
                break
            off = o + sz
        if off + nbytes > self.size:
            return None
        self.used.append((off, nbytes))
        self.used.sort()
        return off

    def free(self, off: int) -> None:
        self.used = [(o, s) for o, s in self.used if o != off]

    def view(self, off: int, nbytes: int) -> torch.Tensor:
        return self.buf[off:off + ((int(nbytes) + 255) & ~255)]


class Executor:
    """Prepared batch of n clips of one configuration: resident per-unit tables,
    spectra, amplitudes and image buffers; the workspace comes from the arena
    at launch."""

    def __init__(self, plan: Plan, n: int, max_units: int, plain: bool):
        self.plan = plan
        self.n = n
        self.plain = plain
        self.batch = IntensityBatch(plan, n, max_units=max_units, own_work=False)
        self.need = self.batch.work_bytes
        if plain:
            self.batch._plain = self.batch._unit_descs(1)
            self.need = max(self.batch.spec_bytes, max(c[3] for c in self.batch._plain))
        self.hin = torch.zeros(tuple(self.batch.masks.shape), dtype=torch.uint8).pin_memory()
        self.hout = torch.empty(tuple(self.batch.image.shape), dtype=torch.float64).pin_memory()
        self.hstat = torch.zeros(1, dtype=torch.int32).pin_memory()
        b = self.batch
        self.bytes = int(sum(t.numel() * t.element_size() for t in (b.masks, b.spec_raw, b.ax, b.image)))
        self.busy = False

    def launch(self, reqs: List[Request], stream: torch.cuda.Stream, work: torch.Tensor) -> torch.cuda.Event:
        for i, r in enumerate(reqs):
            self.hin[i, 0].copy_(torch.from_numpy(r.mask))
        with torch.cuda.stream(stream):
            self.batch.masks.copy_(self.hin, non_blocking=True)
            if self.plain:
                self.batch.run_plain(work)
            else:
                self.batch.run(work)
            self.hout.copy_(self.batch.image, non_blocking=True)
            # the batch's device status word travels with its image, then restarts at 0
            self.hstat.copy_(self.batch.status, non_blocking=True)
            self.batch.status.zero_()
            ev = torch.cuda.Event()
            ev.record(stream)
        return ev


# Source slots of every Abbe table in grouped launches (the largest source
# count a request may ask for): one source stride for all configurations.
MAX_SOURCES = 200


@dataclasses.dataclass(frozen=True)
class GroupKey:
    """Requests that can share one ampS launch: the same order box (hence the
    same order set and matrix size) and polarisations.  Their periods and
    source counts may differ: each unit carries its own period (euv_amp_desc
    d_dx / d_dy), source columns and Abbe tables."""

    box: int
    pols: Tuple[str, ...]


def group_of(key: ClipKey) -> GroupKey:
    return GroupKey(key.box, key.pols)


def _al(n: int) -> int:
    return (int(n) + 255) & ~255


class Slot:
    """One stream of the server with its device status word and pinned
    staging buffers (grown on demand, reused once the slot's launch is done)."""

    def __init__(self, device):
        self.stream = torch.cuda.Stream(device=device)
        self.status = torch.zeros(1, dtype=torch.int32, device=device)
        self.hstat = torch.zeros(1, dtype=torch.int32).pin_memory()
        self.hin = torch.zeros(0, dtype=torch.uint8)
        self.hout = torch.zeros(0, dtype=torch.float64)

    def staging(self, nin: int, nout: int) -> None:
        if self.hin.numel() < nin:
            self.hin = torch.zeros(nin, dtype=torch.uint8).pin_memory()
        if self.hout.numel() < nout:
            self.hout = torch.zeros(nout, dtype=torch.float64).pin_memory()


class GroupLaunch:
    """Host side of one launch of a group: the requests ordered by
    configuration, the per-unit tables, the device layout and its size.

    Units are clip-major within each configuration; configuration c holds
    clips [c0, c0 + n) and units [u0, u0 + n * tables).  Device region (one
    arena block): masks | per-unit tables | spectra | Ax | images | scratch;
    masks and tables are staged in pinned memory with the same layout and go
    over in one copy."""

    def __init__(self, server: "Server", group: GroupKey, reqs: List[Request]):
        self.group = group
        self.reqs = sorted(reqs, key=lambda r: (r.key.period, r.key.n_src, r.arrival))
        pad = server.n_src_pad
        parts = []  # (plan, tables, [requests])
        for r in self.reqs:
            if parts and parts[-1][2][0].key == r.key:
                parts[-1][2].append(r)
            else:
                plan = server.plan(r.key)
                parts.append((plan, plan.abbe_tables(pad), [r]))
        self.parts = parts
        p0 = parts[0][0]
        self.N = p0.orders.n
        self.npol = len(group.pols)
        self.nabs = p0.cfg.nabs
        self.S = (4 * p0.orders.lmax + 1) * (4 * p0.orders.mmax + 1)
        kx0, ky0, dx, dy, pol, spec, order, kz2 = [], [], [], [], [], [], [], []
        tab, img, nsrc, invw = [], [], [], []
        self.part_units, self.part_images, self.part_masks, self.part_clip0 = [], [], [], []
        mask_off = img_off = 0
        ci = 0
        for plan, tb, rs in parts:
            ntab = len(tb["pol"])
            nf = len(plan.fams)
            cfg = plan.cfg
            u0 = len(kx0)
            self.part_clip0.append(ci)
            for j in range(len(rs)):
                for t in range(ntab):
                    kx0.append(tb["kx0"][t])
                    ky0.append(tb["ky0"][t])
                    dx.append(cfg.dx)
                    dy.append(cfg.dy)
                    pol.append(tb["pol"][t])
                    spec.append(ci + j)
                    order.append(tb["order"][t])
                    kz2.append(tb["kz2"][t])
                    tab.append(t)
                    img.append(j * self.npol + t // nf)
                    nsrc.append(tb["nsrc"][t])
            invw += [1.0 / plan.sdivsum] * (len(rs) * self.npol)
            self.part_units.append((u0, len(kx0) - u0))
            nb = cfg.ndivx * cfg.ndivy // 8
            self.part_masks.append((mask_off, nb))
            mask_off += len(rs) * nb
            isz = self.npol * cfg.xdiv * cfg.ydiv
            self.part_images.append((img_off, isz))
            img_off += len(rs) * isz
            ci += len(rs)
        self.n_clips = ci
        self.U = U = len(kx0)
        self.k0_max = float(max(np.abs(kx0).max(), np.abs(ky0).max()))
        self.dx_min, self.dy_min = float(min(dx)), float(min(dy))
        # host tables, in device layout order
        arrays = [np.asarray(kx0, np.float64), np.asarray(ky0, np.float64),
                  np.asarray(dx, np.float64), np.asarray(dy, np.float64),
                  np.asarray(pol, np.int32), np.asarray(spec, np.int32),
                  np.asarray(order, np.int32).reshape(-1), np.asarray(kz2, np.float64).reshape(-1),
                  np.asarray(tab, np.int32), np.asarray(img, np.int32),
                  np.asarray(nsrc, np.int32), np.asarray(invw, np.float64)]
        self.table_offsets = []
        off = _al(mask_off)
        for a in arrays:
            self.table_offsets.append(off)
            off += _al(a.nbytes)
        self.arrays = arrays
        self.in_bytes = off                         # masks + tables: the staged part
        self.spec_off = off
        off += _al(self.n_clips * self.nabs * self.S * 16)
        self.ax_off = off
        off += _al(U * pad * self.N * 16)
        self.img_off = off
        self.img_count = img_off
        off += _al(img_off * 8)
        self.scratch_off = off
        desc = self._desc(server, 0)
        amp = L.lib().euv_amp_workspace_bytes(C.byref(desc))
        if amp == 0:
            raise ValueError("invalid ampS descriptor for group %s" % (group,))
        spec_ws = max(L.lib().euv_mask_spectrum_workspace_bytes(
            len(rs), plan.cfg.ndivx, plan.cfg.ndivy, plan.cfg.fdivx, plan.cfg.fdivy,
            2 * plan.orders.lmax, 2 * plan.orders.mmax) for plan, _, rs in parts)
        self.scratch_bytes = _al(max(amp, spec_ws))
        self.need = off + self.scratch_bytes

    def _desc(self, server: "Server", base: int) -> L.AmpDesc:
        """ampS descriptor of the launch; ``base`` = device address of the block
        (0 while sizing)."""
        p0 = self.parts[0][0]
        d = p0.amp_desc(p0.orders, p0._t_l, p0._t_m, torch.zeros(1, dtype=torch.float64),
                        torch.zeros(1, dtype=torch.float64), torch.zeros(1, dtype=torch.int32),
                        torch.zeros(1, dtype=torch.int32), torch.zeros((1, 1), dtype=torch.int32),
                        torch.zeros((1, 1), dtype=torch.float64), [])
        d.dx, d.dy = self.dx_min, self.dy_min
        d.n_units = self.U
        d.n_src = server.n_src_pad
        d.k0_max = self.k0_max
        d.euler_f = server.group_euler(self.group)
        o = self.table_offsets
        if base:
            d.d_kx0, d.d_ky0, d.d_dx, d.d_dy = base + o[0], base + o[1], base + o[2], base + o[3]
            d.d_polar, d.d_spec, d.d_src_order, d.d_src_2kz = (base + o[4], base + o[5],
                                                               base + o[6], base + o[7])
        return d

    def launch(self, server: "Server", slot: Slot, work: torch.Tensor) -> torch.cuda.Event:
        base = work.data_ptr()
        slot.staging(self.in_bytes, self.img_count)
        hin = slot.hin.numpy()
        for (plan, _, rs), (moff, nb) in zip(self.parts, self.part_masks):
            for j, r in enumerate(rs):
                hin[moff + j * nb:moff + (j + 1) * nb] = r.mask
        for off, a in zip(self.table_offsets, self.arrays):
            hin[off:off + a.nbytes] = a.view(np.uint8)
        st = slot.stream.cuda_stream
        with torch.cuda.stream(slot.stream):
            work[:self.in_bytes].copy_(slot.hin[:self.in_bytes], non_blocking=True)
            scratch = base + self.scratch_off
            for (plan, _, rs), (moff, nb), c0 in zip(self.parts, self.part_masks,
                                                     self.part_clip0):
                cfg = plan.cfg
                out = base + self.spec_off + c0 * self.nabs * self.S * 16
                if self.nabs > 1:
                    raise ValueError("grouped serving takes one absorber slice")
                L.call("euv_mask_spectrum", base + moff, len(rs), cfg.ndivx, cfg.ndivy, cfg.fdivx,
                       cfg.fdivy, 2 * plan.orders.lmax, 2 * plan.orders.mmax, 0, cfg.yflip_offset,
                       out, scratch, self.scratch_bytes, st)
            d = self._desc(server, base)
            d.d_status = slot.status.data_ptr()
            L.call("euv_amp", C.byref(d), base + self.spec_off, base + self.ax_off, scratch,
                   self.scratch_bytes, st)
            imgs = work[self.img_off:self.img_off + self.img_count * 8]
            imgs.zero_()
            o = self.table_offsets
            for (plan, tb, rs), (u0, nu), (ioff, isz), c0 in zip(
                    self.parts, self.part_units, self.part_images, self.part_clip0):
                cfg = plan.cfg
                a = L.AbbeDesc()
                a.xdiv, a.ydiv, a.lpx, a.lpy = cfg.xdiv, cfg.ydiv, cfg.lpmaxX, cfg.lpmaxY
                a.ncut, a.n_units, a.n_src, a.n_order = plan.ncut, nu, server.n_src_pad, self.N
                a.d_coef, a.d_nidx = tb["coef"].data_ptr(), tb["nidx"].data_ptr()
                a.d_px, a.d_py, a.d_row_start = (tb["px"].data_ptr(), tb["py"].data_ptr(),
                                                 tb["row_start"].data_ptr())
                a.d_tab_of_unit = base + o[8] + 4 * u0
                a.d_img_of_unit = base + o[9] + 4 * u0
                a.d_nsrc_of_unit = base + o[10] + 4 * u0
                a.n_images = len(rs) * self.npol
                a.d_inv_weight = base + o[11] + 8 * c0 * self.npol
                a.precision = plan.precision
                L.call("euv_abbe", C.byref(a), base + self.ax_off + u0 * server.n_src_pad * self.N * 16,
                       base + self.img_off + 8 * ioff, st)
            slot.hout[:self.img_count].copy_(imgs.view(torch.float64), non_blocking=True)
            # the launch's device status word travels with its images, then restarts at 0
            slot.hstat.copy_(slot.status, non_blocking=True)
            slot.status.zero_()
            ev = torch.cuda.Event()
            ev.record(slot.stream)
        return ev

    def results(self, slot: Slot):
        """(request, image [pols, xdiv, ydiv]) pairs from the slot's output."""
        out = slot.hout.numpy()
        for (plan, _, rs), (ioff, isz) in zip(self.parts, self.part_images):
            shp = (self.npol, plan.cfg.xdiv, plan.cfg.ydiv)
            for j, r in enumerate(rs):
                yield r, out[ioff + j * isz:ioff + (j + 1) * isz].reshape(shp).copy()


class Server:
    """Continuous-batching server.  Mixed precision: requests of one group
    (order box and polarisations, any period and source count) share a launch:
    one batched ampS of all their units, then one Abbe launch per
    configuration.  plain=True: the unbatched FP64 form, one unit per call."""

    def __init__(self, device=None, precision: str = "mixed", max_batch: int = 8,
                 n_streams: int = 4, hbm_budget: Optional[int] = None, plain: bool = False,
                 n_src_pad: int = MAX_SOURCES):
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.precision = precision
        self.max_batch = 1 if plain else max_batch
        self.plain = plain
        self.n_src_pad = int(n_src_pad)
        n = 1 if plain else n_streams
        self.slots = [Slot(self.device) for _ in range(n)]
        self.streams = [s.stream for s in self.slots]
        free, _ = torch.cuda.mem_get_info(self.device)
        budget = int(hbm_budget if hbm_budget is not None else 0.5 * free)
        self.arena = Arena(budget, self.device)
        self.plans: Dict[ClipKey, Plan] = {}
        self.execs: Dict[Tuple[ClipKey, int], Executor] = {}
        self.euler: Dict[GroupKey, int] = {}
        self.waits_for_memory = 0
        # the requests of every grouped launch, in launch order (for inspection)
        self.launched_groups: List[List[Request]] = []

    # ---------------------------------------------------------------- set-up
    def plan(self, key: ClipKey) -> Plan:
        p = self.plans.get(key)
        if p is None:
            with torch.cuda.device(self.device):
                p = Plan(config_for(key), device=self.device, pols=key.pols,
                         precision="fp64" if self.plain else self.precision)
                p.abbe_tables() if self.plain else p.abbe_tables(self.n_src_pad)
            self.plans[key] = p
        return p

    def _key_euler(self, key: ClipKey) -> int:
        """Euler factor count ampS derives for this configuration alone."""
        plan = self.plan(key)
        tb = plan.abbe_tables(self.n_src_pad)
        d = plan.amp_desc(plan.orders, plan._t_l, plan._t_m, torch.zeros(1, dtype=torch.float64),
                          torch.zeros(1, dtype=torch.float64), torch.zeros(1, dtype=torch.int32),
                          torch.zeros(1, dtype=torch.int32), torch.zeros((1, 1), dtype=torch.int32),
                          torch.zeros((1, 1), dtype=torch.float64), [])
        d.k0_max = float(max(np.abs(tb["kx0"]).max(), np.abs(tb["ky0"]).max()))
        f = L.lib().euv_amp_euler_factors(C.byref(d))
        if f < -1:
            raise ValueError("invalid ampS descriptor for %s" % (key,))
        return f

    def group_euler(self, group: GroupKey) -> int:
        """The group's fixed Euler factor count: the largest any of its warmed
        configurations needs alone (the FP64 LU, -1, if one needs it), so a
        clip's result does not depend on the clips it shares a launch with."""
        if group not in self.euler:
            fs = [self._key_euler(k) for k in self.plans if group_of(k) == group]
            self.euler[group] = -1 if (not fs or -1 in fs) else max(fs)
        return self.euler[group]

    def batch_sizes(self) -> List[int]:
        """Prepared batch sizes of the plain form: powers of two up to max_batch."""
        out, n = [], 1
        while n <= self.max_batch:
            out.append(n)
            n *= 2
        return out

    def executor(self, key: ClipKey, n: int) -> Executor:
        ex = self.execs.get((key, n))
        if ex is None:
            plan = self.plan(key)
            N = plan.orders.n
            per_unit = 12 * N * N * 16
            # a launch may use at most half of the arena, so two always fit
            max_units = max(1, (self.arena.size // 2) // max(per_unit, 1))
            with torch.cuda.device(self.device):
                ex = Executor(plan, n, max_units, self.plain)
            if ex.need > self.arena.size:
                raise MemoryError("configuration %s needs %d bytes of workspace, arena has %d"
                                  % (key, ex.need, self.arena.size))
            self.execs[(key, n)] = ex
        return ex

    def warm(self, keys: Sequence[ClipKey]) -> None:
        """Resident tables of every configuration the stream will use, the
        groups' Euler factor counts and, for the plain form, prepared batches
        (outside any timing)."""
        for k in keys:
            self.plan(k)
        if self.plain:
            for k in keys:
                for n in self.batch_sizes():
                    self.executor(k, n)
        else:
            self.euler.clear()
            for g in {group_of(k) for k in keys}:
                self.group_euler(g)
        torch.cuda.synchronize(self.device)

    @property
    def resident_bytes(self) -> int:
        n = sum(e.bytes for e in self.execs.values())
        for p in self.plans.values():
            for tb in (p._abbe_tables or {}).values():
                n += sum(v.numel() * v.element_size() for v in tb.values()
                         if isinstance(v, torch.Tensor))
        return n

    # ---------------------------------------------------------------- serve
    def _take(self, q: Deque[Request]) -> List[Request]:
        """Up to max_batch of the oldest requests of a group whose launch fits
        in half of the arena."""
        rs = [q[0]]
        while len(rs) < min(self.max_batch, len(q)):
            trial = GroupLaunch(self, group_of(q[0].key), rs + [q[len(rs)]])
            if trial.need > self.arena.size // 2:
                break
            rs.append(q[len(rs)])
        for _ in rs:
            q.popleft()
        return rs

    def serve(self, requests: Sequence[Request]) -> Dict:
        """Run the arrival trace (request.arrival: seconds from now) to completion;
        returns latency and throughput statistics."""
        if self.plain:
            return self._serve_plain(requests)
        reqs = sorted(requests, key=lambda r: r.arrival)
        pending: Dict[GroupKey, Deque[Request]] = collections.defaultdict(collections.deque)
        inflight = []  # (slot index, launch, event, arena offset)
        free_slots = list(range(len(self.slots)))
        nxt = 0
        t0 = time.perf_counter()
        batches = clips = failed = 0
        while nxt < len(reqs) or inflight or any(pending.values()):
            now = time.perf_counter() - t0
            while nxt < len(reqs) and reqs[nxt].arrival <= now:
                pending[group_of(reqs[nxt].key)].append(reqs[nxt])
                nxt += 1
            still = []
            for si, gl, ev, off in inflight:
                if ev.query():
                    t = time.perf_counter() - t0
                    slot = self.slots[si]
                    err = L.status_message(int(slot.hstat[0]))
                    for r, img in gl.results(slot):
                        r.image = None if err else img
                        r.error = err
                        r.done = t
                    failed += len(gl.reqs) if err else 0
                    self.arena.free(off)
                    free_slots.append(si)
                else:
                    still.append((si, gl, ev, off))
            inflight = still
            launched = False
            while free_slots:
                groups = [g for g, q in pending.items() if q]
                if not groups:
                    break
                g = min(groups, key=lambda k: pending[k][0].arrival)  # oldest request first
                q = pending[g]
                rs = self._take(q)
                gl = GroupLaunch(self, g, rs)
                off = self.arena.alloc(gl.need)
                if off is None:  # HBM footprint: wait for a running batch to finish
                    for r in reversed(rs):
                        q.appendleft(r)
                    self.waits_for_memory += 1
                    break
                si = free_slots.pop()
                ev = gl.launch(self, self.slots[si], self.arena.view(off, gl.need))
                inflight.append((si, gl, ev, off))
                self.launched_groups.append(gl.reqs)
                batches += 1
                clips += len(rs)
                launched = True
            if not launched:
                time.sleep(0.0002)
        return self._stats(reqs, t0, batches, clips, failed)

    def _stats(self, reqs, t0, batches, clips, failed) -> Dict:
        end = time.perf_counter() - t0
        lat = np.array([r.latency for r in reqs])
        first = min(r.arrival for r in reqs)
        return {
            "requests": len(reqs),
            "clips_per_s": len(reqs) / (end - first),
            "p50_ms": float(np.percentile(lat, 50) * 1e3),
            "p99_ms": float(np.percentile(lat, 99) * 1e3),
            "mean_batch": clips / max(batches, 1),
            "batches": batches,
            "wall_s": end - first,
            "arena_bytes": self.arena.size,
            "resident_bytes": self.resident_bytes,
            "waits_for_memory": self.waits_for_memory,
            "failed": failed,
        }

    def _serve_plain(self, requests: Sequence[Request]) -> Dict:
        """The unbatched FP64 form: one request per launch, one unit per ampS call."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        pending: Deque[Request] = collections.deque()
        inflight = None
        nxt = 0
        t0 = time.perf_counter()
        batches = failed = 0
        stream = self.slots[0].stream
        while nxt < len(reqs) or inflight or pending:
            now = time.perf_counter() - t0
            while nxt < len(reqs) and reqs[nxt].arrival <= now:
                pending.append(reqs[nxt])
                nxt += 1
            if inflight is not None and inflight[2].query():
                ex, r, ev, off = inflight[0], inflight[1], inflight[2], inflight[3]
                err = L.status_message(int(ex.hstat[0]))
                r.image = None if err else ex.hout.numpy()[0].copy()
                r.error = err
                r.done = time.perf_counter() - t0
                failed += 1 if err else 0
                ex.busy = False
                self.arena.free(off)
                inflight = None
            if inflight is None and pending:
                r = pending.popleft()
                ex = self.executor(r.key, 1)
                off = self.arena.alloc(ex.need)
                if off is None:
                    raise MemoryError("the arena cannot hold one plain launch")
                ex.busy = True
                ev = ex.launch([r], stream, self.arena.view(off, ex.need))
                inflight = (ex, r, ev, off)
                batches += 1
            else:
                time.sleep(0.0002)
        return self._stats(reqs, t0, batches, batches, failed)


# -------------------------------------------------------------------- workload
PERIODS = (256, 512, 1024, 2048)
BOXES = (5, 10, 15, 20)          # 11x11, 21x21, 31x31, 41x41 orders
SOURCE_COUNTS = (50, 100, 150, 200)


_VALID: Dict[Tuple[int, int, int], bool] = {}


def valid(period: int, box: int, n_src: int) -> bool:
    """The order box propagates and holds every order the pupil reads."""
    k = (period, box, n_src)
    if k not in _VALID:
        ok = propagating(period, box)
        if ok:
            ln, mn = T.required_orders(config_for(ClipKey(period, box, n_src)))
            ok = box >= ln and box >= mn
        _VALID[k] = ok
    return _VALID[k]


def workload(n: int, rate: float, seed: int, periods=PERIODS, boxes=BOXES,
             source_counts=SOURCE_COUNTS) -> List[Request]:
    """Poisson arrivals (mean ``rate`` per second) of seeded clips: period and
    source-point count uniform, order box uniform among the boxes valid for
    them (all orders propagate, every pupil order inside the box)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n):
        t += rng.exponential(1.0 / rate)
        P = int(rng.choice(periods))
        q = int(rng.choice(source_counts))
        ok = [b for b in boxes if valid(P, b, q)]
        if not ok:
            raise ValueError("no valid order box for period %d" % P)
        key = ClipKey(P, int(rng.choice(ok)), q)
        m = MK.pack(MK.synth_mask(P, P, seed=1000 * seed + i))
        out.append(Request(i, key, m, t))
    return out


def main(argv=None) -> int:
    import argparse
    import json
    ap = argparse.ArgumentParser(description="serve a Poisson stream of clips")
    ap.add_argument("--requests", type=int, default=200)
    ap.add_argument("--rate", type=float, default=50.0)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--max-period", type=int, default=2048)
    a = ap.parse_args(argv)
    periods = tuple(p for p in PERIODS if p <= a.max_period)
    out = {}
    for name, kw in (("mixed", dict(precision="mixed")), ("plain_fp64", dict(plain=True))):
        reqs = workload(a.requests, a.rate, a.seed, periods=periods)
        srv = Server(**kw)
        t = time.perf_counter()
        srv.warm(sorted({r.key for r in reqs}, key=lambda k: (k.period, k.box, k.n_src)))
        warm_s = time.perf_counter() - t
        stats = srv.serve(reqs)
        stats["warm_s"] = warm_s
        out[name] = stats
        del srv
        torch.cuda.empty_cache()
    out["rate_per_s"] = a.rate
    out["throughput_ratio"] = out["mixed"]["clips_per_s"] / out["plain_fp64"]["clips_per_s"]
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
