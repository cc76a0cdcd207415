"""Continuous-batching server for Abbe images of mask clips.

Requests are single clips with their own optical configuration (period, order
box, source points, polarisations).  The server keeps, per configuration, a
resident :class:`~euvlitho_b200.engine.Plan` (order/pupil/source tables and the
Abbe E-field factors) and prepared batches (per-unit tables, spectra, amplitude
and image buffers) for 1, 2, 4, .. max_batch clips.  One host loop:

* admits the requests that have arrived into per-configuration queues;
* whenever one of ``n_streams`` stream slots is idle, launches the oldest
  waiting configuration with up to ``max_batch`` of its requests -- requests
  that arrived while other batches were running join the next launch
  (continuous batching), and batches of different configurations run on
  different streams at the same time (their kernels overlap on the device);
* admits a batch only when its workspace fits in the free part of the HBM
  arena (``hbm_budget`` bytes, first fit), so the batches in flight never
  exceed the budget; large configurations run their units in chunks so one
  launch needs at most half of the arena;
* polls CUDA events to complete requests and records their latency from
  arrival to the image being in host memory.

The reference has no serving layer (its drivers read one ``mask.bin`` and write
one file); this is the north-star serving form of the same computation.
"""
from __future__ import annotations

import collections
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


class Server:
    def __init__(self, device=None, precision: str = "mixed", max_batch: int = 4,
                 n_streams: int = 4, hbm_budget: Optional[int] = None, plain: bool = False):
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.precision = precision
        self.max_batch = 1 if plain else max_batch
        self.plain = plain
        self.streams = [torch.cuda.Stream(device=self.device) for _ in range(1 if plain else n_streams)]
        free, _ = torch.cuda.mem_get_info(self.device)
        budget = int(hbm_budget if hbm_budget is not None else 0.5 * free)
        self.arena = Arena(budget, self.device)
        self.plans: Dict[ClipKey, Plan] = {}
        self.execs: Dict[Tuple[ClipKey, int], Executor] = {}
        self.waits_for_memory = 0

    # ---------------------------------------------------------------- set-up
    def plan(self, key: ClipKey) -> Plan:
        p = self.plans.get(key)
        if p is None:
            with torch.cuda.device(self.device):
                p = Plan(config_for(key), device=self.device, pols=key.pols,
                         precision="fp64" if self.plain else self.precision)
                p.abbe_tables()
            self.plans[key] = p
        return p

    def batch_sizes(self) -> List[int]:
        """Prepared batch sizes: powers of two up to max_batch."""
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
            per_unit = 12 * N * N * 16 + (2 * 4 * N * (N + 16) * 4 if plan.precision == L.EUV_PREC_MIXED else 0)
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
        """Resident tables and prepared batches of every configuration the stream
        will use (outside any timing)."""
        for k in keys:
            for n in self.batch_sizes():
                self.executor(k, n)
        torch.cuda.synchronize(self.device)

    @property
    def resident_bytes(self) -> int:
        return sum(e.bytes for e in self.execs.values())

    # ---------------------------------------------------------------- serve
    def serve(self, requests: Sequence[Request]) -> Dict:
        """Run the arrival trace (request.arrival: seconds from now) to completion;
        returns latency and throughput statistics."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        pending: Dict[ClipKey, Deque[Request]] = collections.defaultdict(collections.deque)
        inflight = []  # (slot, executor, requests, event, arena offset)
        free_slots = list(range(len(self.streams)))
        nxt = 0
        t0 = time.perf_counter()
        batches = 0
        clips = 0
        failed = 0
        while nxt < len(reqs) or inflight or any(pending.values()):
            now = time.perf_counter() - t0
            while nxt < len(reqs) and reqs[nxt].arrival <= now:
                pending[reqs[nxt].key].append(reqs[nxt])
                nxt += 1
            still = []
            for slot, ex, rs, ev, off in inflight:
                if ev.query():
                    t = time.perf_counter() - t0
                    img = ex.hout.numpy()
                    err = L.status_message(int(ex.hstat[0]))
                    for i, r in enumerate(rs):
                        r.image = None if err else img[i].copy()
                        r.error = err
                        r.done = t
                    failed += len(rs) if err else 0
                    ex.busy = False
                    self.arena.free(off)
                    free_slots.append(slot)
                else:
                    still.append((slot, ex, rs, ev, off))
            inflight = still
            launched = False
            while free_slots:
                keys = [k for k, q in pending.items() if q]
                if not keys:
                    break
                key = min(keys, key=lambda k: pending[k][0].arrival)  # oldest request first
                q = pending[key]
                sizes = [s for s in self.batch_sizes() if s <= len(q)]
                ex = None
                for n in sorted(sizes, reverse=True):
                    e = self.executor(key, n)
                    if not e.busy:
                        ex = e
                        break
                if ex is None:
                    break
                off = self.arena.alloc(ex.need)
                if off is None:  # HBM footprint: wait for a running batch to finish
                    self.waits_for_memory += 1
                    break
                rs = [q.popleft() for _ in range(ex.n)]
                slot = free_slots.pop()
                ex.busy = True
                ev = ex.launch(rs, self.streams[slot], self.arena.view(off, ex.need))
                inflight.append((slot, ex, rs, ev, off))
                batches += 1
                clips += ex.n
                launched = True
            if not launched:
                time.sleep(0.0002)
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
