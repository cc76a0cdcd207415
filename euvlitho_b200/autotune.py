"""Autotuner for the library's tunable launches.

For a prepared :class:`~euvlitho_b200.engine.IntensityBatch` it times, on the
device, every candidate of each knob on the whole step (spectra, batched ampS,
Abbe) and keeps the fastest per problem shape in the library's tuning table
(``euv_tune_set``).  Picks are cached in a JSON file per GPU model, so later
processes start from them (``load``); shapes without a pick keep the
built-in choice.

Knobs (``EUV_KNOB_*`` in include/euvl_b200.h):

* ``abbe_split``  -- key (units, source slots) of the Abbe launch: how many CTAs
  share a unit's sources (built in: the split that fills the waves of
  resident CTAs);
* ``lu_cluster``  -- key (n, batch) of an LU: the smallest CTA cluster that
  factors a panel (built in: the fewest CTAs whose registers hold its rows);
* ``lu_subst_cols`` -- key (n, batch) of an LU solve: right-hand sides per CTA,
  8 or 12 (built in: 12 where that takes fewer waves of CTAs);
* ``zgemm_rows``  -- key (m, batch) of the FP64 GEMM: 64- or 32-row tiles
  (FP64 form only; the mixed form's products run on the split-FP16x3 kernel).

The cache file is ``$EUVLITHO_TUNE_CACHE`` or
``~/.cache/euvlitho_b200/tuning.json``: ``{gpu name: {"knob/k0/k1": value}}``.
"""
from __future__ import annotations

import json
import os
from typing import Dict, List, Optional, Sequence, Tuple

import torch

from . import _lib as L

KNOBS = {"abbe_split": L.EUV_KNOB_ABBE_SPLIT, "lu_cluster": L.EUV_KNOB_LU_CLUSTER,
         "lu_subst_cols": L.EUV_KNOB_LU_SUBST_COLS, "zgemm_rows": L.EUV_KNOB_ZGEMM_ROWS}
CANDIDATES = {"abbe_split": (1, 2, 3, 4, 6, 8, 12, 16, 24, 32),
              "lu_cluster": (1, 2, 4, 8),
              "lu_subst_cols": (8, 12),
              "zgemm_rows": (64, 32)}


def cache_path() -> str:
    p = os.environ.get("EUVLITHO_TUNE_CACHE")
    if p:
        return p
    return os.path.join(os.path.expanduser("~"), ".cache", "euvlitho_b200", "tuning.json")


def gpu_name(device=None) -> str:
    return torch.cuda.get_device_name(device)


def _read(path: str) -> Dict:
    try:
        with open(path) as f:
            d = json.load(f)
        return d if isinstance(d, dict) else {}
    except (OSError, ValueError):
        return {}


def load(path: Optional[str] = None, device=None) -> int:
    """Apply the cached picks of this GPU model (0 = the built-in choice);
    returns how many."""
    entries = _read(path or cache_path()).get(gpu_name(device), {})
    n = 0
    for key, value in entries.items():
        try:
            name, k0, k1 = key.split("/")
            if L.lib().euv_tune_set(KNOBS[name], int(k0), int(k1), int(value)) == L.EUV_OK:
                n += 1
        except (KeyError, ValueError):
            continue
    return n


def save(picks: Dict[Tuple[str, int, int], int], path: Optional[str] = None, device=None) -> str:
    """Merge picks {(knob, k0, k1): value} into the cache file; value 0 records
    that the built-in choice won for that shape."""
    path = path or cache_path()
    data = _read(path)
    mine = data.setdefault(gpu_name(device), {})
    for (name, k0, k1), v in picks.items():
        mine["%s/%d/%d" % (name, k0, k1)] = int(v)
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    # one temporary file per process: ranks tuning at once (one process per GPU)
    # each replace the cache atomically; the last writer's picks stay
    tmp = "%s.tmp.%d" % (path, os.getpid())
    with open(tmp, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
    os.replace(tmp, path)
    return path


def _time_ms(fn, reps: int) -> float:
    fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s = torch.cuda.current_stream()
    best = float("inf")
    for _ in range(reps):
        e0.record(s)
        fn()
        e1.record(s)
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    return best


def shapes(batch) -> Dict[str, List[Tuple[int, int]]]:
    """The keys each knob sees in one run of the batch."""
    plan = batch.plan
    N, U = plan.orders.n, batch.U
    out = {"abbe_split": [(U, batch.ax.shape[1])], "lu_cluster": [(N, U)],
           "lu_subst_cols": [(N, U)]}
    if plan.precision == L.EUV_PREC_FP64:
        out["zgemm_rows"] = [(N, U)]
    return out


def tune_batch(batch, knobs: Sequence[str] = tuple(KNOBS), reps: int = 3,
               min_gain: float = 0.01) -> Dict:
    """Coordinate descent over the knobs at the batch's shapes: each candidate
    timed on the whole step (best of ``reps`` CUDA-event timings); a pick is
    kept only if it beats the built-in choice by ``min_gain``.  Returns
    {"base_ms", "tuned_ms", "picks": {(knob, k0, k1): value}, "trials": [...]}."""
    lib = L.lib()
    run = batch.run
    sh = shapes(batch)
    for name in knobs:  # start from the built-in choices
        for k0, k1 in sh.get(name, []):
            lib.euv_tune_set(KNOBS[name], k0, k1, 0)
    base = _time_ms(run, reps)
    best_ms = base
    picks: Dict[Tuple[str, int, int], int] = {}
    trials = []
    for name in knobs:
        for k0, k1 in sh.get(name, []):
            cur_val, cur_ms = 0, best_ms
            for v in CANDIDATES[name]:
                L.check("euv_tune_set", lib.euv_tune_set(KNOBS[name], k0, k1, v))
                ms = _time_ms(run, reps)
                trials.append({"knob": name, "key": [k0, k1], "value": v, "ms": ms})
                if ms < cur_ms * (1.0 - min_gain) and ms < cur_ms:
                    cur_val, cur_ms = v, ms
            lib.euv_tune_set(KNOBS[name], k0, k1, cur_val)
            picks[(name, k0, k1)] = cur_val
            best_ms = cur_ms
    batch.check()
    return {"base_ms": base, "tuned_ms": best_ms, "picks": picks, "trials": trials}


def ensure(batch, path: Optional[str] = None, reps: int = 3) -> Dict:
    """Picks for the batch's shapes: from the cache when it has every one of
    them (``tuned`` False), else tuned now and saved (first use)."""
    load(path)
    have = _read(path or cache_path()).get(gpu_name(), {})
    need = [(n, k0, k1) for n, ks in shapes(batch).items() for k0, k1 in ks]
    if all("%s/%d/%d" % k in have for k in need):
        return {"tuned": False, "picks": {k: have["%s/%d/%d" % k] for k in need}}
    res = tune_batch(batch, reps=reps)
    save(res["picks"], path)
    res["tuned"] = True
    return res


def main(argv=None) -> int:
    import argparse
    from . import masks as MK
    from .config import preset
    from .engine import Plan
    ap = argparse.ArgumentParser(description="tune the library's launches for a workload")
    ap.add_argument("--preset", default="batched")
    ap.add_argument("--clips", type=int, default=4)
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--pols", default="XY")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--cache", default=None)
    ap.add_argument("--save", action="store_true", help="merge the picks into the cache file")
    a = ap.parse_args(argv)
    cfg = preset(a.preset)
    plan = Plan(cfg, pols=tuple(a.pols), precision=a.precision)
    b = plan.intensity_batch(a.clips)
    b.masks.copy_(torch.from_numpy(MK.batch(cfg.ndivx, cfg.ndivy, range(a.clips))))
    res = tune_batch(b, reps=a.reps)
    if a.save:
        save(res["picks"], a.cache)
    out = {"preset": a.preset, "clips": a.clips, "precision": a.precision,
           "orders": plan.orders.n, "units": b.U, "gpu": gpu_name(),
           "base_ms": res["base_ms"], "tuned_ms": res["tuned_ms"],
           "picks": {"%s/%d/%d" % k: v for k, v in res["picks"].items()},
           "trials": res["trials"]}
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
