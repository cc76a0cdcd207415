"""Pin the oracle against the reference's golden outputs (test infrastructure).

Runs the oracle once at the reference configuration of
``cnn/intensity/abbe/intensity.cpp:44-91`` and ``cnn/intensity/m3d/m3d.cpp:34-95``
(NA 0.33, MX=MY=4, 2048 nm clip on a 2048^2 grid, annular sigma 0.55-0.9,
Ta absorber 60 nm in one slice, X polarisation, orders: rounded diamond with
cut 6 -> N=8705, narrow ellipse cut 1.5 -> N=1009) on the reference's
``mask.bin`` and compares with its ``emint.csv`` and ``inputxx.csv``.

One wide ampS solve serves both outputs: intensity.cpp has a single Bloch
family (ndivs=1, sx0=kx0) with the same order set, polarisation and incidence
as m3d.cpp:279-285.

Usage:  python oracle/pin_golden.py [--golden tests/golden] [--out DIR]

The golden files are read from ``tests/golden`` (gzip copies of the reference
files made by ``tests/golden/make_golden.py``).  Writes ``pin_summary.json``
with the error figures into ``tests/golden`` and the oracle's own outputs
into ``--out``.  Takes ~20-40 min on 8 cores (one 8705^2 complex zgeev).
"""
from __future__ import annotations

import argparse
import gzip
import io
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

from oracle import euv_oracle as O  # noqa: E402


def reference_config() -> O.SimConfig:
    # reference constants; the golden files come from a revision whose y flip
    # is one row off header.h:1159 (see SimConfig.yflip_offset)
    return O.SimConfig(yflip_offset=1)


def load_gz_text(path: str) -> str:
    with gzip.open(path, "rt") as fh:
        return fh.read()


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--golden", default=os.path.join(os.path.dirname(HERE), "tests", "golden"))
    ap.add_argument("--out", default=os.path.join(os.path.dirname(HERE), "_work", "pin"))
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    cfg = reference_config()
    with gzip.open(os.path.join(args.golden, "ref_mask.bin.gz"), "rb") as fh:
        data = fh.read()
    mask = O.decompress_bits(data, cfg.ndivx * cfg.ndivy)
    LMAX, MMAX = O.order_limits(cfg, "diamond", 6.0)
    lidx, midx = O.order_set("diamond", LMAX, MMAX)
    print("N =", len(lidx), "LMAX", LMAX, flush=True)
    t0 = time.time()
    Ax = O.amp_s("X", mask, cfg, lidx, midx, LMAX, MMAX, cfg.kx0, cfg.ky0)
    t_wide = time.time() - t0
    print("wide ampS %.1f s" % t_wide, flush=True)
    np.savez(os.path.join(args.out, "ax_wide.npz"),
             keys=np.array(list(Ax.keys())), vals=np.array(list(Ax.values())))
    images = O.intensity(cfg, mask, ax_cache={("X", 0, 0): Ax})
    I = images["X"]
    O.write_emint(os.path.join(args.out, "emint.csv"), I)
    t1 = time.time()
    res = O.m3d(cfg, mask, Ax_wide=Ax)
    t_m3d = time.time() - t1
    O.write_inputxx(os.path.join(args.out, "inputxx.csv"), res)
    O.write_inputlm(os.path.join(args.out, "inputlm.csv"), res)

    Ig = O.read_emint(io.StringIO(load_gz_text(os.path.join(args.golden, "ref_emint.csv.gz"))))
    gx = O.read_inputxx(io.StringIO(load_gz_text(os.path.join(args.golden, "ref_inputxx.csv.gz"))))
    lm = np.loadtxt(io.StringIO(load_gz_text(os.path.join(args.golden, "ref_inputlm.csv.gz"))),
                    delimiter=",", dtype=np.int64)
    summary = {
        "config": "reference (NA 0.33, 2048 nm, diamond cut 6, N=%d, X pol)" % len(lidx),
        "seconds_wide_ampS": t_wide,
        "seconds_m3d_rest": t_m3d,
        "inputlm_equal": bool(np.array_equal(lm, np.stack([res["linput"], res["minput"], res["xinput"]], 1))),
        "emint_max_abs_err_over_max": float(np.max(np.abs(I - Ig)) / np.max(np.abs(Ig))),
        "emint_median_rel_err": float(np.median(np.abs(I - Ig) / np.abs(Ig))),
    }
    for key in ("a0", "ax", "ay"):
        a, g = res[key], gx[key]
        summary[key + "_max_abs_err_over_max"] = float(np.max(np.abs(a - g)) / np.max(np.abs(g)))
        summary[key + "_median_abs_err"] = float(np.median(np.abs(a - g)))
    print(json.dumps(summary, indent=1), flush=True)
    with open(os.path.join(args.golden, "pin_summary.json"), "w") as fh:
        json.dump(summary, fh, indent=1)
    return 0


if __name__ == "__main__":
    sys.exit(main())
