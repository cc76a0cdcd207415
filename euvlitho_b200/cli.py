"""Drop-in replacements of the reference executables.

  python -m euvlitho_b200.cli intensity   # int.out: ./mask.bin -> emint.csv
  python -m euvlitho_b200.cli m3d         # m3d.out: ./mask.bin -> inputxx.csv, inputlm.csv
  python -m euvlitho_b200.cli linear      # linear.py: ./mask.bin + inputxx.csv -> intlinear.csv, intft.csv
  python -m euvlitho_b200.cli maskgen     # mask.out: mask.bin (--count masks) + maskimage.csv
  python -m euvlitho_b200.cli predict --models DIR   # predict.py: ./mask.bin -> inputxx.csv

Both run the reference configuration (intensity.cpp:44-91, m3d.cpp:34-95) on
the GPU; --preset picks another workload.
"""
from __future__ import annotations

import argparse
import sys
import time

import numpy as np
import torch

from . import io
from .config import preset
from .engine import Plan


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("what", choices=["intensity", "m3d", "linear", "maskgen", "predict"])
    ap.add_argument("--models", default="../model",
                    help="predict: directory with re0/ im0/ rex/ imx/ rey/ imy/ model.ckpt and factors")
    ap.add_argument("--seed", type=int, default=1, help="srand seed (maskgen; 1 = the reference's)")
    ap.add_argument("--inputxx", default="./inputxx.csv", help="M3D parameters (linear)")
    ap.add_argument("--preset", default="reference")
    ap.add_argument("--mask", default="./mask.bin")
    ap.add_argument("--count", type=int, default=1, help="masks in the file (m3d ndata)")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--pol", default="X", choices=["X", "Y"])
    a = ap.parse_args(argv)
    cfg = preset(a.preset)
    t0 = time.time()
    if a.what == "maskgen":
        from . import masks as MK
        bits = MK.vbf_batch(a.count, cfg.ndivx, cfg.ndivy, seed=a.seed).cpu().numpy()
        bits[:, 0].tofile("mask.bin")                    # mask.cpp:41-48
        first = MK.unpack(bits[0, 0], cfg.ndivx, cfg.ndivy)
        with open("maskimage.csv", "w") as fh:           # mask.cpp:49-59
            for row in first:
                fh.write("".join("%d," % v for v in row))
                fh.write("\n")
        print("elapsed time (s) %.3f" % (time.time() - t0))
        return 0
    if a.what == "predict":
        from . import cnn
        pred = cnn.CnnPredictor.from_checkpoints(a.models)       # predict.py:123-131
        raw = np.fromfile(a.mask, np.uint8)
        outs = pred.predict(raw.reshape(-1, cnn.MASK_BYTES))     # predict.py:133-142
        cnn.write_inputxx("inputxx.csv", outs)                   # predict.py:145-151
        print("elapsed time (s) %.3f" % (time.time() - t0))
        return 0
    plan = Plan(cfg, precision=a.precision, pols=(a.pol,))
    masks = torch.from_numpy(io.read_mask_bin(a.mask, cfg.ndivx, cfg.ndivy, a.count))
    if a.what == "linear":
        p = io.read_inputxx(a.inputxx)
        ax = io.expand_xinput(p["ax"], plan.xinput)
        ay = io.expand_xinput(p["ay"], plan.xinput)
        lin, ft = plan.linear(masks[:1], p["a0"][None], ax[None], ay[None])
        io.write_image_full("intlinear.csv", lin[0].cpu().numpy())
        io.write_image_full("intft.csv", ft[0].cpu().numpy())
    elif a.what == "intensity":
        img = plan.intensity(masks[:1]).cpu().numpy()
        io.write_emint("emint.csv" if a.pol == "X" else "emintY.csv", img[0, 0])
    else:
        res = plan.m3d(masks)
        io.write_inputlm("inputlm.csv", plan.linput, plan.minput, plan.xinput)
        with open("inputxx.csv", "w"):
            pass
        for c in range(masks.shape[0]):
            a0 = res["a0"][c].cpu().numpy()
            ax = res["ax"][c].cpu().numpy()
            ay = res["ay"][c].cpu().numpy()
            io.write_inputxx("inputxx.csv" if c == 0 else "inputxx_%d.csv" % c, a0, ax, ay, plan.xinput)
    print("elapsed time (s) %.3f" % (time.time() - t0))
    return 0


if __name__ == "__main__":
    sys.exit(main())
