"""Golden outputs of the reference's CNN predict (run once, in a container that
holds the reference checkout; writes tests/golden/ref_cnn.npz).

The reference's ``cnn/cnn/predict/predict.py`` defines the networks
``CNNmodel`` / ``CNNmodels`` and ``predict_m3d``; ``compmask.py`` downsamples a
mask.bin raster.  The trained checkpoints are not shipped, so the six networks
are the reference's own classes default-initialised under
``torch.manual_seed(SEEDS[i])``, with BatchNorm statistics set by
``oracle.cnn_oracle.perturb_batchnorm(model, 100 + i)`` and factors from
``oracle.cnn_oracle.seeded_factors()``; the tests rebuild the same parameters
with the oracle's ``CnnNet`` (same layer declaration order, same seeds).

Stand-in, numerically transparent: ``pytorch_lightning`` is not installed, so
a module whose ``LightningModule`` is ``torch.nn.Module`` takes its place (the
networks use nothing else of it).

Masks: the reference's ``cnn/cnn/predict/mask.bin`` and one seeded synthetic
raster (rectangles).  Stored: both rasters (bits), their compmask outputs
(as counts = 16 x value, uint8), and the six output arrays [2, n_out] (float64).

Usage:  python tests/golden/make_cnn_golden.py [REFERENCE_ROOT]   (a few minutes)
"""
import os
import sys
import tempfile
import time
import types

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

SEEDS = (11, 12, 13, 14, 15, 16)


def synthetic_raster(seed: int = 3) -> np.ndarray:
    """2048 x 2048 bits (1 = vacuum) with seeded absorber rectangles, packed."""
    rng = np.random.Generator(np.random.PCG64(seed))
    img = np.ones((2048, 2048), np.uint8)
    for _ in range(60):
        w, h = rng.integers(16, 400, 2)
        x, y = rng.integers(0, 2048, 2)
        img[y:y + h, x:x + w] = 0
    return np.packbits(img.reshape(-1))


def main() -> int:
    from refroot import reference_root
    ref = reference_root()
    d = os.path.join(ref, "cnn", "cnn", "predict")
    pl = types.ModuleType("pytorch_lightning")
    pl.LightningModule = torch.nn.Module
    sys.modules["pytorch_lightning"] = pl
    sys.path.insert(0, d)
    import compmask as CM  # the reference's compmask.py
    import predict as P    # the reference's predict.py
    from oracle import cnn_oracle as O

    raw0 = np.fromfile(os.path.join(d, "mask.bin"), np.uint8)
    raw1 = synthetic_raster()
    t0 = time.perf_counter()
    xs = [CM.compmask(os.path.join(d, "mask.bin"))]
    with tempfile.TemporaryDirectory() as td:
        fn = os.path.join(td, "mask.bin")
        raw1.tofile(fn)
        xs.append(CM.compmask(fn))
    t1 = time.perf_counter()
    models = []
    for i, s in enumerate(SEEDS):
        torch.manual_seed(s)
        m = P.CNNmodel() if i < 2 else P.CNNmodels()
        O.perturb_batchnorm(m, 100 + i)
        models.append(m)
    f0, fx, fy = O.seeded_factors()
    x = torch.from_numpy(np.stack(xs).reshape(-1, 1, 512, 512))
    with torch.no_grad():
        outs = P.predict_m3d(x, *models, f0, fx, fy)
    t2 = time.perf_counter()
    out = os.path.join(HERE, "ref_cnn.npz")
    counts = (np.stack(xs).astype(np.float32) * 16).round().astype(np.uint8)
    np.savez_compressed(out, bits=np.stack([raw0, raw1]), counts=counts,
                        seeds=np.asarray(SEEDS),
                        **{n: np.asarray(a, np.float64) for n, a in zip(O.MODEL_NAMES, outs)})
    print("compmask %.0f s, predict %.0f s; re0[0,:3] %s -> %s"
          % (t1 - t0, t2 - t1, np.asarray(outs[0])[0, :3], out))
    return 0


if __name__ == "__main__":
    sys.exit(main())
