"""CPU oracle for the CNN predict of the M3D parameters.

TEST INFRASTRUCTURE ONLY.  This module is the checker: only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may import
it.  The product (``euvlitho_b200.cnn``) never imports or calls it.

It restates, in PyTorch FP32 on the CPU (the reference runs these networks
with PyTorch FP32 on the CPU), paths relative to the reference repository:

* ``cnn/cnn/predict/compmask.py:17-41`` -- ``compmask``: the 2048 x 2048
  MSB-first bit raster of mask.bin, row-major, reduced to 512 x 512 by
  ``rowmat @ mask @ columnmat`` with 1/4 weights on 4-pixel bins, i.e. the
  mean of each 4 x 4 box (exact in float16: multiples of 1/16);
* ``cnn/cnn/predict/predict.py:16-88`` -- ``CNNmodel`` / ``CNNmodels``: five
  stages conv 3x3 (circular padding 1) -> ReLU -> 2x2 max-pool -> BatchNorm
  (eval), channels 1-16-32-64-128-256, flatten in (c, h, w) order, fc1
  65536 -> 4096 + ReLU, fc2 4096 -> n_out (ncut 1901 for re0/im0, ncuts 1749
  for rex/imx/rey/imy);
* ``predict.py:90-121`` -- ``Fullmodel`` / ``predict_m3d``: the six networks on the same input,
  outputs divided by factor0 (re0, im0), factorx (rex, imx), factory (rey,
  imy); ``predict.py:145-151`` writes the six arrays with ``np.savetxt``.

``CnnNet`` declares its layers in the reference's order (conv1..conv5,
norm1..norm5, pool, fc1, fc2), so under the same ``torch.manual_seed`` its
default initialisation draws the same parameters as the reference's class, and
its ``state_dict`` keys are the reference checkpoints' keys.
"""
from __future__ import annotations

from typing import Dict, List, Sequence

import numpy as np
import torch
from torch import nn
from torch.nn import functional as F

MASK_SIDE = 2048
NET_SIDE = 512
NCUT = 1901
NCUTS = 1749
MODEL_NAMES = ("re0", "im0", "rex", "imx", "rey", "imy")
CHANNELS = (1, 16, 32, 64, 128, 256)


def compmask_bits(raw: bytes | np.ndarray) -> np.ndarray:
    """compmask.py:17-41 on one mask.bin raster -> float32 [512, 512]."""
    b = np.frombuffer(bytes(raw), np.uint8) if not isinstance(raw, np.ndarray) else raw
    bits = np.unpackbits(b.reshape(-1)).reshape(MASK_SIDE, MASK_SIDE)
    f = MASK_SIDE // NET_SIDE
    counts = bits.reshape(NET_SIDE, f, NET_SIDE, f).sum(axis=(1, 3), dtype=np.int32)
    return counts.astype(np.float32) / np.float32(f * f)


class CnnNet(nn.Module):
    """predict.py:16-51 (CNNmodel, n_out = 1901) / 53-88 (CNNmodels, 1749)."""

    def __init__(self, n_out: int):
        super().__init__()
        for i in range(5):
            setattr(self, "conv%d" % (i + 1),
                    nn.Conv2d(CHANNELS[i], CHANNELS[i + 1], (3, 3), padding=1,
                              padding_mode="circular"))
        for i in range(5):
            setattr(self, "norm%d" % (i + 1), nn.BatchNorm2d(CHANNELS[i + 1]))
        self.pool = nn.MaxPool2d(2, 2)
        self.fc1 = nn.Linear(16 * 16 * 256, 4096)
        self.fc2 = nn.Linear(4096, n_out)

    def forward(self, x: torch.Tensor) -> torch.Tensor:
        x = x.to(torch.float32)
        for i in range(1, 6):
            x = self.pool(F.relu(getattr(self, "conv%d" % i)(x)))
            x = getattr(self, "norm%d" % i)(x)
        x = torch.flatten(x, 1)
        return self.fc2(F.relu(self.fc1(x)))


def build_models(seeds: Sequence[int], n_outs: Sequence[int] = (NCUT, NCUT, NCUTS, NCUTS,
                                                                 NCUTS, NCUTS)) -> List[CnnNet]:
    """One network per seed, default-initialised under torch.manual_seed(seed)."""
    out = []
    for s, n in zip(seeds, n_outs):
        torch.manual_seed(int(s))
        out.append(CnnNet(int(n)).eval())
    return out


def perturb_batchnorm(model: nn.Module, seed: int) -> None:
    """Deterministic non-trivial BatchNorm statistics (the default init is the
    identity); applied the same way to reference and oracle modules."""
    g = torch.Generator().manual_seed(int(seed))
    with torch.no_grad():
        for i in range(1, 6):
            bn = getattr(model, "norm%d" % i)
            c = bn.num_features
            bn.running_mean.copy_(0.2 * torch.randn(c, generator=g))
            bn.running_var.copy_(0.5 + torch.rand(c, generator=g))
            bn.weight.copy_(1.0 + 0.2 * torch.randn(c, generator=g))
            bn.bias.copy_(0.2 * torch.randn(c, generator=g))


def seeded_factors(n_outs: Sequence[int] = (NCUT, NCUTS, NCUTS), seed: int = 7) -> List[np.ndarray]:
    """factor0 / factorx / factory stand-ins: positive, O(1) (predict.py:129-131
    loads them from the training's csv files)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return [0.5 + rng.random(int(n)) for n in n_outs]


@torch.no_grad()
def predict_m3d(x: torch.Tensor, models: Sequence[nn.Module],
                factors: Sequence[np.ndarray]) -> List[np.ndarray]:
    """predict.py:108-121: x [B, 1, 512, 512]; six arrays [B, n_out] (float64)."""
    f0, fx, fy = factors
    per = (f0, f0, fx, fx, fy, fy)
    return [m(x).detach().cpu().numpy() / np.asarray(f) for m, f in zip(models, per)]


def write_inputxx(path: str, outs: Sequence[np.ndarray]) -> None:
    """predict.py:145-151: the six arrays, np.savetxt with ',' one after another."""
    with open(path, "w") as f:
        for a in outs:
            np.savetxt(f, a, delimiter=",")


def state_dicts(models: Sequence[nn.Module]) -> List[Dict[str, torch.Tensor]]:
    return [{k: v.detach().clone() for k, v in m.state_dict().items()} for m in models]
