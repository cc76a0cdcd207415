"""CNN predict of the M3D parameters on the GPU.

Mirrors ``predict_m3d`` of cnn/cnn/predict/predict.py:108-121 and its driver
(predict.py:122-151): six networks (re0, im0 with ncut outputs; rex, imx, rey,
imy with ncuts outputs) applied to a mask downsampled by compmask
(cnn/cnn/predict/compmask.py:17-41), outputs divided by factor0 / factorx /
factory, written to inputxx.csv with ``np.savetxt``.

The networks run through ``libeuvl_b200.so`` (``euv_cnn_pack`` once,
``euv_cnn_predict`` per batch of masks): tcgen05 TF32x3 implicit-GEMM
convolutions with fused ReLU / max-pool / BatchNorm epilogues and split-K
fully connected layers.  There is no host fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Dict, List, Mapping, Optional, Sequence

import numpy as np
import torch

from . import _lib as L

MODEL_NAMES = ("re0", "im0", "rex", "imx", "rey", "imy")
# predict.py:129-131: the factor file of each model (re0/im0 share factor0, ...)
FACTOR_FILES = (("re0", "factor0.csv"), ("re0", "factor0.csv"), ("rex", "factorx.csv"),
                ("rex", "factorx.csv"), ("rey", "factory.csv"), ("rey", "factory.csv"))
MASK_BYTES = 2048 * 2048 // 8
_CONV = ("conv1", "conv2", "conv3", "conv4", "conv5")
_NORM = ("norm1", "norm2", "norm3", "norm4", "norm5")


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


def load_checkpoint(path: str) -> Dict[str, torch.Tensor]:
    """The ``state_dict`` of a Lightning ``model.ckpt`` (or a plain state_dict
    file), loaded without unpickling arbitrary objects."""
    obj = torch.load(path, map_location="cpu", weights_only=True)
    if isinstance(obj, Mapping) and "state_dict" in obj:
        obj = obj["state_dict"]
    if not isinstance(obj, Mapping) or "fc2.weight" not in obj:
        raise ValueError("%s: not a CNNmodel state_dict (no fc2.weight)" % path)
    return dict(obj)


class CnnPredictor:
    """Resident packed weights of up to six networks and a workspace.

    ``state_dicts``: one mapping per network with the reference's keys
    (conv1.weight ... norm5.running_var, fc1.weight, fc2.bias).
    ``factors``: one 1-D array per network (its n_out divisors).
    """

    def __init__(self, state_dicts: Sequence[Mapping[str, torch.Tensor]],
                 factors: Sequence[np.ndarray], device: Optional[torch.device] = None,
                 bn_eps: float = 1e-5):
        L.lib()  # fail loudly if the library is missing
        if not torch.cuda.is_available():
            raise RuntimeError("CnnPredictor needs a CUDA device (no host fallback)")
        m = len(state_dicts)
        if not 1 <= m <= L.EUV_CNN_MAX_MODELS or len(factors) != m:
            raise ValueError("need 1..6 state_dicts and one factor array per network")
        self.device = torch.device(device or "cuda")
        self.n_models = m
        self.n_out = [int(sd["fc2.weight"].shape[0]) for sd in state_dicts]
        self.max_out = max(self.n_out)
        for n, f in zip(self.n_out, factors):
            if np.asarray(f).reshape(-1).size != n:
                raise ValueError("a factor array does not match its network's n_out")
        fac = np.zeros((m, self.max_out))
        for i, f in enumerate(factors):
            fac[i, :self.n_out[i]] = np.asarray(f, np.float64).reshape(-1)
            fac[i, self.n_out[i]:] = 1.0
        self.factors = torch.from_numpy(fac).to(self.device)
        nbytes = L.lib().euv_cnn_blob_bytes(m, self.max_out)
        if nbytes == 0:
            raise ValueError("unsupported network count or output size")
        self.blob = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
        self._work: Optional[torch.Tensor] = None
        self.status = torch.zeros(1, dtype=torch.int32, device=self.device)
        self._pack(state_dicts, bn_eps)

    @classmethod
    def from_checkpoints(cls, model_dir: str, device: Optional[torch.device] = None,
                         names: Sequence[str] = MODEL_NAMES) -> "CnnPredictor":
        """predict.py:123-131: ``<model_dir>/<name>/model.ckpt`` and the factor
        csv files (``re0/factor0.csv``, ``rex/factorx.csv``, ``rey/factory.csv``)."""
        sds = [load_checkpoint(os.path.join(model_dir, n, "model.ckpt")) for n in names]
        facs = []
        for n in names:
            sub, fn = FACTOR_FILES[MODEL_NAMES.index(n)]
            facs.append(np.loadtxt(os.path.join(model_dir, sub, fn), delimiter=","))
        return cls(sds, facs, device)

    def _pack(self, sds: Sequence[Mapping[str, torch.Tensor]], eps: float) -> None:
        keep: List[torch.Tensor] = []

        def dev(sd, key, shape=None) -> int:
            t = sd[key].detach().to(self.device, torch.float32).contiguous()
            if shape is not None and tuple(t.shape) != shape:
                raise ValueError("%s has shape %s, expected %s" % (key, tuple(t.shape), shape))
            keep.append(t)
            return t.data_ptr()

        arr = (L.CnnModelWeights * self.n_models)()
        ch = (1, 16, 32, 64, 128, 256)
        for i, sd in enumerate(sds):
            w = arr[i]
            for l in range(5):
                w.conv_w[l] = dev(sd, _CONV[l] + ".weight", (ch[l + 1], ch[l], 3, 3))
                w.conv_b[l] = dev(sd, _CONV[l] + ".bias", (ch[l + 1],))
                w.bn_w[l] = dev(sd, _NORM[l] + ".weight", (ch[l + 1],))
                w.bn_b[l] = dev(sd, _NORM[l] + ".bias", (ch[l + 1],))
                w.bn_mean[l] = dev(sd, _NORM[l] + ".running_mean", (ch[l + 1],))
                w.bn_var[l] = dev(sd, _NORM[l] + ".running_var", (ch[l + 1],))
            w.fc1_w = dev(sd, "fc1.weight", (4096, 65536))
            w.fc1_b = dev(sd, "fc1.bias", (4096,))
            w.fc2_w = dev(sd, "fc2.weight", (self.n_out[i], 4096))
            w.fc2_b = dev(sd, "fc2.bias", (self.n_out[i],))
            w.n_out = self.n_out[i]
        with torch.cuda.device(self.device):
            L.call("euv_cnn_pack", self.n_models, arr, self.max_out, float(eps),
                   self.blob.data_ptr(), self.blob.numel(), _stream())
            torch.cuda.current_stream().synchronize()  # the torch copies in `keep` die here

    def workspace(self, n_masks: int) -> torch.Tensor:
        nbytes = L.lib().euv_cnn_workspace_bytes(self.n_models, n_masks, self.max_out)
        if nbytes == 0:
            raise ValueError("unsupported batch of %d masks" % n_masks)
        if self._work is None or self._work.numel() < nbytes:
            self._work = None
            self._work = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
        return self._work

    def as_bits(self, masks) -> torch.Tensor:
        """mask.bin rasters -> uint8 [B, 524288] on the device."""
        if isinstance(masks, (bytes, bytearray)):
            masks = [masks]
        if isinstance(masks, torch.Tensor):
            t = masks
        else:
            t = torch.from_numpy(np.stack([np.frombuffer(bytes(m), np.uint8)
                                           if not isinstance(m, np.ndarray) else m.reshape(-1)
                                           for m in masks]))
        t = t.reshape(-1, MASK_BYTES)
        if t.dtype != torch.uint8:
            raise TypeError("mask rasters must be uint8 (mask.bin bytes)")
        return t.to(self.device, non_blocking=True).contiguous()

    def predict_device(self, bits: torch.Tensor, out: Optional[torch.Tensor] = None) -> torch.Tensor:
        """Enqueue one batch on the current stream: bits uint8 [B, 524288] on the
        device -> out float64 [n_models, B, max_out] (no synchronisation)."""
        b = int(bits.shape[0])
        if out is None:
            out = torch.empty((self.n_models, b, self.max_out), dtype=torch.float64,
                              device=self.device)
        d = L.CnnDesc()
        d.n_models, d.n_masks, d.max_out = self.n_models, b, self.max_out
        for i, n in enumerate(self.n_out):
            d.n_out[i] = n
        d.d_factors = self.factors.data_ptr()
        d.d_status = self.status.data_ptr()
        ws = self.workspace(b)
        L.call("euv_cnn_predict", C.byref(d), bits.data_ptr(), self.blob.data_ptr(),
               out.data_ptr(), ws.data_ptr(), ws.numel(), _stream())
        return out

    def check(self) -> None:
        """Raise EuvError if a bounded device wait gave up (synchronises)."""
        bits = int(self.status.item())
        if bits:
            self.status.zero_()
            L.check_status("CnnPredictor", bits)

    def predict(self, masks) -> List[np.ndarray]:
        """predict_m3d: six (or n_models) float64 arrays [B, n_out]."""
        bits = self.as_bits(masks)
        out = self.predict_device(bits)
        self.check()
        host = out.cpu().numpy()
        return [host[i, :, :n] for i, n in enumerate(self.n_out)]


def predict_m3d(masks, predictor: CnnPredictor) -> List[np.ndarray]:
    """predict.py:108-121 on the GPU: re0, im0, rex, imx, rey, imy."""
    return predictor.predict(masks)


def write_inputxx(path: str, outs: Sequence[np.ndarray]) -> None:
    """predict.py:145-151: each array with np.savetxt(delimiter=','), in order."""
    with open(path, "w") as f:
        for a in outs:
            np.savetxt(f, a, delimiter=",")
