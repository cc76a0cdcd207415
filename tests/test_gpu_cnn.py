"""CNN predict on the GPU (euv_cnn_downsample / euv_cnn_pack / euv_cnn_predict)
against the reference's golden outputs and the FP32 oracle.  Tolerance: max
|GPU - reference| <= 1e-4 x max |reference| per output array (TF32x3 products
with FP32 accumulation, split-K sums in a different order)."""
import os

import numpy as np
import pytest
import torch

from euvlitho_b200 import _lib as L
from euvlitho_b200 import cnn
from oracle import cnn_oracle as O

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_cnn.npz")
TOL = 1e-4


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


@pytest.fixture(scope="module")
def models(golden):
    ms = O.build_models(golden["seeds"])
    for i, m in enumerate(ms):
        O.perturb_batchnorm(m, 100 + i)
    return ms


@pytest.fixture(scope="module")
def predictor(cuda, models):
    facs = O.seeded_factors()
    per = [facs[0], facs[0], facs[1], facs[1], facs[2], facs[2]]
    return cnn.CnnPredictor(O.state_dicts(models), per, cuda)


def rasters(n, seed):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        img = np.ones((2048, 2048), np.uint8)
        for _ in range(int(rng.integers(5, 80))):
            w, h = rng.integers(8, 500, 2)
            x, y = rng.integers(0, 2048, 2)
            img[y:y + h, x:x + w] = 0
        out.append(np.packbits(img.reshape(-1)))
    return np.stack(out)


def _rel(got, ref):
    return float(np.max(np.abs(got - ref)) / np.max(np.abs(ref)))


def test_downsample_is_exact(cuda, golden):
    bits = torch.from_numpy(golden["bits"]).to(cuda)
    x0 = torch.empty((bits.shape[0], 512, 512), dtype=torch.float32, device=cuda)
    L.call("euv_cnn_downsample", bits.shape[0], bits.data_ptr(), x0.data_ptr(),
           torch.cuda.current_stream().cuda_stream)
    np.testing.assert_array_equal(x0.cpu().numpy() * 16, golden["counts"].astype(np.float32))


def test_predict_matches_the_reference(predictor, golden):
    outs = predictor.predict(golden["bits"])
    for name, got in zip(O.MODEL_NAMES, outs):
        err = _rel(got, golden[name])
        assert err < TOL, (name, err)


@pytest.mark.parametrize("n,seed", [(1, 5), (3, 6), (20, 7)])
def test_predict_matches_the_oracle(cuda, predictor, models, n, seed):
    """Batches of 1, 3 (one 16-mask tile) and 20 (a 32-mask tile) against the
    oracle run in FP32 on the GPU (TF32 off)."""
    raw = rasters(n, seed)
    x = torch.from_numpy(np.stack([O.compmask_bits(r) for r in raw])).reshape(-1, 1, 512, 512)
    prev = (torch.backends.cuda.matmul.allow_tf32, torch.backends.cudnn.allow_tf32)
    torch.backends.cuda.matmul.allow_tf32 = False
    torch.backends.cudnn.allow_tf32 = False
    try:
        ref = []
        for m in models:
            m.to(cuda)
            with torch.no_grad():
                ref.append(m(x.to(cuda)).double().cpu().numpy())
            m.to("cpu")
    finally:
        torch.backends.cuda.matmul.allow_tf32, torch.backends.cudnn.allow_tf32 = prev
    facs = O.seeded_factors()
    per = [facs[0], facs[0], facs[1], facs[1], facs[2], facs[2]]
    got = predictor.predict(raw)
    for name, g, r, f in zip(O.MODEL_NAMES, got, ref, per):
        assert g.shape == r.shape
        err = _rel(g, r / f)
        assert err < TOL, (name, n, err)


def test_predict_rejects_a_bad_batch(predictor):
    with pytest.raises(TypeError):
        predictor.as_bits(torch.zeros((1, cnn.MASK_BYTES), dtype=torch.float32))
    with pytest.raises(ValueError):
        predictor.workspace(0)


def test_predict_more_masks_than_one_tile(cuda, models):
    """260 masks (two 256-mask tiles of the fc layers, the second holding 4):
    one network, 10 distinct rasters repeated; every repeat matches its first
    occurrence (to 1e-6) and a sample of them the FP32 oracle."""
    facs = O.seeded_factors()
    pred = cnn.CnnPredictor(O.state_dicts(models[:1]), [facs[0]], cuda)
    base = rasters(10, 11)
    raw = np.concatenate([base] * 26)
    got = pred.predict(raw)[0]
    assert got.shape == (260, O.NCUT)
    for i in range(10, 260):
        assert _rel(got[i], got[i % 10]) < 1e-6, i
    x = torch.from_numpy(np.stack([O.compmask_bits(r) for r in base])).reshape(-1, 1, 512, 512)
    prev = (torch.backends.cuda.matmul.allow_tf32, torch.backends.cudnn.allow_tf32)
    torch.backends.cuda.matmul.allow_tf32 = False
    torch.backends.cudnn.allow_tf32 = False
    try:
        m = models[0].to(cuda)
        with torch.no_grad():
            ref = m(x.to(cuda)).double().cpu().numpy() / facs[0]
        models[0].to("cpu")
    finally:
        torch.backends.cuda.matmul.allow_tf32, torch.backends.cudnn.allow_tf32 = prev
    for i in (0, 7, 256, 259):
        err = _rel(got[i], ref[i % 10])
        assert err < TOL, (i, err)
