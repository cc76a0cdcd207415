"""CNN predict oracle (CPU): compmask and the six networks pinned against the
reference's own compmask / predict_m3d outputs (tests/golden/ref_cnn.npz,
made by tests/golden/make_cnn_golden.py), and the inputxx.csv writer."""
import os

import numpy as np
import pytest
import torch

from oracle import cnn_oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_cnn.npz")


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


def oracle_models(seeds):
    models = O.build_models(seeds)
    for i, m in enumerate(models):
        O.perturb_batchnorm(m, 100 + i)
    return models


def test_compmask_matches_the_reference(golden):
    for raw, counts in zip(golden["bits"], golden["counts"]):
        x = O.compmask_bits(raw)
        assert x.shape == (512, 512)
        np.testing.assert_array_equal(x * 16, counts.astype(np.float32))


def test_oracle_networks_match_the_reference(golden):
    """Same seeds, same layer order -> the reference's parameters; the outputs
    agree to FP32 rounding (tolerance 1e-5 of each array's max)."""
    torch.set_num_threads(max(1, min(8, os.cpu_count() or 1)))
    models = oracle_models(golden["seeds"])
    x = torch.from_numpy(golden["counts"].astype(np.float32) / 16).reshape(-1, 1, 512, 512)
    outs = O.predict_m3d(x, models, O.seeded_factors())
    for name, got in zip(O.MODEL_NAMES, outs):
        ref = golden[name]
        assert got.shape == ref.shape, name
        err = np.max(np.abs(got - ref)) / np.max(np.abs(ref))
        assert err < 1e-5, (name, err)


def test_inputxx_layout(tmp_path):
    outs = [np.arange(6.0).reshape(2, 3) * (i + 1) for i in range(6)]
    p = tmp_path / "inputxx.csv"
    O.write_inputxx(str(p), outs)
    rows = np.loadtxt(p, delimiter=",")
    assert rows.shape == (12, 3)
    np.testing.assert_array_equal(rows[4:6], outs[2])
