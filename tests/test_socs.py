"""STCC-SOCS (cnn/intensity/stccsocs), CPU side: the oracle's restatement
against the reference's own eigenfunction + intsocs
(tests/golden/make_socs_golden.py) at the reference configuration."""
import gzip
import os

import numpy as np
import pytest

from oracle import euv_oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def golden():
    p = os.path.join(GOLDEN, "ref_socs.npz")
    if not os.path.exists(p):
        pytest.skip("ref_socs.npz not generated")
    return np.load(p)


@pytest.fixture(scope="module")
def eig():
    cfg = O.SimConfig()
    tccs = O.socs_tcc(cfg, 0.0)
    z, copies = O.socs_padding(cfg)  # the reference's padded pupil list
    return cfg, [O.socs_eigen(t, z, copies) for t in tccs]


def test_tcc_eigenvalues_match_the_reference(golden, eig):
    _, e = eig
    for (alpha, _), name in zip(e, ("alpha_s0", "alpha_sx", "alpha_sy")):
        ref = np.abs(golden[name])  # the sign order within +-lambda ties is rounding
        err = np.max(np.abs(np.abs(alpha[:len(ref)]) - ref)) / np.max(ref)
        assert err < 1e-12, (name, err)


def test_oracle_reproduces_the_reference_socs_image(golden, eig):
    cfg, e = eig
    with gzip.open(os.path.join(GOLDEN, "ref_mask.bin.gz")) as fh:
        mask2d = O.decompress_bits(fh.read(), cfg.ndivx * cfg.ndivy)
    with gzip.open(os.path.join(GOLDEN, "ref_inputxx.csv.gz"), "rt") as fh:
        p = O.read_inputxx(fh)
    lin, mn, xin, _ = O.pupil_set(cfg)
    img = O.socs_image(cfg, mask2d, p["a0"], O.expand_xinput(p["ax"], xin),
                       O.expand_xinput(p["ay"], xin), complex(golden["ampvc"]),
                       complex(golden["ampab"]), (e[0][0], e[0][1], e[1][0], e[1][1], e[2][0], e[2][1]))
    ref = golden["intsocs"].astype(np.float64)
    err = np.max(np.abs(img - ref)) / np.max(ref)
    assert err < 2e-7, err  # float32 storage of the fixture
