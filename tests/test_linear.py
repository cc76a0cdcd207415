"""Linear Abbe model from the M3D parameters (cnn/intensity/linear/linear.py),
CPU side: the host tables against the oracle, and the oracle against images
made by the reference's own int_linear (tests/golden/make_linear_golden.py)."""
import gzip
import os

import numpy as np
import pytest

from euvlitho_b200 import tables as T
from euvlitho_b200.config import SimConfig, preset
from oracle import euv_oracle as O
from tests.helpers import to_oracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _configs():
    ref = SimConfig()
    small = preset("small")
    return [ref, small, small.with_(illum_type=0), small.with_(illum_type=2, openangle=60.0),
            small.with_(illum_type=3)]


@pytest.mark.parametrize("cfg", _configs(), ids=["ref", "small", "circ", "dipx", "dipy"])
def test_source_grid_matches_the_oracle(cfg):
    dsx, dsy = T.linear_sources(cfg)
    ox, oy = O.linear_sources(to_oracle(cfg))
    assert len(dsx) > 0
    np.testing.assert_array_equal(dsx, ox)
    np.testing.assert_array_equal(dsy, oy)


@pytest.mark.parametrize("obsc", [0.0, 0.2])
def test_abbe_factors_match_the_oracle_field(obsc):
    """coef = i k R(:,0) phase / sqrt(k^2 - kx^2) point by point, as the oracle's
    high-NA E-field and Abbe phase (electro_field.py:45-76, linear.py:26-32)."""
    cfg = preset("small").with_(obscuration=obsc, z=20)
    oc = to_oracle(cfg)
    lin, mn, _, _ = O.pupil_set(oc)
    dsx, dsy = T.linear_sources(cfg)
    coef, nidx = T.linear_abbe_table(cfg, dsx, dsy, lin, mn)
    k, MX, MY, NA = oc.k, oc.mx, oc.my, oc.na
    for s in range(0, len(dsx), max(1, len(dsx) // 7)):
        kx = oc.kx0 + dsx[s]
        for i in range(len(lin)):
            kxn = dsx[s] + 2 * O.PI * lin[i] / oc.dx
            kyn = dsy[s] + 2 * O.PI * mn[i] / oc.dy
            p2 = MX * MX * kxn * kxn + MY * MY * kyn * kyn
            if not ((NA * k * obsc) ** 2 <= p2 <= (NA * k) ** 2):
                assert nidx[s, i] == -1 and not coef[s, i].any()
                continue
            assert nidx[s, i] == i
            R = O.rotate(k, MX, MY, kxn, kyn, oc.kx0, oc.ky0)
            ph = np.exp(1j * ((kxn + oc.kx0) ** 2 + (kyn + oc.ky0) ** 2) / (2 * k) * oc.z0
                        + 1j * p2 / (2 * k) * 20.0)
            want = 1j * k * R[:, 0] * ph / np.sqrt(k * k - kx * kx)
            np.testing.assert_allclose(coef[s, i], want, rtol=1e-13, atol=1e-13)


def _golden():
    p = os.path.join(GOLDEN, "ref_linear.npz")
    if not os.path.exists(p):
        pytest.skip("ref_linear.npz not generated")
    return np.load(p)


def test_oracle_reproduces_the_reference_linear_model():
    """The restatement against the reference's own int_linear on the shipped
    mask and inputxx.csv (reference configuration, 2048 nm, NA 0.33; golden
    images stored as float32: 5.1e-8 measured, the float32 rounding)."""
    g = _golden()
    cfg = O.SimConfig()
    with gzip.open(os.path.join(GOLDEN, "ref_mask.bin.gz")) as fh:
        mask2d = O.decompress_bits(fh.read(), cfg.ndivx * cfg.ndivy)
    with gzip.open(os.path.join(GOLDEN, "ref_inputxx.csv.gz"), "rt") as fh:
        p = O.read_inputxx(fh)
    lin, mn, xin, _ = O.pupil_set(cfg)
    a0, ax, ay = p["a0"], O.expand_xinput(p["ax"], xin), O.expand_xinput(p["ay"], xin)
    dsx, dsy = O.linear_sources(cfg)
    alin, athin = O.linear_amplitudes(cfg, mask2d, a0, ax, ay, complex(g["ampvc"]),
                                      complex(g["ampab"]), dsx, dsy, lin, mn)
    for amp, name in ((alin, "intlinear"), (athin, "intft")):
        img = O.linear_image(cfg, amp, dsx, dsy, lin, mn)
        ref = g[name].astype(np.float64)
        err = np.max(np.abs(img - ref)) / np.max(ref)
        assert err < 2e-7, (name, err)
