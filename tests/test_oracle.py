"""Oracle self-checks and its pin against the reference's golden files (CPU)."""
import gzip
import io
import json
import math
import os

import numpy as np
import pytest

from oracle import euv_oracle as O
from tests.helpers import flat_bits, random_mask, rel_err

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_maskamp_fft_equals_direct_dft():
    # header.h:1147-1206 direct DFT vs the FFT of the same pattern, with mesh 2 in x
    cfg = O.SimConfig(ndivx=32, ndivy=32, delta=0.5)
    m = flat_bits(random_mask(32, 32, seed=3))
    a = O.maskamp(m, cfg, 0.9 + 0.05j, 1.0, 3, 2)
    b = O.maskamp(m, cfg, 0.9 + 0.05j, 1.0, 3, 2, direct=True)
    assert np.max(np.abs(a - b)) < 1e-14


def test_reference_set_sizes():
    cfg = O.SimConfig()
    L, M = O.order_limits(cfg, "diamond", 6.0)
    li, mi = O.order_set("diamond", L, M)
    assert (L, M, len(li)) == (75, 75, 8705)
    Ln, Mn = O.order_limits(cfg, "ellipse", 1.5)
    assert len(O.order_set("ellipse", Ln, Mn)[0]) == 1009
    ndivs, fams = O.source(cfg)
    assert ndivs == 1 and sum(len(v) for v in fams.values()) == 256


def test_inputlm_matches_golden():
    cfg = O.SimConfig()
    lin, mn, xin, _ = O.pupil_set(cfg)
    with gzip.open(os.path.join(GOLDEN, "ref_inputlm.csv.gz"), "rt") as fh:
        g = np.loadtxt(fh, delimiter=",", dtype=np.int64)
    assert np.array_equal(g, np.stack([lin, mn, xin], 1))


def test_emint_reader_writer_round_trip(tmp_path):
    I = np.random.default_rng(0).random((8, 4))
    p = str(tmp_path / "e.csv")
    O.write_emint(p, I)
    J = O.read_emint(p)
    assert J.shape == I.shape and np.max(np.abs(I - J) / I) < 1e-5


def _eigen_free_amp(polar, masks, cfg, lidx, midx, L, M, kx0, ky0):
    """The library's eigen-free algebra restated in NumPy (exact eigh-free
    matrix functions via the eigendecomposition here, only to check the algebra)."""
    k = cfg.k
    coefs = O.mask_coefficients(masks, cfg, L, M)
    LL, MM = O._toeplitz_index(lidx, midx, L, M)
    kxp = kx0 + 2 * O.PI * lidx / cfg.dx
    kyp = ky0 + 2 * O.PI * midx / cfg.dy
    kxy2 = kxp ** 2 + kyp ** 2
    klm = np.sqrt(k * k - kxy2).astype(complex)
    URUU, URUB = O.multilayer_s(polar, k, kxp, kyp, kxy2, cfg.stack)
    eru = cfg.stack.n_ru ** 2
    alru = np.sqrt(k * k * eru - kxy2 + 0j)
    kp = kxp if polar == "X" else kyp
    Bru = 1j * k - 1j / k / eru * kp ** 2
    G = lambda sig: 1j * (k * np.eye(len(lidx)) - (kp[:, None] / k) * sig[LL, MM] * kp[None, :])
    X = np.diag(URUU + URUB)
    Y = np.diag(alru * (URUU - URUB))
    Gprev = np.diag(Bru)
    sig_b = coefs[cfg.nabs - 1][1]
    for n in range(cfg.nabs - 1, -1, -1):
        eps, sig, eta, zeta = coefs[n]
        D = O._build_D(polar, LL, MM, k, kxp, kyp, kxy2, eps, eta, zeta)
        Gn = G(sig if cfg.refresh_sigma else sig_b)
        Z = np.linalg.solve(Gn, Gprev @ X)
        w, V = np.linalg.eig(D)
        r = np.sqrt(w)
        d = float(cfg.dabs[n])
        Vi = np.linalg.inv(V)
        c = (V * np.cos(r * d)) @ Vi
        s = (V * (np.sin(r * d) / r)) @ Vi
        X, Y = c @ Z - 1j * (s @ Y), -1j * (D @ (s @ Z)) + c @ Y
        Gprev = Gn
    FG = (1 / klm)[:, None] * (Y @ np.linalg.inv(klm[:, None] * X + Y))
    pos = {(int(a), int(b)): i for i, (a, b) in enumerate(zip(lidx, midx))}
    out = {}
    for (ls, ms), i in pos.items():
        if O._in_na(cfg, ls, ms) and abs(ls) <= cfg.lsmaxX and abs(ms) <= cfg.lsmaxY:
            kx = kx0 + ls * 2 * O.PI / cfg.dx
            ky = ky0 + ms * 2 * O.PI / cfg.dy
            v = -FG[:, i] * 2 * math.sqrt(k * k - kx * kx - ky * ky)
            v[i] += 1
            out[(ls, ms)] = v
    return out


@pytest.mark.parametrize("nsl,refresh,pol", [(1, False, "X"), (1, False, "Y"), (3, False, "X"), (3, True, "Y")])
def test_eigen_free_algebra_matches_oracle(nsl, refresh, pol):
    cfg = O.SimConfig(ndivx=128, ndivy=128, na=0.55, mx=4, my=8, order_kind="box", lbox=4, mbox=3,
                      eabs=tuple([(0.95 + 0.031j) ** 2] * nsl), dabs=tuple([60.0 / nsl] * nsl),
                      refresh_sigma=refresh)
    masks = [flat_bits(random_mask(128, 128, seed=10 + i)) for i in range(nsl)]
    li, mi = O.order_set("box", 4, 3)
    A = O.amp_s(pol, masks, cfg, li, mi, 4, 3, cfg.kx0 + 0.002, cfg.ky0)
    B = _eigen_free_amp(pol, masks, cfg, li, mi, 4, 3, cfg.kx0 + 0.002, cfg.ky0)
    assert set(B) <= set(A)
    for key in B:
        assert rel_err(B[key], A[key]) < 1e-10


def test_pin_summary_within_print_precision():
    """The oracle was run once at the reference configuration (N=8705) by
    oracle/pin_golden.py; its errors against emint.csv / inputxx.csv are kept."""
    p = os.path.join(GOLDEN, "pin_summary.json")
    if not os.path.exists(p):
        pytest.skip("pin not run yet")
    s = json.load(open(p))
    assert s["inputlm_equal"]
    assert s["emint_max_abs_err_over_max"] < 2e-6  # print precision of emint.csv
    # inputxx: the golden run read undefined memory for one mask row of the thin
    # mask and of the uniform-mask solves; what is reproducible agrees to:
    assert s["a0_max_abs_err_over_max"] < 4e-3
    assert s["ax_max_abs_err_over_max"] < 1e-3 and s["ay_max_abs_err_over_max"] < 1e-3
    assert s["a0_median_abs_err"] < 5e-6


@pytest.mark.parametrize("pol", ["X", "Y"])
def test_abbe_fields_array_form_equals_pupil_loop(pol):
    """The oracle's Abbe fields, written as array operations over the pupil
    points, equal the point-by-point loop of intensity.cpp:276-366."""
    from euvlitho_b200.config import preset
    from tests.helpers import to_oracle
    cfg = preset("small")
    oc = to_oracle(cfg)
    m = flat_bits(random_mask(cfg.ndivx, cfg.ndivy, seed=5))
    L, M = cfg.order_limits()
    li, mi = O.order_set(cfg.order_kind, L, M)
    nd, fams = O.source(oc)
    lin, mn, _, _ = O.pupil_set(oc)
    for (nsx, nsy), pts in fams.items():
        if not pts:
            continue
        sx0 = 2 * O.PI / oc.dx * nsx / nd + oc.kx0
        sy0 = 2 * O.PI / oc.dy * nsy / nd + oc.ky0
        Ax = O.amp_s(pol, m, oc, li, mi, L, M, sx0, sy0, source_orders=pts)
        a = O.abbe_family_fields(oc, pol, Ax, li, mi, nsx, nsy, nd, pts, lin, mn, 20)
        b = O._abbe_family_fields_loop(oc, pol, Ax, li, mi, nsx, nsy, nd, pts, lin, mn, 20)
        for x, y in zip(a, b):
            assert np.max(np.abs(x - y)) <= 1e-13 * max(1.0, np.max(np.abs(y)))
