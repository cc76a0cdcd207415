"""Host-side tables of the product against the oracle (CPU)."""
import numpy as np
import pytest

from euvlitho_b200 import tables as T
from euvlitho_b200.config import SimConfig, preset
from oracle import euv_oracle as O
from tests.helpers import to_oracle

CFGS = ["reference", "small", "batched", "mixed"]


@pytest.mark.parametrize("kind,L,M", [("diamond", 75, 75), ("ellipse", 18, 18), ("box", 5, 7), ("diamond", 3, 9)])
def test_order_sets(kind, L, M):
    a = T.order_set(kind, L, M)
    b = O.order_set(kind, L, M)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


@pytest.mark.parametrize("name", CFGS)
def test_pupil_and_sources(name):
    cfg = preset(name)
    oc = to_oracle(cfg)
    lin, mn, xin, sn = T.pupil_set(cfg)
    olin, omn, oxin, osn = O.pupil_set(oc)
    assert np.array_equal(lin, olin) and np.array_equal(mn, omn) and np.array_equal(xin, oxin)
    nd, fams = T.sources(cfg)
    ond, ofams = O.source(oc)
    assert nd == ond
    assert [(f.nsx, f.nsy, f.pts) for f in fams] == [(k[0], k[1], v) for k, v in ofams.items() if v]


def test_preset_sizes():
    # sizes of the measured workloads
    small, batched, large = preset("small"), preset("batched"), preset("large")
    assert len(T.order_set("box", 5, 5)[0]) == 121
    assert sum(len(f.pts) for f in T.sources(small)[1]) == 26
    assert sum(len(f.pts) for f in T.sources(batched)[1]) == 200
    assert len(T.order_set("box", 15, 15)[0]) == 961 and len(T.order_set("box", 20, 20)[0]) == 1681
    assert (small.xdiv, small.ydiv) == (64, 32)


def test_rotate_matches_oracle():
    rng = np.random.default_rng(1)
    k = 2 * np.pi / 13.5
    px = rng.uniform(-0.05, 0.05, 20)
    py = rng.uniform(-0.03, 0.03, 20)
    px[0] = py[0] = 0.0
    R = T.rotate(k, 4, 8, px, py, 0.0, -0.0486)
    for i in range(20):
        assert np.allclose(R[i], O.rotate(k, 4, 8, px[i], py[i], 0.0, -0.0486), atol=1e-15)


@pytest.mark.parametrize("pol", ["X", "Y"])
def test_abbe_tables_match_oracle_fields(pol):
    cfg = preset("small")
    oc = to_oracle(cfg)
    L, M = cfg.order_limits()
    li, mi = T.order_set("box", L, M)
    pos = T.order_positions(li, mi)
    lin, mn, _, _ = T.pupil_set(cfg)
    nd, fams = T.sources(cfg)
    rng = np.random.default_rng(2)
    for f in fams:
        coef, nidx = T.abbe_table(cfg, pol, nd, f, pos, lin, mn, len(f.pts))
        Ax = {p: rng.standard_normal(len(li)) + 1j * rng.standard_normal(len(li)) for p in f.pts}
        F = O.abbe_family_fields(oc, pol, Ax, li, mi, f.nsx, f.nsy, nd, f.pts, lin, mn, cfg.z)
        for s, p in enumerate(f.pts):
            G = np.zeros_like(F[s])
            for i in range(len(lin)):
                if nidx[s, i] >= 0:
                    G[:, lin[i] % cfg.xdiv, mn[i] % cfg.ydiv] = coef[s, i] * Ax[p][nidx[s, i]]
            assert np.max(np.abs(G - F[s])) < 1e-13 * max(1.0, np.max(np.abs(F[s])))


def test_io_round_trip(tmp_path):
    from euvlitho_b200 import io
    rng = np.random.default_rng(3)
    m = (rng.random((16, 24)) < 0.5).astype(np.uint8)
    pk = io.pack_mask(m)
    p = str(tmp_path / "mask.bin")
    io.write_mask_bin(p, pk)
    back = io.read_mask_bin(p, 24, 16)
    assert np.array_equal(io.unpack_mask(back[0], 24, 16), m)
    a0 = rng.standard_normal(5) + 1j * rng.standard_normal(5)
    xin = np.array([1, 0, 1, 1, 0])
    io.write_inputxx(str(tmp_path / "x.csv"), a0, a0 * 2, a0 * 3, xin)
    r = io.read_inputxx(str(tmp_path / "x.csv"))
    assert np.allclose(r["a0"], a0, rtol=1e-5) and np.allclose(r["ax"], 2 * a0[xin == 1], rtol=1e-5)
