"""The C plan's configuration tables against the Python host tables (CPU).

euv_plan_create builds, in C++, the tables the reference drivers compute
before their loops (order/pupil/source sets, rotate() E-field factors and
the orders each pupil point reads, the M3D pairs); the Python host
(euvlitho_b200.tables) builds the same tables for the torch-based engine.
Both follow intensity.cpp / m3d.cpp; here they must agree: index tables
exactly, E-field factors to rounding.  Nothing is launched on a GPU."""
import ctypes as C

import numpy as np
import pytest

from euvlitho_b200 import _lib as L
from euvlitho_b200 import build
from euvlitho_b200 import tables as T
from euvlitho_b200.config import SimConfig, preset


@pytest.fixture(scope="module")
def lib():
    build.build()
    return L.lib()


def _plan(lib, cfg, pols):
    p = C.c_void_p()
    c = L.config_struct(cfg, pols)
    rc = lib.euv_plan_create(C.byref(c), C.byref(p))
    assert rc == 0, lib.euv_last_error()
    info = L.PlanInfo()
    assert lib.euv_plan_get_info(p, C.byref(info)) == 0
    return p, info


def _arr(n, dtype=np.int32):
    return np.zeros(n, dtype)


CONFIGS = [
    ("small", preset("small"), ("X", "Y")),
    ("batched", preset("batched"), ("X", "Y")),
    ("mixed", preset("mixed"), ("X",)),
    ("large", preset("large"), ("X", "Y")),
    ("reference", SimConfig(), ("X",)),
    ("ellipse-512", SimConfig(ndivx=512, ndivy=512, order_kind="ellipse", cut=3.0), ("Y",)),
    ("xdipole-defocus", preset("small").with_(illum_type=2, openangle=60.0, z=40), ("X", "Y")),
    ("ydipole", preset("small").with_(illum_type=3, ndivs=3), ("Y",)),
    ("conventional", preset("small").with_(illum_type=0, sigma1=0.5, ndivs=1), ("X",)),
]


@pytest.mark.parametrize("name,cfg,pols", CONFIGS, ids=[c[0] for c in CONFIGS])
def test_plan_tables_match_python_tables(lib, name, cfg, pols):
    p, info = _plan(lib, cfg, pols)
    try:
        Lm, Mm = cfg.order_limits()
        li, mi = T.order_set(cfg.order_kind, Lm, Mm)
        assert (info.n_orders, info.lmax, info.mmax) == (len(li), Lm, Mm)
        gl, gm = _arr(info.n_orders), _arr(info.n_orders)
        lib.euv_plan_get_orders(p, gl.ctypes.data, gm.ctypes.data)
        assert np.array_equal(gl, li) and np.array_equal(gm, mi)
        lin, mn, xin, _ = T.pupil_set(cfg)
        assert (info.ncut, info.lpx, info.lpy) == (len(lin), cfg.lpmaxX, cfg.lpmaxY)
        pl, pm, px = _arr(info.ncut), _arr(info.ncut), _arr(info.ncut)
        lib.euv_plan_get_pupil(p, pl.ctypes.data, pm.ctypes.data, px.ctypes.data)
        assert np.array_equal(pl, lin) and np.array_equal(pm, mn) and np.array_equal(px, xin)
        ndivs, fams = T.sources(cfg)
        assert (info.ndivs, info.n_families) == (ndivs, len(fams))
        assert info.sdivsum == sum(len(f.pts) for f in fams)
        nsx, nsy, cnt = _arr(info.n_families), _arr(info.n_families), _arr(info.n_families)
        sl, sm = _arr(info.sdivsum), _arr(info.sdivsum)
        lib.euv_plan_get_sources(p, nsx.ctypes.data, nsy.ctypes.data, cnt.ctypes.data,
                                 sl.ctypes.data, sm.ctypes.data)
        o = 0
        for f, a, b, n in zip(fams, nsx, nsy, cnt):
            assert (f.nsx, f.nsy, len(f.pts)) == (a, b, n)
            assert [tuple(x) for x in zip(sl[o:o + n], sm[o:o + n])] == f.pts
            o += n
        na = T.na_sources(cfg)
        nl, nm = _arr(info.n_na_sources), _arr(info.n_na_sources)
        lib.euv_plan_get_na_sources(p, nl.ctypes.data, nm.ctypes.data)
        assert list(zip(nl.tolist(), nm.tolist())) == na
        assert abs(info.k - cfg.k) < 1e-15 and abs(info.kx0 - cfg.kx0) < 1e-15
        assert abs(info.ky0 - cfg.ky0) < 1e-15 and abs(info.z0 - cfg.z0) < 1e-12
        assert (info.xdiv, info.ydiv) == (cfg.xdiv, cfg.ydiv)
        # Abbe tables: t = polarisation index * families + family
        pos = T.order_positions(li, mi)
        ns = info.n_src_max
        assert ns == max(len(f.pts) for f in fams)
        t = 0
        for pol in pols:
            for f in fams:
                coef, nidx = T.abbe_table(cfg, pol, ndivs, f, pos, lin, mn, ns)
                gc = np.zeros((ns, info.ncut, 3), np.complex128)
                gn = np.zeros((ns, info.ncut), np.int32)
                assert lib.euv_plan_get_abbe_table(p, t, gc.ctypes.data, gn.ctypes.data) == 0
                assert np.array_equal(gn, nidx), (pol, f.nsx, f.nsy)
                scale = max(np.abs(coef).max(), 1e-300)
                assert np.abs(gc - coef).max() <= 1e-13 * scale, (pol, f.nsx, f.nsy)
                t += 1
        assert info.units_per_clip == t
    finally:
        lib.euv_plan_destroy(p)


def test_plan_narrow_set_of_m3d(lib):
    """m3d.cpp's narrow order set (ellipse, cut 1.5) at the reference
    configuration: 1009 orders."""
    p, info = _plan(lib, SimConfig(), ("X",))
    try:
        assert info.n_orders == 8705 and info.n_orders_narrow == 1009 and info.ncut == 1901
    finally:
        lib.euv_plan_destroy(p)


def test_reference_config_defaults_match_simconfig(lib):
    c = L.Config()
    lib.euv_config_reference(C.byref(c))
    want = L.config_struct(SimConfig(), ("X",))
    for name, _ in L.Config._fields_:
        a, b = getattr(c, name), getattr(want, name)
        if name in ("eabs", "dabs"):
            for n in range(c.n_slices):
                av, bv = a[n], b[n]
                if name == "eabs":
                    assert abs(complex(av.re, av.im) - complex(bv.re, bv.im)) < 1e-15
                else:
                    assert av == bv
        elif name == "stack":
            for fn, _ in L.Stack._fields_:
                x, y = getattr(a, fn), getattr(b, fn)
                if isinstance(x, L.c64):
                    assert abs(complex(x.re, x.im) - complex(y.re, y.im)) < 1e-15, fn
                else:
                    assert x == y, fn
        elif name == "pols":
            assert a[0] == b[0]
        else:
            assert a == b, name


@pytest.mark.parametrize("bad", [
    dict(lbox=40, mbox=40, order_kind="box", ndivx=256, ndivy=256),   # evanescent orders
    dict(ndivx=250),                                                  # not a multiple of MX
    dict(sigma1=0.01, sigma2=0.009),                                  # no source point
])
def test_plan_rejects_invalid_configurations(lib, bad):
    cfg = preset("small").with_(**bad)
    p = C.c_void_p()
    c = L.config_struct(cfg, ("X",))
    assert lib.euv_plan_create(C.byref(c), C.byref(p)) == L.EUV_ERR_BAD_ARG
    assert not p.value
    assert lib.euv_last_error()


@pytest.mark.parametrize("name,cfg,pols", CONFIGS[:4], ids=[c[0] for c in CONFIGS[:4]])
def test_plan_workspaces_hold_the_batched_solve(lib, name, cfg, pols):
    """The run functions' workspace queries include the batched ampS scratch
    (twelve N x N complex blocks per unit) on top of spectra and amplitudes."""
    p, info = _plan(lib, cfg, pols)
    try:
        N = info.n_orders
        for clips in (1, 3):
            U = clips * info.units_per_clip
            need = 12 * N * N * 16 * U
            assert lib.euv_plan_intensity_workspace_bytes(p, clips, 1) > need
            assert lib.euv_plan_amp_workspace_bytes(p, clips, 1) > 12 * N * N * 16 * clips
            assert lib.euv_plan_m3d_workspace_bytes(p, clips, 1) > 12 * N * N * 16 * clips
    finally:
        lib.euv_plan_destroy(p)
