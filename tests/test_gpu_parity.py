"""The CUDA path (through the C ABI) against the FP64 oracle on seeded masks.

Tolerance: FP64 form within 1e-8 relative (max |x - x_ref| / max |x_ref| per
output array); the oracle is eigen-based (LAPACK zgeev), the library
eigen-free, so agreement is to rounding of two different algorithms."""
import numpy as np
import pytest

from euvlitho_b200.config import SimConfig, preset
from oracle import euv_oracle as O
from tests.helpers import flat_bits, packed, random_mask, rel_err, to_oracle

pytestmark = pytest.mark.gpu
TOL = 1e-8


def _masks(cfg, seeds, per_slice=False):
    ms = [random_mask(cfg.ndivx, cfg.ndivy, seed=s) for s in seeds]
    if per_slice:
        # sidewall: slice n (0 = top) is eroded by n pixels on each side of every feature
        out = []
        for m in ms:
            sl = []
            for n in range(cfg.nabs):
                e = m.copy()
                for _ in range(n % 3):
                    e = np.minimum(e, np.roll(e, 1, 1)) if _ % 2 == 0 else np.maximum(e, np.roll(e, -1, 0))
                sl.append(e)
            out.append(sl)
        return out
    return ms


def _plan(cfg, cuda, pols=("X",)):
    from euvlitho_b200.engine import Plan
    return Plan(cfg, device=cuda, pols=pols)


@pytest.mark.parametrize("name,pol", [("small", "X"), ("small", "Y"), ("mixed", "X")])
def test_amp_matches_oracle(cuda, name, pol):
    import torch
    cfg = preset(name)
    oc = to_oracle(cfg)
    plan = _plan(cfg, cuda, (pol,))
    ms = _masks(cfg, [1, 2])
    bits = torch.from_numpy(np.stack([packed(m) for m in ms]))
    ax, srcs = plan.amp(bits, polar=pol)
    ax = ax.cpu().numpy()
    L, M = cfg.order_limits()
    for c, m in enumerate(ms):
        ref = O.amp_s(pol, flat_bits(m), oc, plan.orders.lidx, plan.orders.midx, L, M, oc.kx0, oc.ky0)
        for s, key in enumerate(srcs):
            assert rel_err(ax[c, s], ref[key]) < TOL, (c, key)


@pytest.mark.parametrize("refresh", [False, True])
def test_amp_sidewall_slices(cuda, refresh):
    import torch
    cfg = preset("mixed").with_(refresh_sigma=refresh)
    oc = to_oracle(cfg)
    plan = _plan(cfg, cuda)
    sl = _masks(cfg, [5], per_slice=True)[0]
    bits = torch.from_numpy(np.stack([packed(m) for m in sl])[None])
    ax, srcs = plan.amp(bits)
    ax = ax.cpu().numpy()
    L, M = cfg.order_limits()
    ref = O.amp_s("X", [flat_bits(m) for m in sl], oc, plan.orders.lidx, plan.orders.midx, L, M,
                  oc.kx0, oc.ky0)
    for s, key in enumerate(srcs):
        assert rel_err(ax[0, s], ref[key]) < TOL, key


def test_amp_diamond_orders_na033(cuda):
    import torch
    cfg = SimConfig(ndivx=512, ndivy=512)  # reference optics on a 512 nm clip (N=545)
    oc = to_oracle(cfg)
    plan = _plan(cfg, cuda)
    m = random_mask(512, 512, seed=9)
    ax, srcs = plan.amp(torch.from_numpy(packed(m)[None]))
    L, M = cfg.order_limits()
    ref = O.amp_s("X", flat_bits(m), oc, plan.orders.lidx, plan.orders.midx, L, M, oc.kx0, oc.ky0)
    ax = ax.cpu().numpy()
    for s, key in enumerate(srcs):
        assert rel_err(ax[0, s], ref[key]) < TOL


@pytest.mark.parametrize("pols", [("X",), ("X", "Y")])
def test_intensity_matches_oracle(cuda, pols):
    import torch
    cfg = preset("small")
    oc = to_oracle(cfg)
    plan = _plan(cfg, cuda, pols)
    ms = _masks(cfg, [3, 4])
    img = plan.intensity(torch.from_numpy(np.stack([packed(m) for m in ms]))).cpu().numpy()
    for c, m in enumerate(ms):
        ref = O.intensity(oc, flat_bits(m), polars=pols)
        for p, pol in enumerate(pols):
            assert rel_err(img[c, p], ref[pol]) < TOL


@pytest.mark.parametrize("ndivx,ndivy", [(232, 256), (264, 256), (300, 256), (304, 256), (352, 256),
                                         (400, 256), (256, 264), (256, 288), (256, 320), (256, 416),
                                         (256, 512)])
def test_intensity_image_sizes(cuda, ndivx, ndivy):
    """Image sizes XDIV x YDIV = NDIVX/4 x NDIVY/8.  Widths 58, 66, 75 take the
    one-column-per-thread x stage; 76, 88, 100 the four-way split (XDIV and
    YDIV divisible by 4) with pupil half-widths 6, 7, 8 (every residue mod 4
    with the default's 5); heights 33 (no split), 36, 40, 52, 64 (split y
    stage, a CTA's rows Y/4 apart, pupil half-heights 2, 3, 4, 5)."""
    import torch
    cfg = preset("small").with_(ndivx=ndivx, ndivy=ndivy)
    oc = to_oracle(cfg)
    plan = _plan(cfg, cuda)
    m = random_mask(cfg.ndivx, cfg.ndivy, seed=ndivx + ndivy)
    img = plan.intensity(torch.from_numpy(packed(m)[None])).cpu().numpy()
    ref = O.intensity(oc, flat_bits(m), polars=("X",))
    assert rel_err(img[0, 0], ref["X"]) < TOL


def test_intensity_same_alone_and_batched(cuda):
    """A clip's image does not depend on the other clips in the launch."""
    import torch
    cfg = preset("small")
    plan = _plan(cfg, cuda)
    ms = _masks(cfg, [11, 12, 13])
    allb = plan.intensity(torch.from_numpy(np.stack([packed(m) for m in ms]))).cpu().numpy()
    one = plan.intensity(torch.from_numpy(packed(ms[1])[None])).cpu().numpy()
    assert rel_err(one[0], allb[1]) < 1e-13


def test_m3d_matches_oracle(cuda):
    import torch
    cfg = SimConfig(ndivx=512, ndivy=512)  # reference m3d optics on a 512 nm clip
    oc = to_oracle(cfg)
    plan = _plan(cfg, cuda)
    m = random_mask(512, 512, seed=21)
    res = plan.m3d(torch.from_numpy(packed(m)[None]))
    ref = O.m3d(oc, flat_bits(m))
    xin = plan.xinput == 1
    assert np.array_equal(ref["xinput"], plan.xinput)
    assert rel_err(res["a0"][0].cpu().numpy(), ref["a0"]) < TOL
    if xin.any():
        assert rel_err(res["ax"][0].cpu().numpy()[xin], ref["ax"]) < 1e-7
        assert rel_err(res["ay"][0].cpu().numpy()[xin], ref["ay"]) < 1e-7


@pytest.mark.parametrize("name", ["small", "mixed"])
def test_mixed_precision_intensity_within_1e4(cuda, name):
    """North-star bar of the mixed form: intensity within 1e-4 of the FP64 oracle."""
    import torch
    from euvlitho_b200.engine import Plan
    cfg = preset(name)
    oc = to_oracle(cfg)
    plan = Plan(cfg, device=cuda, pols=("X", "Y"), precision="mixed")
    ms = _masks(cfg, [31, 32])
    img = plan.intensity(torch.from_numpy(np.stack([packed(m) for m in ms]))).cpu().numpy()
    for c, m in enumerate(ms):
        ref = O.intensity(oc, flat_bits(m), polars=("X", "Y"))
        for p, pol in enumerate(("X", "Y")):
            assert rel_err(img[c, p], ref[pol]) < 1e-4


# Mixed form, outputs other than the image: the amplitudes and the M3D
# parameters against the FP64 oracle, max |x - x_ref| / max |x_ref| per array.
MIXED_AMP_TOL = 1e-4


@pytest.mark.parametrize("name", ["small", "mixed"])
def test_mixed_precision_amplitudes(cuda, name):
    import torch
    from euvlitho_b200.engine import Plan
    cfg = preset(name)
    oc = to_oracle(cfg)
    plan = Plan(cfg, device=cuda, pols=("X",), precision="mixed")
    ms = _masks(cfg, [41, 42])
    ax, srcs = plan.amp(torch.from_numpy(np.stack([packed(m) for m in ms])), polar="X")
    ax = ax.cpu().numpy()
    L, M = cfg.order_limits()
    worst = 0.0
    for c, m in enumerate(ms):
        ref = O.amp_s("X", flat_bits(m), oc, plan.orders.lidx, plan.orders.midx, L, M, oc.kx0, oc.ky0)
        for s, key in enumerate(srcs):
            worst = max(worst, rel_err(ax[c, s], ref[key]))
    print("mixed amplitudes %s: max rel err %.2e" % (name, worst))
    assert worst < MIXED_AMP_TOL


@pytest.mark.parametrize("refresh", [False, True])
def test_mixed_precision_sidewall_slices(cuda, refresh):
    """Mixed form through several absorber slices, with the bottom slice's
    sigma for all of them and with each slice's own."""
    import torch
    from euvlitho_b200.engine import Plan
    cfg = preset("mixed").with_(refresh_sigma=refresh)
    oc = to_oracle(cfg)
    plan = Plan(cfg, device=cuda, pols=("X",), precision="mixed")
    sl = _masks(cfg, [7], per_slice=True)[0]
    ax, srcs = plan.amp(torch.from_numpy(np.stack([packed(m) for m in sl])[None]))
    ax = ax.cpu().numpy()
    L, M = cfg.order_limits()
    ref = O.amp_s("X", [flat_bits(m) for m in sl], oc, plan.orders.lidx, plan.orders.midx, L, M,
                  oc.kx0, oc.ky0)
    worst = max(rel_err(ax[0, s], ref[key]) for s, key in enumerate(srcs))
    print("mixed sidewall slices (refresh %s): max rel err %.2e" % (refresh, worst))
    assert worst < MIXED_AMP_TOL


# M3D parameters of the mixed form: ax, ay are least-squares slopes over the
# sources that see a pupil order, and a slope can vanish (ax is ~1e-15 on this
# clip: no x tilt of the chief ray), so every parameter's error is measured
# against the scale of a0; the fit amplifies amplitude errors about 5-10x
# (1e-5 noise on the oracle's amplitudes gives 5e-5 on a0, 1e-4 on ay), yet
# the mixed form stays within the image's 1e-4 bar here.
MIXED_M3D_TOL = 1e-4


def test_mixed_precision_m3d_parameters(cuda):
    import torch
    from euvlitho_b200.engine import Plan
    cfg = SimConfig(ndivx=512, ndivy=512)
    oc = to_oracle(cfg)
    plan = Plan(cfg, device=cuda, pols=("X",), precision="mixed")
    m = random_mask(512, 512, seed=43)
    res = plan.m3d(torch.from_numpy(packed(m)[None]))
    ref = O.m3d(oc, flat_bits(m))
    xin = plan.xinput == 1
    scale = np.max(np.abs(ref["a0"]))
    errs = {"a0": np.max(np.abs(res["a0"][0].cpu().numpy() - ref["a0"])) / scale}
    if xin.any():
        for k in ("ax", "ay"):
            errs[k] = np.max(np.abs(res[k][0].cpu().numpy()[xin] - ref[k])) / scale
    print("mixed M3D parameters (max abs err / max |a0|): " +
          ", ".join("%s %.2e" % kv for kv in errs.items()))
    for k, e in errs.items():
        assert e < MIXED_M3D_TOL, (k, e)
