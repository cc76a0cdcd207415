"""Linear Abbe model on the GPU (euv_linear_amp + euv_abbe through the C ABI)
against the oracle's restatement of cnn/intensity/linear/linear.py, and at the
reference configuration against the images of the reference's own int_linear."""
import gzip
import os

import numpy as np
import pytest

from euvlitho_b200 import io
from euvlitho_b200.config import SimConfig
from oracle import euv_oracle as O
from tests.helpers import random_mask, packed, to_oracle

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("obsc,z", [(0.0, 0), (0.2, 30)])
def test_linear_images_match_the_oracle(cuda, obsc, z):
    import torch
    from euvlitho_b200.engine import Plan
    # reference optics on a 512 nm clip (the narrow order set of the uniform
    # solves needs it, as in m3d.cpp)
    cfg = SimConfig(ndivx=512, ndivy=512, obscuration=obsc, z=z)
    oc = to_oracle(cfg)
    plan = Plan(cfg, device=cuda)
    rng = np.random.default_rng(5)
    ncut = plan.ncut
    masks = [random_mask(cfg.ndivx, cfg.ndivy, s) for s in (1, 2)]
    par = [(rng.standard_normal((2, ncut)) + 1j * rng.standard_normal((2, ncut))) * 1e-3
           for _ in range(3)]
    par[1][:, plan.xinput == 0] = 0
    par[2][:, plan.xinput == 0] = 0
    bits = torch.from_numpy(np.stack([packed(m) for m in masks]))
    lin, ft = plan.linear(bits, *par)
    tb = plan.linear_tables()
    for c in range(2):
        alin, athin = O.linear_amplitudes(oc, masks[c].reshape(-1), par[0][c], par[1][c], par[2][c],
                                          tb["amp_vc"], tb["amp_ab"], tb["dsx"], tb["dsy"],
                                          plan.linput, plan.minput)
        for got, amp in ((lin[c], alin), (ft[c], athin)):
            want = O.linear_image(oc, amp, tb["dsx"], tb["dsy"], plan.linput, plan.minput,
                                  z=float(z), obscuration=obsc)
            err = np.max(np.abs(got.cpu().numpy() - want)) / np.max(want)
            assert err < 1e-10, err


@pytest.mark.slow
def test_reference_config_matches_the_reference_linear_model(cuda):
    """Shipped mask + inputxx.csv at the reference configuration against
    ref_linear.npz (float32 images of the reference's int_linear)."""
    import torch
    from euvlitho_b200.engine import Plan
    p = os.path.join(GOLDEN, "ref_linear.npz")
    if not os.path.exists(p):
        pytest.skip("ref_linear.npz not generated")
    g = np.load(p)
    cfg = SimConfig()
    plan = Plan(cfg, device=cuda)
    with gzip.open(os.path.join(GOLDEN, "ref_mask.bin.gz")) as fh:
        bits = np.frombuffer(fh.read(), np.uint8).copy()
    with gzip.open(os.path.join(GOLDEN, "ref_inputxx.csv.gz"), "rt") as fh:
        xx = io.read_inputxx(fh)
    ax = io.expand_xinput(xx["ax"], plan.xinput)
    ay = io.expand_xinput(xx["ay"], plan.xinput)
    lin, ft = plan.linear(torch.from_numpy(bits)[None], xx["a0"][None], ax[None], ay[None])
    tb = plan.linear_tables()
    assert abs(tb["amp_vc"] - complex(g["ampvc"])) < 1e-7 * abs(tb["amp_vc"])
    for got, name in ((lin[0], "intlinear"), (ft[0], "intft")):
        ref = g[name].astype(np.float64)
        err = np.max(np.abs(got.cpu().numpy() - ref)) / np.max(ref)
        assert err < 2e-7, (name, err)
